"""Parity at the benchmark's sizes.

  * 1200-atom LJ system on the 480x480x240 grid (the headline workload): the
    GPU grid against the FP64 oracle pair sums on 2e5 sampled nodes -- 1e5
    uniform over the grid and 1e5 in the z-band the scan reaches (the tip's
    z-range +-1 A) -- with the grid-build tolerance of the other tests
    (|gpu - fp64| <= 2e-5 |ref| + 2e-6 max|ref| + 1e-5 S + 16 |F| delta / r per
    channel: S the node's sum of the atoms' contribution magnitudes -- FP32
    sums err in proportion to S, which the slab's alternating charges make
    100-1000x the value -- and the last term the float32 rounding delta of
    the node position seen at distance r from the nearest atom); then the whole
    480x480-pixel x 60-z-step relaxation on that GPU grid, bit-identical to the
    canonical-FP32 oracle on the same grid, and the df of every column within
    rtol 1e-6 of the oracle's;
  * the 38-atom workload (200^3 grid, 100x100 pixels x 40 z-steps): the whole
    scan bit-identical to the FP32 oracle;
  * LJ beyond one 256-atom shared-memory tile, against the FP64 oracle;
  * the Morse-vs-LJ relation of the reference's own gate
    (tests/SPM/test_afm_morse.py:276-303) through the drop-in AFMulator: raw Fz
    scans of the two pair laws correlated (r > 0.3) but different
    (RMSE > 1e-3 of the peak).
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from spammm_b200 import AFM, gpu, synthetic
from spammm_b200.AFM import AFMulator

pytestmark = pytest.mark.gpu

GRID_TOL_REL, GRID_TOL_ABS = 2e-5, 2e-6
# A node value is a sum over every atom; FP32 rounding (and the MUFU rsqrt) errs in proportion to the
# sum of the contributions' magnitudes S, which on an ionic slab exceeds the value 100-1000x (alternating
# +-0.8 e charges cancel).  Bound: |gpu - fp64| <= 2e-5 |ref| + 2e-6 max|ref| + GRID_TOL_SUM * S.
GRID_TOL_SUM = 1e-5


def pos_term(q, atoms, ref):
    """Error bound of FP32 node positions: the kernel forms node coordinates in float32 (rounded by up to
    ulp(|x|)/2), so dp = node - atom carries an absolute error delta ~ 2^-24 |x|; the pair law varies on the
    scale of the distance r to the nearest atom (the LJ force as r^-13), so a node value can move by
    ~16 |F| delta / r -- O(1) of a component that is small against the others at a node 0.02 A from an
    atom (deep in the |E| > 100 cap)."""
    from scipy.spatial import cKDTree
    r = cKDTree(np.asarray(atoms, np.float64)[:, :3]).query(q)[0]
    delta = 2.0 ** -24 * max(float(np.abs(q).max()), float(np.abs(np.asarray(atoms)[:, :3]).max()))
    F = np.linalg.norm(ref[:, :3], axis=1)
    return (16.0 * delta * F / np.maximum(r, 1e-3))[:, None]


def _check_sampled_grid(got, ref, S, what, P=0.0):
    scale = np.abs(ref).max(axis=0)
    err = np.abs(got - ref)
    bad = err > GRID_TOL_REL * np.abs(ref) + GRID_TOL_ABS * scale + GRID_TOL_SUM * S + P
    print(f"\n{what}: max |gpu-fp64| / max|ref| per channel {(err.max(axis=0) / scale).round(9).tolist()}, "
          f"max |gpu-fp64| / S {float((err / np.maximum(S, 1e-300)).max()):.2e}")
    assert not bad.any(), f"{what}: {bad.sum()} of {bad.size} values out of tolerance"


def _vectors(cfg):
    s = cfg.step
    return (np.array([*cfg.origin, 0], np.float32), np.array([s, 0, 0, 0], np.float32),
            np.array([0, s, 0, 0], np.float32), np.array([0, 0, s, 0], np.float32))


def _points(cfg):
    gx, gy = np.meshgrid(cfg.scan_xs, cfg.scan_ys, indexing="ij")
    pts = np.zeros((cfg.n_pix, 4), np.float32)
    pts[:, 0], pts[:, 1], pts[:, 2] = gx.ravel(), gy.ravel(), np.float32(cfg.z_top)
    return pts


def _scan_params(cfg):
    from spammm_b200 import _lib
    L = np.array(cfg.ngrid) * cfg.step
    dinv = AFMulator._make_dinv_axis_aligned(L, np.asarray(cfg.origin, np.float32), cfg.ngrid)
    P = _lib.make_scan_params(dinv=dinv, dTip=[0, 0, -cfg.dz, 0], stiffness=cfg.stiffness, dpos0=cfg.dpos0,
                              relax_params=[0.5, 0.1, 0.02, 0.5], nz=cfg.nz, max_iter=cfg.max_iter,
                              f2conv=cfg.f2conv, flip_z=True, raster_ny=len(cfg.scan_ys))
    return dinv, P


def _fp64_nodes(cfg, idx):
    """FP64 grid values (capped as the kernels cap) at flattened node indices idx, and the sums of the
    contributions' magnitudes S (scaled by the same cap factor)."""
    nx, ny, _ = cfg.ngrid
    ix, iy, iz = idx % nx, (idx // nx) % ny, idx // (nx * ny)
    p0, dA, dB, dC = (v.astype(np.float64) for v in _vectors(cfg))
    q = np.stack([p0[0] + ix * dA[0], p0[1] + iy * dB[1], p0[2] + iz * dC[2]], 1)
    a64, p64 = cfg.atoms.astype(np.float64), cfg.params.astype(np.float64)
    ref = O.pair_fe(cfg.kind, a64, p64, q, cfg.tipQs, cfg.tipQZs)
    S = O.pair_fe_abs(cfg.kind, a64, p64, q, cfg.tipQs, cfg.tipQZs)
    scale = np.minimum(1.0, 100.0 / np.abs(ref[:, 3]))
    ref = ref * scale[:, None]
    return ref, S * scale[:, None], pos_term(q, a64, ref)


def test_headline_workload_grid_and_full_scan(cuda):
    cfg = synthetic.plain_large()
    p0, dA, dB, dC = _vectors(cfg)
    grid = gpu.grid_build(cfg.kind, cfg.atoms, cfg.params, cfg.ngrid, p0, dA, dB, dC, cfg.tipQs, cfg.tipQZs)
    nx, ny, nzg = cfg.ngrid
    rng = np.random.default_rng(12)
    n_all = nx * ny * nzg
    # the z-band the probe reaches: tip heights z_top .. z_top - (nz-1) dz, +-1 A
    z_hi = cfg.z_top + 1.0
    z_lo = cfg.z_top - (cfg.nz - 1) * cfg.dz - 1.0
    k_lo = int(np.floor((z_lo - cfg.origin[2]) / cfg.step))
    k_hi = int(np.ceil((z_hi - cfg.origin[2]) / cfg.step))
    band = rng.integers(k_lo * nx * ny, (k_hi + 1) * nx * ny, 100000)
    idx = np.concatenate([rng.integers(0, n_all, 100000), band])
    got = grid.view(-1, 4)[torch.from_numpy(idx).cuda()].cpu().numpy().astype(np.float64)
    ref, S, P = _fp64_nodes(cfg, idx)
    _check_sampled_grid(got, ref, S, "1200-atom grid, 2e5 sampled nodes", P)
    # the whole scan on this grid against the FP32 oracle on the same grid
    dinv, P = _scan_params(cfg)
    pts = _points(cfg)
    FEs, disps = gpu.relax_strokes(grid, P, torch.from_numpy(pts).cuda())
    g_host = grid.cpu().numpy()
    del grid
    oFE, oD = O.relax_strokes(g_host, dinv, pts, cfg.nz, [0, 0, -cfg.dz, 0], cfg.stiffness, cfg.dpos0,
                              [0.5, 0.1, 0.02, 0.5], cfg.max_iter, cfg.f2conv, True, True)
    fe_h, d_h = FEs.cpu().numpy(), disps.cpu().numpy()
    n_diff = int((fe_h != oFE).any(axis=-1).sum() + (d_h != oD).any(axis=-1).sum())
    assert n_diff == 0, f"{n_diff} states differ from the FP32 oracle"
    npx = len(cfg.scan_xs)
    spacing = (cfg.step, cfg.step, cfg.dz)
    df = gpu.df_amp_dir(FEs.view(npx, npx, cfg.nz, 4), spacing, (0., 0., 1.), cfg.amp).cpu().numpy()
    odf = O.compute_df_amp_dir(oFE.reshape(npx, npx, cfg.nz, 4), spacing, (0., 0., 1.), cfg.amp)
    np.testing.assert_allclose(df, odf, rtol=1e-6, atol=1e-6 * np.abs(odf).max())


def test_38_atom_workload_full_scan_bit_exact(cuda):
    cfg = synthetic.plain_small()
    p0, dA, dB, dC = _vectors(cfg)
    grid = gpu.grid_build(cfg.kind, cfg.atoms, cfg.params, cfg.ngrid, p0, dA, dB, dC, cfg.tipQs, cfg.tipQZs)
    dinv, P = _scan_params(cfg)
    pts = _points(cfg)
    FEs, disps = gpu.relax_strokes(grid, P, torch.from_numpy(pts).cuda())
    oFE, oD = O.relax_strokes(grid.cpu().numpy(), dinv, pts, cfg.nz, [0, 0, -cfg.dz, 0], cfg.stiffness, cfg.dpos0,
                              [0.5, 0.1, 0.02, 0.5], cfg.max_iter, cfg.f2conv, True, True)
    assert np.array_equal(FEs.cpu().numpy(), oFE) and np.array_equal(disps.cpu().numpy(), oD)
    # and the grid on 1e5 sampled nodes against FP64
    idx = np.random.default_rng(3).integers(0, int(np.prod(cfg.ngrid)), 100000)
    got = grid.view(-1, 4)[torch.from_numpy(idx).cuda()].cpu().numpy().astype(np.float64)
    ref, S, P = _fp64_nodes(cfg, idx)
    _check_sampled_grid(got, ref, S, "38-atom grid, 1e5 sampled nodes", P)


def test_lj_grid_beyond_one_atom_tile(cuda):
    """600 LJ atoms (> one 256-atom shared-memory tile), ragged grid, capped cores."""
    rng = np.random.default_rng(19)
    na = 600
    atoms = np.zeros((na, 4), np.float32)
    atoms[:, :2] = rng.uniform(-6, 6, (na, 2))
    atoms[:, 2] = rng.normal(0, 0.4, na)
    atoms[:, 3] = rng.uniform(-0.3, 0.3, na)
    R0, E0 = rng.uniform(3.0, 3.5, na), rng.uniform(2e-3, 3e-3, na)
    prm = np.stack([2 * E0 * R0 ** 6, E0 * R0 ** 12], 1).astype(np.float32)
    n = (33, 35, 19)
    p0 = np.array([-6, -6, -1.0, 0], np.float32)
    dA, dB, dC = (np.array(v, np.float32) for v in ([0.35, 0, 0, 0], [0, 0.35, 0, 0], [0, 0, 0.35, 0]))
    g = gpu.grid_build(0, atoms, prm, n, p0, dA, dB, dC, [-0.05, 0, 0, 0], [0, 0, 0, 0]).cpu().numpy()
    ref = O.grid_build(0, atoms, prm, n, p0, dA, dB, dC, [-0.05, 0, 0, 0], [0, 0, 0, 0], prec="f64")
    assert np.abs(ref[..., 3]).max() == pytest.approx(100.0)  # the cap is exercised
    iz, iy, ix = np.meshgrid(*(np.arange(k) for k in n[::-1]), indexing="ij")
    q = np.stack([p0[0] + ix * 0.35, p0[1] + iy * 0.35, p0[2] + iz * 0.35], -1).reshape(-1, 3).astype(np.float64)
    raw = O.pair_fe(0, atoms.astype(np.float64), prm.astype(np.float64), q, [-0.05, 0, 0, 0], [0, 0, 0, 0])
    S = O.pair_fe_abs(0, atoms.astype(np.float64), prm.astype(np.float64), q, [-0.05, 0, 0, 0], [0, 0, 0, 0])
    S *= np.minimum(1.0, 100.0 / np.abs(raw[:, 3]))[:, None]
    _check_sampled_grid(g.reshape(-1, 4).astype(np.float64), ref.reshape(-1, 4), S, "600-atom LJ grid",
                        pos_term(q, atoms, ref.reshape(-1, 4)))


def test_morse_and_lj_scans_correlated_but_different(cuda):
    """The reference's Morse-vs-LJ gate (tests/SPM/test_afm_morse.py:276-303) on a benzene-sized ring."""
    pos, Z, q = synthetic.planar_molecule({"C": 6, "H": 6}, 7)
    out = {}
    for morse in (True, False):
        afm = AFMulator(use_morse=morse)
        afm.mol = AFM._Molecule(pos, ["C" if z == 6 else "H" for z in Z], q)
        afm.assign_params()
        afm.setup_grid(n=(50, 50, 30), margin=3.0, z_top=12.0)
        afm.make_forcefield()
        FEs, _ = afm.get_raw_FE(nxy=(30, 30), nz=15, dtip=-0.2)
        assert np.isfinite(FEs).all()
        out[morse] = FEs[..., 2]
    Fm, Fl = out[True], out[False]
    r = np.corrcoef(Fm.ravel(), Fl.ravel())[0, 1]
    rms = np.sqrt(np.mean((Fm - Fl) ** 2))
    peak = max(np.abs(Fm).max(), np.abs(Fl).max())
    print(f"\nMorse vs LJ raw Fz: r = {r:.4f}, RMSE = {rms:.3e}, peak = {peak:.3e}")
    assert r > 0.3
    assert rms > 1e-3 * peak
