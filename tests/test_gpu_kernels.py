"""GPU parity tests: every kernel of libspmb200.so against the oracle and the
reference goldens, through the C ABI (spammm_b200.gpu -> ctypes).

Tolerances (written per test):
  * relaxation paths (relaxStrokes / relaxStrokesTilted / raw sampling) on an
    identical FP32 grid: bit-identical to the canonical-FP32 oracle;
  * grid build (MUFU rsqrt/ex2 fast math): |gpu - fp64| <= 2e-5 |ref| + 2e-6 max|ref| per channel;
  * df / loss / dissipation (FP64 on device): rtol 1e-6 against the reference's own outputs.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from spammm_b200 import _lib, gpu

pytestmark = pytest.mark.gpu


def _mol(na, seed, morse):
    rng = np.random.default_rng(seed)
    atoms = np.zeros((na, 4), np.float32)
    atoms[:, :2] = rng.uniform(-3, 3, (na, 2))
    atoms[:, 2] = rng.normal(0, 0.05, na)
    atoms[:, 3] = rng.uniform(-0.3, 0.3, na)
    if morse:
        prm = np.stack([rng.uniform(3.0, 3.5, na), rng.uniform(2e-3, 3e-3, na), np.full(na, -1.8), np.zeros(na)], 1)
    else:
        R0, E0 = rng.uniform(3.0, 3.5, na), rng.uniform(2e-3, 3e-3, na)
        prm = np.stack([2 * E0 * R0 ** 6, E0 * R0 ** 12], 1)
    return atoms, prm.astype(np.float32)


def _grid_geom(n=(37, 29, 41), step=0.2, origin=(-3.7, -2.9, -2.0)):
    p0 = np.array([*origin, 0], np.float32)
    return n, p0, np.array([step, 0, 0, 0], np.float32), np.array([0, step, 0, 0], np.float32), \
        np.array([0, 0, step, 0], np.float32)


def _check_grid(g, ref):
    scale = np.abs(ref).reshape(-1, 4).max(axis=0)
    err = np.abs(g.astype(np.float64) - ref)
    bad = err > 2e-5 * np.abs(ref) + 2e-6 * scale
    assert not bad.any(), f"{bad.sum()} nodes out of tolerance; worst {err.max():.3e} scale {scale}"


@pytest.mark.parametrize("kind", [0, 1])
@pytest.mark.parametrize("qs", [(0, 0, 0, 0), (-0.05, 0, 0, 0), (0, -0.1, 0.1, 0), (-0.1, 0.05, -0.02, 0.2)])
def test_grid_build_matches_fp64_oracle(cuda, kind, qs):
    atoms, prm = _mol(19, 4 + kind, kind == 1)
    n, p0, dA, dB, dC = _grid_geom()
    QZs = np.array([0.0, 1.8, 3.6, -0.7], np.float32)
    g = gpu.grid_build(kind, atoms, prm, n, p0, dA, dB, dC, np.array(qs, np.float32), QZs).cpu().numpy()
    ref = O.grid_build(kind, atoms, prm, n, p0, dA, dB, dC, qs, QZs, prec="f64")
    assert g.shape == (n[2], n[1], n[0], 4)
    _check_grid(g, ref)


def test_grid_build_many_atoms_and_cap(cuda):
    """> one shared-memory tile of atoms (600), ragged dims, capped cores."""
    atoms, prm = _mol(600, 9, True)
    n, p0, dA, dB, dC = _grid_geom((33, 35, 19), 0.35, (-6, -6, -1.0))
    g = gpu.grid_build(1, atoms, prm, n, p0, dA, dB, dC, [-0.05, 0, 0, 0], [0, 0, 0, 0]).cpu().numpy()
    ref = O.grid_build(1, atoms, prm, n, p0, dA, dB, dC, [-0.05, 0, 0, 0], [0, 0, 0, 0], prec="f64")
    assert np.abs(ref[..., 3]).max() == pytest.approx(100.0)  # the cap is exercised
    _check_grid(g, ref)


def test_grid_build_no_atoms_is_zero(cuda):
    n, p0, dA, dB, dC = _grid_geom((8, 8, 8))
    g = gpu.grid_build(0, np.zeros((0, 4), np.float32), np.zeros((0, 2), np.float32), n, p0, dA, dB, dC,
                       [0, 0, 0, 0], [0, 0, 0, 0])
    assert torch.count_nonzero(g).item() == 0


def test_grid_build_rejects_skewed_dC(cuda):
    n, p0, dA, dB, dC = _grid_geom((8, 8, 8))
    atoms, prm = _mol(3, 1, False)
    with pytest.raises(RuntimeError, match="dC"):
        gpu.grid_build(0, atoms, prm, n, p0, dA, dB, np.array([0.1, 0, 0.2, 0], np.float32), [0] * 4, [0] * 4)


def _relax_setup(seed=0, n_side=11, nz=9):
    atoms, prm = _mol(12, seed, True)
    n, p0, dA, dB, dC = _grid_geom((48, 44, 40), 0.25, (-6.0, -5.5, -3.0))
    grid = gpu.grid_build(1, atoms, prm, n, p0, dA, dB, dC, [-0.05, 0, 0, 0], [0, 0, 0, 0])
    L = np.array(n) * 0.25
    dinv = O.dinv_axis_aligned(L, p0[:3], n)
    rng = np.random.default_rng(seed + 1)
    pts = np.zeros((n_side * (n_side + 2), 4), np.float32)
    pts[:, :2] = rng.uniform(-2.5, 2.5, (pts.shape[0], 2))
    pts[:, 2] = 5.0
    return grid, dinv, pts, nz


@pytest.mark.parametrize("fire", [True, False])
@pytest.mark.parametrize("flip", [False, True])
def test_relax_strokes_bit_exact(cuda, fire, flip):
    grid, dinv, pts, nz = _relax_setup()
    stiff = [-0.0156, -0.0156, -1.248, 0.0]
    relax = [0.5, 0.1, 0, 0] if fire else [0.3, 0.2, 0.03, 0.3]
    for max_iter, f2 in ((128, 1e-8), (1000, 1e-10), (0, 1e-8), (3, 1e-8)):
        P = _lib.make_scan_params(dinv=dinv, dTip=[0, 0, -0.1, 0], stiffness=stiff, dpos0=[0, 0, 0, 0],
                                  relax_params=relax, nz=nz, max_iter=max_iter, f2conv=f2, fire=fire, flip_z=flip,
                                  raster_ny=11 + 2)
        FEs, disps = gpu.relax_strokes(grid, P, torch.from_numpy(pts).cuda())
        oFE, oD = O.relax_strokes(grid.cpu().numpy(), dinv, pts, nz, [0, 0, -0.1, 0], stiff, [0, 0, 0, 0], relax,
                                  max_iter, f2, fire, flip, prec="f32")
        assert np.array_equal(FEs.cpu().numpy(), oFE), f"FEs differ (max_iter={max_iter})"
        assert np.array_equal(disps.cpu().numpy(), oD), f"disps differ (max_iter={max_iter})"


def test_relax_strokes_pixel_mapping_does_not_change_results(cuda):
    grid, dinv, pts, nz = _relax_setup(seed=3)
    kw = dict(dinv=dinv, dTip=[0, 0, -0.1, 0], stiffness=[-0.03, -0.03, -0.5, -1.0], dpos0=[0, 0, -0.5, 0.5],
              relax_params=[0.5, 0.1, 0, 0], nz=nz, max_iter=200, f2conv=1e-9)
    pt = torch.from_numpy(pts).cuda()
    a = gpu.relax_strokes(grid, _lib.make_scan_params(raster_ny=13, **kw), pt)
    b = gpu.relax_strokes(grid, _lib.make_scan_params(raster_ny=0, **kw), pt)
    c = gpu.relax_strokes(grid, _lib.make_scan_params(raster_ny=7, **kw), pt)  # not a divisor: 1-D map
    for x, y in ((a, b), (a, c)):
        assert torch.equal(x[0], y[0]) and torch.equal(x[1], y[1])


def test_relax_dynamic_schedule_is_bit_identical(cuda):
    """Pixel counter (dynamic) vs one-pixel-per-lane (static) schedule, raster and
    1-D maps, strokes and tilted: identical FEs, displacements and step counts."""
    grid, dinv, pts, nz = _relax_setup(seed=8, n_side=23)
    pt = torch.from_numpy(pts).cuda()
    for ny in (25, 0):
        P = _lib.make_scan_params(dinv=dinv, dTip=[0, 0, -0.1, 0], stiffness=[-0.0156, -0.0156, -1.25, 0],
                                  relax_params=[0.5, 0.1, 0.02, 0.5], nz=nz, max_iter=1000, f2conv=1e-10,
                                  flip_z=True, raster_ny=ny)
        ca = torch.empty(pt.shape[0], dtype=torch.int32, device="cuda")
        cb = torch.empty_like(ca)
        a = gpu.relax_strokes(grid, P, pt, iter_count=ca, dynamic=True)
        b = gpu.relax_strokes(grid, P, pt, iter_count=cb, dynamic=False)
        assert torch.equal(a[0], b[0]) and torch.equal(a[1], b[1]) and torch.equal(ca, cb)
        assert int(ca.min()) >= nz
        t1 = gpu.relax_strokes_tilted(grid, P, pt, dynamic=True)
        t2 = gpu.relax_strokes_tilted(grid, P, pt, dynamic=False)
        assert torch.equal(t1, t2)


def test_relax_strokes_empty_and_ragged(cuda):
    grid, dinv, pts, nz = _relax_setup()
    P = _lib.make_scan_params(dinv=dinv, dTip=[0, 0, -0.1, 0], stiffness=[-0.02, -0.02, -1, 0],
                              relax_params=[0.5, 0.1, 0, 0], nz=nz)
    FEs, disps = gpu.relax_strokes(grid, P, torch.zeros((0, 4), device="cuda"))
    assert FEs.shape == (0, nz, 4)
    sub = pts[:5]
    FEs, _ = gpu.relax_strokes(grid, P, torch.from_numpy(sub).cuda())
    oFE, _ = O.relax_strokes(grid.cpu().numpy(), dinv, sub, nz, [0, 0, -0.1, 0], [-0.02, -0.02, -1, 0], [0, 0, 0, 0],
                             [0.5, 0.1, 0, 0])
    assert np.array_equal(FEs.cpu().numpy(), oFE)


def _tip_frame():
    th = 0.3
    a = np.array([np.cos(th), 0, -np.sin(th), 0], np.float32)
    b = np.array([0, 1, 0, 0], np.float32)
    c = np.array([np.sin(th), 0, np.cos(th), -0.1], np.float32)
    return a, b, c


def test_relax_tilted_bit_exact(cuda):
    grid, dinv, pts, nz = _relax_setup(seed=5)
    a, b, c = _tip_frame()
    kw = dict(stiffness=[-0.03, -0.03, -0.03, -1.0], dpos0=[0, 0, -4.0, 4.0], relax_params=[0.5, 0.1, 0.02, 0.5])
    pts2 = pts.copy()
    pts2[:, 2] = 9.0
    P = _lib.make_scan_params(dinv=dinv, tipA=a, tipB=b, tipC=c, surfFF=[0.01, 0, 0, 0], nz=nz, raster_ny=13, **kw)
    FEs = gpu.relax_strokes_tilted(grid, P, torch.from_numpy(pts2).cuda())
    o = O.relax_tilted(grid.cpu().numpy(), dinv, pts2, nz, a, b, c, kw["stiffness"], kw["dpos0"], kw["relax_params"],
                       [0.01, 0, 0, 0])
    assert np.array_equal(FEs.cpu().numpy(), o)


def test_raw_sampling_bit_exact(cuda):
    grid, dinv, pts, nz = _relax_setup(seed=6)
    a, b, c = _tip_frame()
    P = _lib.make_scan_params(dinv=dinv, tipA=a, tipB=b, tipC=c, dTip=[0, 0, -0.2, 0], dpos0=[0.1, 0, -4.0, 4.0],
                              nz=nz)
    FEs = gpu.fe_in_strokes_tilted(grid, P, torch.from_numpy(pts).cuda())
    o = O.raw_tilted(grid.cpu().numpy(), dinv, pts, nz, a, b, c, [0, 0, -0.2, 0], [0.1, 0, -4.0, 4.0])
    assert np.array_equal(FEs.cpu().numpy(), o)


def test_relax_on_reference_grid_vs_reference_fp64_loops(cuda, golden):
    """FP32 kernels on the reference's FP64 Morse grid against the FP64 reference loops."""
    g = golden("gridrelax_golden.npz")
    grid = torch.from_numpy(g["grid"].astype(np.float32)).cuda()
    dinv, pts, nz = g["dinv"].astype(np.float32), g["pts"], int(g["nzs"])
    P = _lib.make_scan_params(dinv=dinv, dTip=g["dTip"], stiffness=g["stiffness"], dpos0=g["dpos0"],
                              relax_params=g["relax"], nz=nz)
    FEs, disps = gpu.relax_strokes(grid, P, torch.from_numpy(pts).cuda())
    FEs, disps = FEs.cpu().numpy(), disps.cpu().numpy()
    scale = np.abs(g["strokes_FEs"]).max()
    # FP32 vs FP64 FIRE at the reference's loose |F|<1e-4: positions agree to ~1e-3 A
    assert np.abs(disps - g["strokes_disps"]).max() < 5e-3
    assert np.abs(FEs - g["strokes_FEs"]).max() < 2e-2 * scale
    Pt = _lib.make_scan_params(dinv=dinv, tipC=g["tipC"], stiffness=g["stiffness"], dpos0=g["dpos0"],
                               relax_params=g["relax"], nz=nz)
    FEt = gpu.relax_strokes_tilted(grid, Pt, torch.from_numpy(pts).cuda()).cpu().numpy()
    assert np.abs(FEt - g["tilted_FEs"]).max() < 2e-2 * scale
    Pr = _lib.make_scan_params(dinv=dinv, dTip=g["dTip"], dpos0=g["dpos0"], nz=nz)
    raw = gpu.fe_in_strokes_tilted(grid, Pr, torch.from_numpy(pts).cuda()).cpu().numpy()
    np.testing.assert_allclose(raw, g["raw_FEs"], rtol=1e-5, atol=1e-6 * scale)


# ---------------------------------------------------------------- stage (c)
def test_df_kernels_match_reference(cuda, golden):
    from spammm_b200 import AFM
    g = golden("df_golden.npz")
    for i in range(int(g["n_cases"])):
        FEs, sp, od, amp = g[f"c{i}_FEs"], g[f"c{i}_spacing"], g[f"c{i}_osc"], float(g[f"c{i}_amp"])
        sp = float(sp) if sp.ndim == 0 else sp
        ref = g[f"c{i}_amp_dir"]
        ours = AFM.compute_df_amp_dir(FEs, sp, od, amp)
        assert ours.dtype == np.float32
        np.testing.assert_allclose(ours, ref, rtol=1e-6, atol=1e-6 * np.abs(ref).max(), err_msg=f"amp case {i}")
        np.testing.assert_allclose(AFM.compute_df_dir(FEs, sp, od), g[f"c{i}_dir"], rtol=1e-6, atol=1e-6)
    np.testing.assert_allclose(AFM.compute_df(g["Fz"], 0.1), g["compute_df"], rtol=1e-6, atol=1e-6)
    np.testing.assert_allclose(AFM.compute_df_amp(g["Fz"], 0.1, 0.6), g["compute_df_amp"], rtol=1e-6, atol=1e-6)


def test_df_z_column_kernel_matches_generic_kernel(cuda):
    """n = z takes the column kernel; n = (1e-300, 0, 1) takes the generic kernel with
    exactly the same arithmetic (the x shift rounds to zero) -> identical bits."""
    rng = np.random.default_rng(11)
    for dt in (np.float32, np.float64):
        FEs = rng.standard_normal((7, 5, 43, 4)).astype(dt)
        a = gpu.df_amp_dir(FEs, (0.1, 0.1, 0.1), (0, 0, 1), 1.0).cpu().numpy()
        b = gpu.df_amp_dir(FEs, (0.1, 0.1, 0.1), (1e-300, 0, 1), 1.0).cpu().numpy()
        assert np.array_equal(a, b)
        a = gpu.df_amp_dir(FEs, (0.1, 0.1, 0.1), (0, 0, -1), 0.37, out_iz=[0, 42, 5]).cpu().numpy()
        b = gpu.df_amp_dir(FEs, (0.1, 0.1, 0.1), (1e-300, 0, -1), 0.37, out_iz=[0, 42, 5]).cpu().numpy()
        assert np.array_equal(a, b)


def test_df_selected_slices(cuda):
    rng = np.random.default_rng(2)
    FEs = rng.standard_normal((9, 8, 31, 4)).astype(np.float32)
    full = gpu.df_amp_dir(FEs, (0.1, 0.1, 0.1), (0, 0, 1), 1.0).cpu().numpy()
    sel = [0, 3, 30, 17]
    part = gpu.df_amp_dir(FEs, (0.1, 0.1, 0.1), (0, 0, 1), 1.0, out_iz=sel).cpu().numpy()
    assert np.array_equal(part, full[:, :, sel])


def test_df_loss_seed_matches_reference(cuda, golden):
    from spammm_b200 import AFM
    g = golden("loss_golden.npz")
    for i in range(int(g["n_cases"])):
        w = g[f"c{i}_w"]
        loss, df, dL = AFM.df_loss_seed(g[f"c{i}_FEs"], g[f"c{i}_tgt"], float(g[f"c{i}_dtip"]), w if w.size else None)
        assert loss == pytest.approx(float(g[f"c{i}_loss"]), rel=1e-12)
        np.testing.assert_allclose(df, g[f"c{i}_df"], rtol=1e-12, atol=1e-12)
        np.testing.assert_allclose(dL, g[f"c{i}_dL"], rtol=1e-6, atol=1e-7 * np.abs(g[f"c{i}_dL"]).max())
    with pytest.raises(ValueError, match="dtip must be"):
        AFM.df_loss_seed(np.zeros((2, 2, 5, 4), np.float32), np.zeros((2, 2, 5)), 0.1)
    with pytest.raises(ValueError, match="nz>=3"):
        AFM.df_loss_seed(np.zeros((2, 2, 2, 4), np.float32), np.zeros((2, 2, 2)), -0.1)


def test_dissipation_and_postprocess_match_reference(cuda, golden):
    from spammm_b200 import AFM, AFM_utils as U
    g = golden("diss_golden.npz")
    E = AFM.compute_dissipation(g["Ff"], g["Fb"], g["h_scan"], g["h_df"], 1.0, (0., 0., 1.))
    np.testing.assert_allclose(E, g["E_z"], rtol=1e-6, atol=1e-7)
    E = AFM.compute_dissipation(g["Ff"], g["Fb"], g["h_scan"], g["h_df"], 0.6, (0.5, 0., 1.))
    np.testing.assert_allclose(E, g["E_t"], rtol=1e-6, atol=1e-7)
    spec = U.ScanSpec(scan_xs=np.arange(4, dtype=np.float32) * 0.1, scan_ys=np.arange(3, dtype=np.float32) * 0.1,
                      h_df=g["h_df"], h_Fz=g["h_Fz"], h_scan=g["h_scan"], amplitude=1.0, osc_dir=(0., 0., 1.),
                      K_LAT=0.03, K_RAD=20.0, bond_length=3.0)
    res = U.shared_postprocess(g["Ff"], spec, FEs_bwd=g["Fb"])
    np.testing.assert_allclose(res.df, g["pp_df"], rtol=1e-6, atol=1e-6 * np.abs(g["pp_df"]).max())
    assert np.array_equal(res.Fz, g["pp_Fz"])
    np.testing.assert_allclose(res.E_diss, g["pp_E"], rtol=1e-6, atol=1e-7)


@pytest.mark.parametrize("nzw", [0, 1, 9, 64, 200])
def test_convolve_z_matches_oracle(cuda, nzw):
    """convolveZ (kernels/AFM.cl:666-701): bit-identical to the canonical-FP32 oracle."""
    rng = np.random.default_rng(nzw)
    nz_in = 230
    F = rng.normal(size=(7, 5, nz_in, 4)).astype(np.float32)
    w = rng.normal(size=nzw).astype(np.float32)
    out = gpu.convolve_z(F, w, nz_in - nzw)
    torch.cuda.synchronize()
    assert out.shape == (7, 5, nz_in - nzw, 4)
    assert np.array_equal(out.cpu().numpy(), O.convolve_z(F, w, nz_in - nzw))


def test_izo_z_matches_oracle(cuda):
    """izoZ (kernels/AFM.cl:705-723): bit-identical to the oracle, including
    columns that never cross, cross at once, hold NaN, and nz = 1."""
    rng = np.random.default_rng(7)
    F = rng.normal(size=(33, 17, 40, 4)).astype(np.float32)
    F[..., 2] = np.cumsum(np.abs(F[..., 2]), axis=-1) * rng.choice([-1.0, 1.0], size=(33, 17, 1)).astype(np.float32)
    F[0, :, :, 2] = np.nan
    F[1, 3, 5, 2] = np.nan
    for iso in (0.0, 3.5, 1e6, -2.0):
        z = gpu.izo_z(F, iso)
        torch.cuda.synchronize()
        assert z.shape == (33, 17)
        np.testing.assert_array_equal(z.cpu().numpy(), O.izo_z(F, iso), err_msg=str(iso))  # NaN == NaN here
    one = np.ones((4, 1, 4), np.float32)
    assert np.array_equal(gpu.izo_z(one, 0.5).cpu().numpy(), np.full(4, -1.0, np.float32))
    with pytest.raises(ValueError, match="weights"):
        gpu.convolve_z(F, np.ones(3, np.float32), 40)


@pytest.mark.parametrize("kind", [0, 1])
def test_pair_fe_points_matches_fp64_oracle(cuda, kind):
    """spm_pair_fe_points (cs_brute_afm_morse_c_points semantics: uncapped) against the FP64 pair sums,
    with the reference gate's bar (tests/SPM/test_afm_morse.py:864-900: rtol 5e-5, atol 1e-5 + 1e-5 scale)."""
    atoms, prm = _mol(40, 17 + kind, kind == 1)
    rng = np.random.default_rng(5)
    q = np.stack([rng.uniform(-4, 4, 3000), rng.uniform(-4, 4, 3000), rng.uniform(0.8, 6.0, 3000)], 1)
    q = q.astype(np.float32)
    Qs, QZs = [-0.05, 0.02, 0, 0], [0, 1.8, 0, 0]
    got = gpu.pair_fe_points(kind, atoms, prm, torch.from_numpy(q).cuda(), Qs, QZs).cpu().numpy()
    ref = O.pair_fe(kind, atoms.astype(np.float64), prm.astype(np.float64), q.astype(np.float64), Qs, QZs)
    for c in range(4):
        scale = float(np.abs(ref[:, c]).max())
        np.testing.assert_allclose(got[:, c], ref[:, c], rtol=5e-5, atol=1e-5 + 1e-5 * scale)
