"""Newton polish of the relaxed states (SPM_FLAG_POLISH) on the GPU against the
canonical-FP32 oracle with the same polish.

The polish is opt-in and not in the reference: after FIRE stops, up to four
Newton steps on the total force of the interpolated grid and the spring take
each state to the equilibrium of the interpolated field.  Bars:
  * relaxStrokes, relaxStrokesTilted and the PP relaxation, under the tile
    (pixel counter) and the flattened (one pixel per lane) schedules:
    bit-identical to the FP32 oracle with the same polish;
  * the FIRE trajectory is unchanged (per-pixel step counts equal to the
    unpolished run), and the polished states have a smaller residual force.
The accuracy against the FP64 oracle at the workload's threshold is in
test_gpu_accuracy.py.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from spammm_b200 import _lib, gpu

from test_gpu_kernels import _relax_setup, _tip_frame

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dynamic", [True, False])
@pytest.mark.parametrize("flip", [False, True])
def test_polished_relax_strokes_bit_exact(cuda, dynamic, flip):
    grid, dinv, pts, nz = _relax_setup(seed=11)
    pt = torch.from_numpy(pts).cuda()
    for stiff, d0 in (([-0.0156, -0.0156, -1.248, 0.0], [0, 0, 0, 0]),
                      ([-0.03, -0.03, -0.03, -1.0], [0, 0, -0.5, 0.5])):  # plain spring, radial bond
        P = _lib.make_scan_params(dinv=dinv, dTip=[0, 0, -0.1, 0], stiffness=stiff, dpos0=d0,
                                  relax_params=[0.5, 0.1, 0.02, 0.5], nz=nz, max_iter=1000, f2conv=1e-10,
                                  flip_z=flip, raster_ny=13, polish=True)
        cnt = torch.empty(pt.shape[0], dtype=torch.int32, device="cuda")
        FEs, disps = gpu.relax_strokes(grid, P, pt, iter_count=cnt, dynamic=dynamic)
        oFE, oD = O.relax_strokes(grid.cpu().numpy(), dinv, pts, nz, [0, 0, -0.1, 0], stiff, d0, [0.5, 0.1, 0.02, 0.5],
                                  1000, 1e-10, True, flip, prec="f32", polish=True)
        assert np.array_equal(FEs.cpu().numpy(), oFE), "polished FEs differ from the oracle"
        assert np.array_equal(disps.cpu().numpy(), oD), "polished displacements differ from the oracle"
        # the FIRE trajectory is the unpolished one
        P0 = _lib.make_scan_params(dinv=dinv, dTip=[0, 0, -0.1, 0], stiffness=stiff, dpos0=d0,
                                   relax_params=[0.5, 0.1, 0.02, 0.5], nz=nz, max_iter=1000, f2conv=1e-10,
                                   flip_z=flip, raster_ny=13)
        cnt0 = torch.empty_like(cnt)
        FE0, D0 = gpu.relax_strokes(grid, P0, pt, iter_count=cnt0, dynamic=dynamic)
        assert torch.equal(cnt, cnt0)
        assert not torch.equal(D0, disps)  # the polish moved the states


def test_polished_relax_tilted_bit_exact(cuda):
    grid, dinv, pts, nz = _relax_setup(seed=12)
    a, b, c = _tip_frame()
    kw = dict(stiffness=[-0.03, -0.03, -0.03, -1.0], dpos0=[0, 0, -4.0, 4.0], relax_params=[0.5, 0.1, 0.02, 0.5])
    pts2 = pts.copy()
    pts2[:, 2] = 9.0
    pt = torch.from_numpy(pts2).cuda()
    o = O.relax_tilted(grid.cpu().numpy(), dinv, pts2, nz, a, b, c, kw["stiffness"], kw["dpos0"], kw["relax_params"],
                       [0.01, 0, 0, 0], 1000, 1e-10, prec="f32", polish=True)
    for dynamic in (True, False):
        P = _lib.make_scan_params(dinv=dinv, tipA=a, tipB=b, tipC=c, surfFF=[0.01, 0, 0, 0], nz=nz, raster_ny=13,
                                  max_iter=1000, f2conv=1e-10, polish=True, **kw)
        FEs = gpu.relax_strokes_tilted(grid, P, pt, dynamic=dynamic)
        assert np.array_equal(FEs.cpu().numpy(), o)


def test_polished_relax_pp_bit_exact_and_smaller_residual(cuda):
    grid, dinv, pts, nz = _relax_setup(seed=13)
    a, b, c = _tip_frame()
    kw = dict(stiffness=[-0.0156, -0.0156, -1.248, 0.0], dpos0=[0, 0, 0, 0], relax_params=[0.5, 0.1, 0.02, 0.5])
    pts2 = pts.copy()
    pts2[:, 2] = 6.0
    pt = torch.from_numpy(pts2).cuda()
    g = grid.cpu().numpy()
    res = {}
    for polish in (False, True):
        oFE, oPP = O.relax_pp(g, dinv, pts2, nz, a, b, c, kw["stiffness"], kw["dpos0"], kw["relax_params"],
                              [0.005, 0, 0, 0], 1000, 1e-10, prec="f32", polish=polish)
        for dynamic in (True, False):
            P = _lib.make_scan_params(dinv=dinv, tipA=a, tipB=b, tipC=c, surfFF=[0.005, 0, 0, 0], nz=nz, raster_ny=13,
                                      max_iter=1000, f2conv=1e-10, polish=polish, **kw)
            FEs, PPs = gpu.relax_pp(grid, P, pt, dynamic=dynamic)
            assert np.array_equal(FEs.cpu().numpy(), oFE) and np.array_equal(PPs.cpu().numpy(), oPP)
        res[polish] = _residual(g, dinv, pts2, nz, a, b, c, kw, 0.005, oPP)
    conv = np.isfinite(res[True])
    assert conv.mean() > 0.95
    # FIRE stopped below |F| = 1e-5 eV/A (median 7.6e-6 measured); the polish takes the states down to
    # the float32 floor: a position is stored to ulp(z) ~ 4.8e-7 A at z ~ 6 A, and k_z * ulp(z) ~ 6e-7 eV/A
    assert np.median(res[True][conv]) < 2e-6
    assert np.median(res[True][conv]) < 0.25 * np.median(res[False][conv])
    assert np.percentile(res[True][conv], 99) < 1e-5


def _residual(grid, dinv, pts, nz, a, b, c, kw, surf, PPs):
    """|G| at each stored position in FP64 on the same (FP32) grid: trilinear sample + spring + surf."""
    g64 = grid.astype(np.float64)
    q = PPs[..., :3].reshape(-1, 3).astype(np.float64)
    raw = O.raw_tilted(g64, dinv, np.concatenate([q, np.zeros((len(q), 1))], 1).astype(np.float32), 1,
                       [1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 1, 0], [0, 0, 0, 0], [0, 0, 0, 0], prec="f64")[:, 0, :3]
    # the positions were rounded to float32 for the sampler: evaluate the spring at the same points
    q32 = q.astype(np.float32).astype(np.float64)
    dz = c[3]
    iz = np.tile(np.arange(nz), len(pts))
    tip = np.repeat(pts[:, :3].astype(np.float64), nz, 0) + iz[:, None] * dz * np.asarray(c[:3], np.float64)
    R = np.stack([a[:3], b[:3], c[:3]]).astype(np.float64)
    d = (q32 - tip) @ R.T
    k = np.asarray(kw["stiffness"], np.float64)
    f = (d - np.asarray(kw["dpos0"][:3], np.float64)) * k[:3]
    G = raw + f @ R + np.asarray(c[:3], np.float64) * surf
    r = np.linalg.norm(G, axis=1)
    r[PPs[..., 3].ravel() <= 0] = np.nan
    return r


def test_polish_rejected_for_2d_and_raw(cuda):
    grid, dinv, pts, nz = _relax_setup()
    P = _lib.make_scan_params(dinv=dinv, dTip=[0, 0, -0.1, 0], stiffness=[0.03, 0, 0, 0], relax_params=[0.3, 0.2, 0, 0],
                              nz=nz, fire=False, polish=True)
    with pytest.raises(ValueError, match="POLISH"):
        gpu.relax_2d(grid, P, torch.from_numpy(pts).cuda())
    with pytest.raises(ValueError, match="POLISH"):
        gpu.fe_in_strokes_tilted(grid, P, torch.from_numpy(pts).cuda())


def test_afmulator_newton_polish_attribute(cuda):
    """AFMulator.newton_polish (not in the reference) turns the polish on for scan_fdbm and scan_fdbm_pair:
    the results equal the oracle's polished relaxStrokes; the default leaves them unpolished."""
    from spammm_b200.AFM import AFMulator
    rng = np.random.default_rng(21)
    F_total = (0.02 * rng.standard_normal((24, 22, 30, 4))).astype(np.float32)
    origin = np.array([-3., -2.75, -1.0], np.float32)
    afm = AFMulator(use_morse=True)
    afm.setup_fdbm_grid(F_total, origin, 0.25)
    xs = np.linspace(-1, 1, 5).astype(np.float32)
    ys = np.linspace(-1, 1, 4).astype(np.float32)
    hs = np.linspace(3.0, 3.5, 6).astype(np.float32)
    grid = np.ascontiguousarray(F_total.transpose(2, 1, 0, 3))
    dinv = (afm.fdbm_dinvA, afm.fdbm_dinvB, afm.fdbm_dinvC)
    pts, dTip = afm._scan_fdbm_points(xs, ys, hs, 0.2, 3.0, np.zeros(3, np.float32), False)
    outs = {}
    for polish in (False, True):
        afm.newton_polish = polish
        FEs, disp = afm.scan_fdbm(xs, ys, hs, mol_z=0.2)
        oFE, oD = O.relax_strokes(grid, dinv, pts, 6, dTip, [-0.03, -0.03, -0.03, -20.0], [0, 0, -3.0, 3.0],
                                  afm.relax_pars, flip=True, polish=polish)
        assert np.array_equal(FEs, oFE.reshape(5, 4, 6, 4))
        assert np.array_equal(disp["dx"], oD.reshape(5, 4, 6, 4)[..., 0])
        (Ff, dff), _ = afm.scan_fdbm_pair(xs, ys, hs, mol_z=0.2)
        assert np.array_equal(Ff, FEs)
        outs[polish] = FEs
    assert not np.array_equal(outs[False], outs[True])
