"""Drop-in AFMulator API on the GPU, mirroring the reference's own tests
(tests/SPM/test_afm_morse.py, tests/SPM/test_scan_contract.py) plus parity of
the direct Morse path and its VJP against the reference's FP64 oracles."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from spammm_b200 import AFM, _lib, gpu
from spammm_b200.AFM import AFMulator

pytestmark = pytest.mark.gpu


def test_scan_fdbm_oscillation_direction_does_not_replace_z_approach(cuda):
    """(tests/SPM/test_afm_morse.py:128-148) df direction leaves the acquired xyz volume unchanged."""
    step = 0.25
    origin = np.array([-2., -2., 0.], dtype=np.float32)
    F_total = np.zeros((16, 16, 20, 4), dtype=np.float32)
    F_total[..., 3] = origin[2] + step * np.arange(F_total.shape[2], dtype=np.float32)[None, None, :]
    afm = AFMulator(use_morse=False, nloc=32)
    afm.setup_fdbm_grid(F_total, origin, step)
    xs = np.array([-1., 0., 1.], dtype=np.float32)
    heights = np.array([1., 2., 3.], dtype=np.float32)
    kw = dict(mol_z=0., ppm_mode=False, K_LAT=0., K_RAD=0., bond_length=0.)
    F_z, _ = afm.scan_fdbm(xs, xs, heights, osc_dir=(0., 0., 1.), **kw)
    F_x, _ = afm.scan_fdbm(xs, xs, heights, osc_dir=(1., 0., 0.), **kw)
    assert np.array_equal(F_x, F_z)
    assert np.ptp(F_x[..., 3].mean(axis=(0, 1))) > 1.0
    with pytest.raises(ValueError):
        afm.scan_fdbm(xs, xs, heights, osc_dir=(0., 0., 0.), **kw)


def test_scan_fdbm_flip_and_reverse_match_oracle(cuda):
    rng = np.random.default_rng(0)
    F_total = (0.02 * rng.standard_normal((24, 22, 30, 4))).astype(np.float32)
    afm = AFMulator(use_morse=True)
    origin = np.array([-3., -2.75, -1.0], np.float32)
    afm.setup_fdbm_grid(F_total, origin, 0.25)
    xs = np.linspace(-1, 1, 5).astype(np.float32)
    ys = np.linspace(-1, 1, 4).astype(np.float32)
    hs = np.linspace(3.0, 3.5, 6).astype(np.float32)
    for reverse in (False, True):
        FEs, disp = afm.scan_fdbm(xs, ys, hs, mol_z=0.2, reverse=reverse)
        assert FEs.shape == (5, 4, 6, 4) and FEs.dtype == np.float32
        pts, dTip = afm._scan_fdbm_points(xs, ys, hs, 0.2, 3.0, np.zeros(3, np.float32), reverse)
        grid = np.ascontiguousarray(F_total.transpose(2, 1, 0, 3))
        dinv = (afm.fdbm_dinvA, afm.fdbm_dinvB, afm.fdbm_dinvC)
        oFE, oD = O.relax_strokes(grid, dinv, pts, 6, dTip, [-0.03, -0.03, -0.03, -20.0], [0, 0, -3.0, 3.0],
                                  afm.relax_pars, flip=not reverse)
        assert np.array_equal(FEs, oFE.reshape(5, 4, 6, 4))
        assert np.array_equal(disp["dz"], oD.reshape(5, 4, 6, 4)[..., 2])


def test_scan_fdbm_pair_equals_two_scans(cuda):
    """Forward + backward strokes in one launch (SPM_FLAG_PAIRED) give the two
    scan_fdbm calls' results bit for bit; the C ABI rejects the flag elsewhere."""
    rng = np.random.default_rng(2)
    F_total = (0.02 * rng.standard_normal((24, 22, 30, 4))).astype(np.float32)
    afm = AFMulator(use_morse=True)
    afm.setup_fdbm_grid(F_total, np.array([-3., -2.75, -1.0], np.float32), 0.25)
    xs = np.linspace(-1, 1, 7).astype(np.float32)
    ys = np.linspace(-1, 1, 5).astype(np.float32)
    hs = np.linspace(3.0, 3.7, 8).astype(np.float32)
    kw = dict(mol_z=0.2, K_LAT=0.03, K_RAD=20.0, bond_length=3.0, base_pos=(0.05, -0.02, 0.0))
    (Ff, df_), (Fb, db_) = afm.scan_fdbm_pair(xs, ys, hs, **kw)
    Ff1, d1 = afm.scan_fdbm(xs, ys, hs, **kw)
    Fb1, d2 = afm.scan_fdbm(xs, ys, hs, reverse=True, **kw)
    assert Ff.shape == Fb.shape == (7, 5, 8, 4)
    assert np.array_equal(Ff, Ff1) and np.array_equal(Fb, Fb1)
    for c in ("dx", "dy", "dz"):
        assert np.array_equal(df_[c], d1[c]) and np.array_equal(db_[c], d2[c])
    assert not np.array_equal(Ff, Fb)  # the strokes differ: hysteresis or at least different start
    # the flag is relaxStrokes-only and needs an even stroke count
    from spammm_b200 import gpu
    P = _lib.make_scan_params(dinv=(afm.fdbm_dinvA, afm.fdbm_dinvB, afm.fdbm_dinvC), nz=4, paired=True)
    pts = torch.zeros((3, 4), dtype=torch.float32, device="cuda")
    with pytest.raises(ValueError, match="PAIRED"):
        gpu.relax_strokes(afm.img_FF_fdbm, P, pts)
    with pytest.raises(ValueError, match="PAIRED"):
        gpu.relax_strokes_tilted(afm.img_FF_fdbm, P, torch.zeros((4, 4), dtype=torch.float32, device="cuda"))


def _toy(n_atoms, seed):
    """_make_toy_system of tests/SPM/test_afm_morse.py:626-642 (same RNG draws)."""
    rng = np.random.default_rng(seed)
    atoms = np.zeros((n_atoms, 4))
    atoms[:, :3] = rng.uniform(-1.0, 1.0, (n_atoms, 3))
    atoms[:, 3] = rng.uniform(-0.3, 0.3, n_atoms)
    cMs = np.zeros((n_atoms, 4))
    cMs[:, 0] = rng.uniform(2.5, 3.5, n_atoms)
    cMs[:, 1] = rng.uniform(1e-3, 5e-3, n_atoms)
    cMs[:, 2] = -1.8
    return atoms, cMs, np.array([0., -0.1, 0.1, 0.]), np.array([0., 1.8, 3.6, 0.])


def _toy_afm(n_atoms=2, seed=7):
    atoms, cMs, tQ, tQZ = _toy(n_atoms, seed)
    afm = AFMulator(use_morse=True)
    afm.atoms_arr = atoms.astype(np.float32)
    afm.cLJs_arr = cMs.astype(np.float32)
    afm.tipQs = tQ.astype(np.float32)
    afm.tipQZs = tQZ.astype(np.float32)
    return afm, atoms, cMs


def _toy_scan(atoms, nxy=(3, 3)):
    nx, ny = nxy
    mn, mx = atoms[:, :3].min(axis=0), atoms[:, :3].max(axis=0)
    p0 = np.array([mn[0] + (mx[0] - mn[0]) * 0.05, mn[1] + (mx[1] - mn[1]) * 0.05, float(mx[2]) + 5.0 + 4.0],
                  np.float32)
    da = np.array([(mx[0] - mn[0]) * 0.9 / max(nx - 1, 1), 0., 0.], np.float32)
    db = np.array([0., (mx[1] - mn[1]) * 0.9 / max(ny - 1, 1), 0.], np.float32)
    return p0, da, db


def test_direct_toy_matches_reference_golden(cuda, golden):
    """GPU direct forward on the reference's toy; residual < 1e-4 eV/A at every
    PP re-evaluated in FP64, same convergence branch and PPs within 2e-3 A of
    the FP64 oracle run with the kernel's loop semantics."""
    g = golden("direct_golden.npz")
    afm, atoms, cMs = _toy_afm(2, 97)
    assert np.allclose(atoms, g["r_atoms"]) and np.allclose(cMs, g["r_cMs"])
    p0, da, db = _toy_scan(atoms)
    FEs, pts, PPs = afm.run_scan_morse_direct(nxy=(3, 3), nz=5, dtip=-0.1, scan_p0=p0, scan_da=da, scan_db=db)
    assert FEs.shape == (3, 3, 5, 4) and PPs.shape == (3, 3, 5, 4) and pts.shape == (3, 3, 3)
    assert np.allclose(pts.reshape(-1, 3), g["r_pts"])
    assert (PPs[..., 3] > 0).all()
    ref_FE, ref_PP = O.relax_direct(atoms, cMs, np.c_[pts.reshape(-1, 3), np.zeros(9)].astype(np.float32), 5,
                                    afm.tipA, afm.tipB, afm.tipC, afm.stiffness, afm.dpos0, afm.relax_pars,
                                    afm.surfFF, afm.tipQs, afm.tipQZs)
    tip = pts.reshape(-1, 3).astype(np.float64)
    for iz in range(5):
        q = PPs.reshape(-1, 5, 4)[:, iz, :3].astype(np.float64)
        fe = O.pair_fe(1, atoms, cMs, q, afm.tipQs, afm.tipQZs)
        dpos = q - (tip + iz * np.array([0, 0, -0.1]))
        ft = (dpos - afm.dpos0[:3]) * afm.stiffness[:3] + dpos * (afm.stiffness[3] * (np.linalg.norm(dpos, axis=1) -
                                                                                    afm.dpos0[3]) /
                                                                  np.linalg.norm(dpos, axis=1))[:, None]
        resid = np.linalg.norm(fe[:, :3] + ft, axis=1)
        assert resid.max() < 1e-4, f"iz={iz} residual {resid.max():.3e}"
    assert np.array_equal(np.sign(PPs[..., 3]).ravel(), np.sign(ref_PP[..., 3]).ravel())
    assert np.abs(PPs.reshape(-1, 5, 4)[..., :3] - ref_PP[..., :3]).max() < 2e-3


@pytest.mark.parametrize("na,nxy", [(10, (100, 100)), (30, (80, 80)), (60, (60, 60)), (60, (20, 20))])
def test_direct_lane_groups(cuda, na, nxy):
    """The direct relaxation's lane groups (4, 8, 16 and 32 lanes per pixel for these atom counts and
    scan sizes): every state converged with an FP64 residual below the reference's 1e-4 eV/A gate, the
    same convergence branch as the FP64 oracle run with the kernel's loop semantics, and PPs within the
    stopping slack of it (the lanes' partial sums round differently from the oracle's one loop)."""
    from spammm_b200 import synthetic
    pos, Z, q = synthetic.planar_molecule({"C": max(1, na - na // 4), "H": na // 4}, 900 + na)
    atoms, cMs = synthetic._morse_atoms_from_Z(pos, Z)
    atoms[:, 3] = q.astype(np.float32)
    afm = AFMulator(use_morse=True)
    afm.atoms_arr, afm.cLJs_arr = atoms.astype(np.float32), cMs.astype(np.float32)
    nz, dtip = 6, -0.1
    span = np.abs(pos[:, :2]).max() + 1.0
    p0 = np.array([-span, -span, 6.0 + 4.0], np.float32)  # the probe from 6 A above the plane
    da = np.array([2 * span / (nxy[0] - 1), 0, 0], np.float32)
    db = np.array([0, 2 * span / (nxy[1] - 1), 0], np.float32)
    FEs, pts, PPs = afm.run_scan_morse_direct(nxy=nxy, nz=nz, dtip=dtip, scan_p0=p0, scan_da=da, scan_db=db)
    assert (PPs[..., 3] > 0).all()
    n = nxy[0] * nxy[1]
    ref_FE, ref_PP = O.relax_direct(atoms, cMs, np.c_[pts.reshape(-1, 3), np.zeros(n)].astype(np.float32), nz,
                                    afm.tipA, afm.tipB, afm.tipC.copy() * np.array([1, 1, 1, 0], np.float32) +
                                    np.array([0, 0, 0, dtip], np.float32), afm.stiffness, afm.dpos0,
                                    afm.relax_pars, afm.surfFF, afm.tipQs, afm.tipQZs)
    PPf = PPs.reshape(-1, nz, 4)
    tip = pts.reshape(-1, 3).astype(np.float32)  # stepped down in float32 as the kernel does
    for iz in range(nz):
        qz = PPf[:, iz, :3].astype(np.float64)
        fe = O.pair_fe(1, atoms.astype(np.float64), cMs.astype(np.float64), qz, afm.tipQs, afm.tipQZs)
        dpos = qz - tip.astype(np.float64)
        tip[:, 2] = tip[:, 2] + np.float32(dtip)
        rn = np.linalg.norm(dpos, axis=1)
        ft = (dpos - afm.dpos0[:3]) * afm.stiffness[:3] + dpos * (afm.stiffness[3] * (rn - afm.dpos0[3]) / rn)[:, None]
        assert np.linalg.norm(fe[:, :3] + ft, axis=1).max() < 1e-4, iz
    assert np.array_equal(np.sign(PPf[..., 3]), np.sign(ref_PP[..., 3]))
    # both stop at |F| < 1e-4 eV/A: along the softest spring mode (k = 0.03 eV/A^2) two converged states
    # may differ by up to 2 * 1e-4 / 0.03 = 6.7e-3 A; almost all agree to ~1e-6 A
    dq = np.abs(PPf[..., :3] - ref_PP[..., :3]).max(axis=-1)
    assert dq.max() < 6.7e-3 and np.quantile(dq, 0.999) < 2e-3


def test_direct_contract_errors(cuda):
    afm, atoms, cMs = _toy_afm(129, 129)
    p0, da, db = _toy_scan(atoms, (2, 2))
    with pytest.raises((ValueError, RuntimeError, AssertionError)):
        afm.run_scan_morse_direct(nxy=(2, 2), nz=3, dtip=-0.2, scan_p0=p0, scan_da=da, scan_db=db)
    afm, atoms, cMs = _toy_afm(2, 7)
    with pytest.raises((ValueError, TypeError, AssertionError)):
        afm.run_scan_morse_direct(nxy=(2, 2), nz=3, dtip=-0.2, scan_p0=None, scan_da=None, scan_db=None)
    p0, da, db = _toy_scan(atoms, (2, 2))
    with pytest.raises(ValueError):
        afm.run_scan_morse_direct(nxy=(2, 2), nz=3, dtip=0.2, scan_p0=p0, scan_da=da, scan_db=db)


def test_direct_padded_scan_converges(cuda):
    afm, atoms, cMs = _toy_afm(3, 19)
    p0, da, db = _toy_scan(atoms, (5, 7))
    FEs, pts, PPs = afm.run_scan_morse_direct(nxy=(5, 7), nz=4, dtip=-0.2, scan_p0=p0, scan_da=da, scan_db=db)
    assert np.isfinite(FEs).all() and np.isfinite(PPs).all() and (PPs[..., 3] > 0).all()


def test_vjp_matches_reference_oracle(cuda, golden):
    """GPU adjoint at the reference's tightly converged PPs vs its FP64 VJP oracle
    (tests/SPM/test_afm_morse.py:1633-1667: rel 2e-3 per channel)."""
    from spammm_b200 import _lib, gpu
    g = golden("direct_golden.npz")
    tipC = AFMulator.DEFAULT_tipC.copy()
    tipC[3] = -0.2
    P = _lib.make_scan_params(tipA=AFMulator.DEFAULT_tipA, tipB=AFMulator.DEFAULT_tipB, tipC=tipC,
                              stiffness=AFMulator.DEFAULT_stiffness, dpos0=AFMulator.DEFAULT_dpos0,
                              relax_params=AFMulator.DEFAULT_relax_pars, surfFF=AFMulator.DEFAULT_surfFF, nz=5)
    pts = np.zeros((9, 4), np.float32)
    pts[:, :3] = g["v_pts"]
    PPs = g["v_PPs"].astype(np.float32).reshape(-1, 4)
    dL = g["v_dL"].astype(np.float32).reshape(-1, 4)
    atoms, cMs = g["v_atoms"].astype(np.float32), g["v_cMs"].astype(np.float32)
    lam, diag = gpu.adjoint_direct_state(atoms, cMs, pts, P, g["v_Qs"], g["v_QZs"], PPs, dL)
    assert (diag[:, 3] == 0).all(), diag.cpu().numpy()
    grad = gpu.adjoint_direct_params(atoms, cMs, pts, P, g["v_Qs"], g["v_QZs"], PPs, dL, lam).cpu().numpy()
    ref = g["v_grad"]
    for p in range(6):
        wd = np.abs(grad[:, p] - ref[:, p]).max()
        scale = np.abs(ref[:, p]).max() + 1e-30
        assert wd / scale < 2e-3 or wd < 1e-4, f"channel {p}: {grad[:, p]} vs {ref[:, p]}"


def test_vjp_is_deterministic_and_validates(cuda):
    afm, atoms, cMs = _toy_afm(2, 7)
    p0, da, db = _toy_scan(atoms, (2, 2))
    FEs, pts, PPs = afm.run_scan_morse_direct(nxy=(2, 2), nz=3, dtip=-0.2, scan_p0=p0, scan_da=da, scan_db=db)
    _, _, dL = AFM.df_loss_seed(FEs, np.zeros((2, 2, 3)), -0.2)
    g1, d1 = afm.vjp_scan_morse_direct(PPs, pts, -0.2, dL.astype(np.float32))
    g2, _ = afm.vjp_scan_morse_direct(PPs, pts, -0.2, dL.astype(np.float32))
    assert np.array_equal(g1, g2) and g1.shape == (2, 6) and g1.dtype == np.float64
    bad = PPs.copy()
    bad[0, 0, 0, 3] = -5.0
    with pytest.raises((ValueError, RuntimeError)):
        afm.vjp_scan_morse_direct(bad, pts, -0.2, dL.astype(np.float32))
    with pytest.raises((ValueError, AssertionError)):
        afm.vjp_scan_morse_direct(PPs, pts, -0.2, np.zeros((3, 3, 3, 4), np.float32))
    afm.atoms_arr = afm.atoms_arr.copy()
    afm.atoms_arr[0, 0] += 0.01
    with pytest.raises(RuntimeError, match="stale"):
        afm.vjp_scan_morse_direct(PPs, pts, -0.2, dL.astype(np.float32))


def test_make_forcefield_run_scan_and_raw(cuda):
    """LJ and Morse grids through the drop-in calls; raw vs relaxed behave as the
    reference tests require (tests/SPM/test_afm_morse.py:188-243)."""
    from spammm_b200.synthetic import planar_molecule
    pos, Z, q = planar_molecule({"C": 6, "H": 6}, 1)
    for morse in (True, False):
        afm = AFMulator(use_morse=morse)
        afm.mol = AFM._Molecule(pos, ["C" if z == 6 else "H" for z in Z], q)
        afm.assign_params()
        afm.setup_grid(n=(50, 50, 30), margin=3.0, z_top=12.0)
        afm.make_forcefield()
        img = afm.download_image_rgba_xyz(afm.img_FF, afm.n)
        assert img.shape == (50, 50, 30, 4) and np.isfinite(img).all() and img[..., 3].min() < 0
        raw, pts = afm.get_raw_FE(nxy=(30, 30), nz=15, dtip=-0.2)
        rel, pts2 = afm.run_scan(nxy=(30, 30), nz=15, dtip=-0.2)
        assert np.isfinite(raw).all() and np.isfinite(rel).all()
        assert np.max(np.abs(raw[:, :, -1, 2])) > np.max(np.abs(raw[:, :, 0, 2]))
        r = np.corrcoef(raw[..., 2].ravel(), rel[..., 2].ravel())[0, 1]
        assert r > 0.5
        assert np.sqrt(np.mean((raw[..., 2] - rel[..., 2]) ** 2)) > 1e-6 * np.abs(rel[..., 2]).max()


def test_pair_dissipation_fused_equals_separate_calls(cuda):
    """spm_relax_pair_dissipation: the forward + backward strokes and compute_dissipation in one launch
    (the second stroke of each pixel integrates it) give scan_fdbm_pair's strokes and spm_dissipation's
    E_diss bit for bit, for a window sweep of h_df / amplitudes and a tilted oscillation direction."""
    rng = np.random.default_rng(31)
    F_total = (0.02 * rng.standard_normal((24, 22, 30, 4))).astype(np.float32)
    afm = AFMulator(use_morse=True)
    afm.setup_fdbm_grid(F_total, np.array([-3., -2.75, -1.0], np.float32), 0.25)
    xs = np.linspace(-1, 1, 9).astype(np.float32)
    ys = np.linspace(-1, 1, 7).astype(np.float32)
    hs = np.linspace(3.0, 4.5, 16).astype(np.float32)
    kw = dict(mol_z=0.2, K_LAT=0.03, K_RAD=20.0, bond_length=3.0, return_device=True)
    for h_df, amp, osc in ((hs[3:13:2], 0.3, (0., 0., 1.)), (np.array([3.6, 4.0]), 0.55, (0.3, 0., 1.)),
                           (np.array([3.0, 4.5]), 0.01, (0., 0., 1.))):  # the last: windows of < 2 heights
        (Ff, df_), (Fb, db_), E = afm.scan_fdbm_pair(xs, ys, hs, osc_dir=osc, dissipation=(hs, h_df, amp), **kw)
        (Ff2, _), (Fb2, _) = afm.scan_fdbm_pair(xs, ys, hs, osc_dir=osc, **kw)
        assert torch.equal(Ff, Ff2) and torch.equal(Fb, Fb2)
        E2 = gpu.dissipation(Ff2, Fb2, hs, h_df, amp, osc)
        assert E.shape == E2.shape == (9, 7, len(h_df))
        assert torch.equal(E, E2)
        assert float(E.abs().max()) > 0
