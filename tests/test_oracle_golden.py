"""Pins the oracle (and the host-side mirrors) to outputs of the SPAMMM
reference itself (tests/golden/*.npz, written by tests/golden/gen_golden.py)."""
import numpy as np
import pytest

from oracle import oracle as O


def test_df_amp_dir_matches_reference(golden):
    g = golden("df_golden.npz")
    for i in range(int(g["n_cases"])):
        FEs, sp, od, amp = g[f"c{i}_FEs"], g[f"c{i}_spacing"], g[f"c{i}_osc"], float(g[f"c{i}_amp"])
        sp = float(sp) if sp.ndim == 0 else sp
        ours = O.compute_df_amp_dir(FEs, sp, od, amp)
        ref = g[f"c{i}_amp_dir"]
        assert ours.dtype == ref.dtype == np.float32
        np.testing.assert_allclose(ours, ref, rtol=1e-6, atol=1e-6 * np.abs(ref).max(), err_msg=f"case {i}")


def test_df_dir_matches_reference(golden):
    g = golden("df_golden.npz")
    for i in range(int(g["n_cases"])):
        FEs, sp, od = g[f"c{i}_FEs"], g[f"c{i}_spacing"], g[f"c{i}_osc"]
        sp = float(sp) if sp.ndim == 0 else sp
        np.testing.assert_allclose(O.compute_df_dir(FEs, sp, od), g[f"c{i}_dir"], rtol=1e-12, atol=1e-12)


def test_compute_df_and_amp_match_reference(golden):
    g = golden("df_golden.npz")
    np.testing.assert_allclose(O.compute_df(g["Fz"], 0.1), g["compute_df"], rtol=1e-6, atol=1e-6)
    np.testing.assert_allclose(O.compute_df_amp(g["Fz"], 0.1, 0.6), g["compute_df_amp"], rtol=1e-6, atol=1e-6)


def test_df_loss_seed_matches_reference(golden):
    g = golden("loss_golden.npz")
    for i in range(int(g["n_cases"])):
        w = g[f"c{i}_w"]
        loss, df, dL = O.df_loss_seed(g[f"c{i}_FEs"], g[f"c{i}_tgt"], float(g[f"c{i}_dtip"]), w if w.size else None)
        assert loss == pytest.approx(float(g[f"c{i}_loss"]), rel=1e-13)
        np.testing.assert_allclose(df, g[f"c{i}_df"], rtol=1e-13, atol=1e-13)
        np.testing.assert_allclose(dL, g[f"c{i}_dL"], rtol=1e-12, atol=1e-15)


def test_dissipation_matches_reference(golden):
    g = golden("diss_golden.npz")
    E = O.compute_dissipation(g["Ff"], g["Fb"], g["h_scan"], g["h_df"], 1.0, (0., 0., 1.))
    np.testing.assert_allclose(E, g["E_z"], rtol=1e-6, atol=1e-7)
    E = O.compute_dissipation(g["Ff"], g["Fb"], g["h_scan"], g["h_df"], 0.6, (0.5, 0., 1.))
    np.testing.assert_allclose(E, g["E_t"], rtol=1e-6, atol=1e-7)


def test_height_stacks_match_reference(golden):
    from spammm_b200.AFM_utils import afm_df_height_stacks
    g = golden("diss_golden.npz")
    for pre, args, kw in (("h", (3.7, 4.7, 0.1), dict(amp=1.0)),
                          ("h2", (3.0, 4.0, 0.2), dict(amp=0.5, osc_dir=(1., 0., 1.))),
                          ("h3", (3.7, 4.7, 0.1), dict(amp=1.0, osc_dir=(1., 0., 0.)))):
        h_df, h_Fz, h_scan = afm_df_height_stacks(*args, **kw)
        assert np.array_equal(h_df, g[f"{pre}_df"])
        assert np.array_equal(h_Fz, g[f"{pre}_Fz"])
        assert np.array_equal(h_scan, g[f"{pre}_scan"])


def test_texel_frames_match_reference(golden):
    from spammm_b200.AFM import AFMulator
    g = golden("frame_golden.npz")
    for i in range(3):
        L, o, n = g[f"c{i}_L"], g[f"c{i}_o"].astype(np.float32), tuple(int(v) for v in g[f"c{i}_n"])
        ours = np.stack(AFMulator._make_dinv_axis_aligned(L, o, n))
        assert np.array_equal(ours, g[f"c{i}_dinv"])
        assert np.array_equal(np.stack(O.dinv_axis_aligned(L, o, n)), g[f"c{i}_dinv"])


def test_texel_centre_convention():
    """Node i maps to normalized coordinate (i+0.5)/n (tests/SPM/test_texel_centers.py)."""
    dA, dB, dC = O.dinv_axis_aligned((10.0, 20.0, 30.0), np.zeros(3, np.float32), (50, 100, 150))
    for i in (0, 1, 25, 49):
        assert abs(i * 0.2 * dA[0] + dA[3] - (i + 0.5) / 50) < 1e-5
    assert dA[3] != 0 and dB[3] != 0 and dC[3] != 0


def test_morse_mixing_matches_reference(golden):
    from spammm_b200.AFM_utils import _morse_atoms_from_Z
    g = golden("frame_golden.npz")
    at, cm = _morse_atoms_from_Z(g["mix_pos"], g["mix_Z"])
    assert np.array_equal(at, g["mix_atoms"])
    assert np.array_equal(cm, g["mix_cMs"])


def test_pair_law_matches_reference(golden):
    g = golden("pair_golden.npz")
    for i in range(int(g["n_cases"])):
        fe = O.pair_fe(1, g[f"c{i}_atoms"], g[f"c{i}_cMs"], g[f"c{i}_q"], g[f"c{i}_Qs"], g[f"c{i}_QZs"])
        np.testing.assert_allclose(fe, g[f"c{i}_fe"], rtol=1e-12, atol=1e-14)


def test_direct_relax_matches_reference_fp64(golden):
    from spammm_b200.AFM import AFMulator as A
    g = golden("direct_golden.npz")
    pts = np.zeros((9, 4), np.float32)
    pts[:, :3] = g["r_pts"]
    FEs, PPs = O.relax_direct(g["r_atoms"], g["r_cMs"], pts, 5, A.DEFAULT_tipA, A.DEFAULT_tipB, A.DEFAULT_tipC,
                              A.DEFAULT_stiffness, A.DEFAULT_dpos0, A.DEFAULT_relax_pars, A.DEFAULT_surfFF,
                              g["r_Qs"], g["r_QZs"], test_oracle_loop=True)
    assert np.array_equal(PPs[..., 3], g["r_PPs"][..., 3]), "iteration counts / convergence signs differ"
    np.testing.assert_allclose(PPs[..., :3], g["r_PPs"][..., :3], atol=1e-9)
    np.testing.assert_allclose(FEs, g["r_FEs"], rtol=1e-6, atol=1e-9)


def test_direct_relax_tight_matches_reference_fp64(golden):
    from spammm_b200.AFM import AFMulator as A
    g = golden("direct_golden.npz")
    pts = np.zeros((9, 4), np.float32)
    pts[:, :3] = g["v_pts"]
    tipC = A.DEFAULT_tipC.copy()
    tipC[3] = -0.2
    FEs, PPs = O.relax_direct(g["v_atoms"], g["v_cMs"], pts, 5, A.DEFAULT_tipA, A.DEFAULT_tipB, tipC,
                              A.DEFAULT_stiffness, A.DEFAULT_dpos0, A.DEFAULT_relax_pars, A.DEFAULT_surfFF,
                              g["v_Qs"], g["v_QZs"], max_iter=2000, f2conv=1e-16, test_oracle_loop=True)
    np.testing.assert_allclose(PPs[..., :3], g["v_PPs"][..., :3], atol=1e-9)
    np.testing.assert_allclose(FEs, g["v_FEs"], rtol=1e-6, atol=1e-9)


def _golden_grid_args(g):
    n = tuple(int(v) for v in g["n"])
    step = float(g["step"])
    o = g["origin"]
    p0 = np.array([o[0], o[1], o[2], 0.0], np.float32)
    return n, p0, np.array([step, 0, 0, 0]), np.array([0, step, 0, 0]), np.array([0, 0, step, 0])


def test_grid_build_morse_matches_reference_nodes(golden):
    g = golden("gridrelax_golden.npz")
    n, p0, dA, dB, dC = _golden_grid_args(g)
    grid = O.grid_build(1, g["atoms"].astype(np.float32), g["cMs"].astype(np.float32), n, p0, dA, dB, dC, g["Qs"],
                        g["QZs"], prec="f64")
    # the golden nodes use float64 atoms; the grid builder takes float32 inputs like the reference kernel
    ref = g["grid"]
    scale = np.abs(ref).max(axis=(0, 1, 2))
    assert np.all(np.abs(grid - ref) <= 1e-5 * np.abs(ref) + 1e-6 * scale)


def test_grid_relaxation_matches_reference_loops(golden):
    g = golden("gridrelax_golden.npz")
    grid, dinv, pts, nz = g["grid"], g["dinv"], g["pts"], int(g["nzs"])
    FEs, disps = O.relax_strokes(grid, dinv, pts, nz, g["dTip"], g["stiffness"], g["dpos0"], g["relax"], prec="f64")
    np.testing.assert_allclose(FEs, g["strokes_FEs"], rtol=1e-6, atol=1e-9)
    np.testing.assert_allclose(disps, g["strokes_disps"], atol=1e-8)
    FEt = O.relax_tilted(grid, dinv, pts, nz, [1, 0, 0, 0], [0, 1, 0, 0], g["tipC"], g["stiffness"], g["dpos0"],
                         g["relax"], [0, 0, 0, 0], prec="f64")
    np.testing.assert_allclose(FEt, g["tilted_FEs"], rtol=1e-6, atol=1e-9)
    raw = O.raw_tilted(grid, dinv, pts, nz, [1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 1, 0], g["dTip"], g["dpos0"],
                       prec="f64")
    np.testing.assert_allclose(raw, g["raw_FEs"], rtol=1e-12, atol=1e-14)


def test_oracle_relax_2d_uniform_field_equilibrium():
    """relaxStrokes2D restatement (kernels/AFM.cl:410-450): in a uniform lateral
    force F the damped MD settles at anchor + F/K_lat; z is fixed per slice and
    the slices are stored lowest-first under flip."""
    from oracle import oracle as O
    nx = ny = nz = 16
    g = np.zeros((nz, ny, nx, 4), np.float32)
    g[..., 0], g[..., 1], g[..., 3] = 0.01, -0.02, np.arange(nz, dtype=np.float32)[:, None, None]
    dinv = O.dinv_axis_aligned(np.array([1.6, 1.6, 1.6]), np.zeros(3), (nx, ny, nz))
    pts = np.array([[0.8, 0.8, 1.2, 0]], np.float32)
    K = 0.05
    FEs, D = O.relax_2d(g, dinv, pts, 4, K, 0.1, 0.3, 0.2, 5000, 1e-16, flip=True)
    np.testing.assert_allclose(D[0, :, 0], 0.01 / K, rtol=1e-4)
    np.testing.assert_allclose(D[0, :, 1], -0.02 / K, rtol=1e-4)
    assert not D[..., 2:].any()
    # E channel = layer index; node k sits at z = k*0.1: slices at z = 1.2 .. 0.9, stored lowest first
    np.testing.assert_allclose(FEs[0, :, 3], [9.0, 10.0, 11.0, 12.0], atol=1e-4)


def test_oracle_convolve_z_and_izo_z_known_answers():
    """convolveZ / izoZ restatements (kernels/AFM.cl:666-723).  The reference has
    no host caller for these kernels and its OpenCL does not run here, so they
    are pinned to known answers of the kernel loops: a z-convolution equals the
    float64 sum of the same products (within FP32 accumulation), a one-weight
    convolution is a scaled copy, an empty one is zero; the iso height follows
    the kernel's iz + fraction-from-iz-1 rule, -1 without a crossing."""
    from oracle import oracle as O
    rng = np.random.default_rng(3)
    F = rng.normal(size=(4, 3, 20, 4)).astype(np.float32)
    for nzw in (0, 1, 5, 17):
        w = rng.normal(size=nzw).astype(np.float32)
        out = O.convolve_z(F, w, 20 - nzw)
        ref = np.zeros(out.shape, np.float64)
        for jz in range(nzw):
            ref += F[..., jz:jz + 20 - nzw, :].astype(np.float64) * np.float64(w[jz])
        np.testing.assert_allclose(out, ref, rtol=0, atol=4e-7 * max(1, nzw) * np.abs(F).max() * max(1.0, np.abs(w).max(initial=0)))
    np.testing.assert_array_equal(O.convolve_z(F, np.array([2.0], np.float32), 19), 2 * F[..., :19, :])
    # iso heights
    z = np.zeros((4, 6, 4), np.float32)
    z[0, :, 2] = [0, 1, 2, 3, 4, 5]        # crosses 2.5 between iz=2 and 3 -> 3 + 0.5
    z[1, :, 2] = [0, 0, 0, 0, 0, 0]        # never -> -1
    z[2, :, 2] = [9, 8, 7, 6, 5, 4]        # Fz[1] > iso at once: 1 + (2.5-9)/(8-9) = 7.5
    z[3, :, 2] = [0, np.nan, 0, 4, 0, 0]   # NaN never compares greater: crossing at iz=3, from iz=2
    np.testing.assert_array_equal(O.izo_z(z, 2.5), np.array([3.5, -1.0, 7.5, 3.625], np.float32))
