"""FDBM stage 4 on the GPU: relaxStrokes2D (AFMulator.scan_fdbm_2d) bit-exact
against the FP32 oracle restatement of kernels/AFM.cl:410-450, and the
compose_and_relax_total caller (AFM_utils.py:3111-3201) in both modes."""
import numpy as np
import pytest

from oracle import oracle as O
from spammm_b200 import AFM, AFM_utils
from spammm_b200.AFM import AFMulator

pytestmark = pytest.mark.gpu


def _field(seed=0, shape=(24, 22, 30)):
    """A smooth random force field (nx,ny,nz,4): sums of a few low-order waves."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = shape
    x, y, z = np.meshgrid(np.arange(nx) / nx, np.arange(ny) / ny, np.arange(nz) / nz, indexing="ij")
    F = np.zeros(shape + (4,), np.float32)
    for c in range(4):
        for _ in range(3):
            k = rng.integers(1, 3, 3)
            ph = rng.uniform(0, 2 * np.pi, 3)
            F[..., c] += 0.05 * rng.normal() * np.cos(2 * np.pi * k[0] * x + ph[0]) * \
                np.cos(2 * np.pi * k[1] * y + ph[1]) * np.cos(np.pi * k[2] * z + ph[2])
    return F


def _expected_2d(afm, F_total, xs, ys, hs, mol_z, K, dt=0.3, damp=0.2):
    heights_desc = np.sort(np.asarray(hs, np.float64))[::-1]
    nz = len(hs)
    dh = float(heights_desc[0] - heights_desc[-1]) / max(nz - 1, 1)
    gx, gy = np.meshgrid(xs, ys, indexing="ij")
    pts = np.zeros((gx.size, 4), np.float32)
    pts[:, 0], pts[:, 1], pts[:, 2] = gx.ravel(), gy.ravel(), float(heights_desc[0]) + mol_z
    grid = np.ascontiguousarray(F_total.transpose(2, 1, 0, 3))
    dinv = (afm.fdbm_dinvA, afm.fdbm_dinvB, afm.fdbm_dinvC)
    FEs, D = O.relax_2d(grid, dinv, pts, nz, K, np.float32(dh), dt, damp, afm.n_relax_max, afm.f2conv, flip=True)
    return FEs.reshape(len(xs), len(ys), nz, 4), D.reshape(len(xs), len(ys), nz, 4)


@pytest.mark.parametrize("K", [0.03, 0.0])
def test_scan_fdbm_2d_matches_oracle(cuda, K):
    F_total = _field(1)
    afm = AFMulator(use_morse=False, use_fire=False)
    origin = np.array([-3., -2.75, -1.0], np.float32)
    afm.setup_fdbm_grid(F_total, origin, 0.25)
    xs = np.linspace(-1.5, 1.5, 9).astype(np.float32)
    ys = np.linspace(-1.2, 1.2, 7).astype(np.float32)
    hs = np.linspace(2.0, 3.5, 7).astype(np.float32)
    FEs, disp = afm.scan_fdbm_2d(xs, ys, hs, mol_z=0.3, K_LAT=K)
    oFE, oD = _expected_2d(afm, F_total, xs, ys, hs, 0.3, K)
    assert FEs.shape == (9, 7, 7, 4) and FEs.dtype == np.float32
    assert np.array_equal(FEs, oFE)
    assert np.array_equal(disp["dx"], oD[..., 0]) and np.array_equal(disp["dy"], oD[..., 1])
    assert not disp["dz"].any()
    if K > 0:
        assert np.abs(disp["dx"]).max() > 1e-4  # the probe moved


def test_scan_fdbm_2d_step_cap_and_convergence(cuda):
    F_total = _field(2)
    origin = np.array([-3., -2.75, -1.0], np.float32)
    xs = np.linspace(-1, 1, 5).astype(np.float32)
    hs = np.linspace(2.0, 3.0, 5).astype(np.float32)
    for n_max, f2 in ((1, 1e-8), (7, 1e-8), (200, 1e-14), (0, 1e-8)):
        afm = AFMulator(use_morse=False, use_fire=False)
        afm.n_relax_max, afm.f2conv = n_max, f2
        afm.setup_fdbm_grid(F_total, origin, 0.25)
        FEs, disp = afm.scan_fdbm_2d(xs, xs, hs, mol_z=0.0, K_LAT=0.02)
        oFE, oD = _expected_2d(afm, F_total, xs, xs, hs, 0.0, 0.02)
        assert np.array_equal(FEs, oFE) and np.array_equal(disp["dx"], oD[..., 0]), (n_max, f2)


def test_compose_and_relax_total_both_modes(cuda):
    F_total = _field(3)
    origin = np.array([-3., -2.75, -1.0], np.float32)
    step = 0.25
    xs = np.linspace(-1.5, 1.5, 7).astype(np.float32)
    ys = np.linspace(-1.0, 1.0, 5).astype(np.float32)
    hs = np.linspace(1.5, 3.0, 6).astype(np.float32)
    atomPos = np.array([[0., 0., -0.5], [0.5, 0.2, 0.1]])
    # 2-D lateral mode: scan_fdbm_2d + compute_df_dir
    df, tip, FEs = AFM_utils.compose_and_relax_total(F_total, xs, ys, hs, origin, step, atomPos, K_LAT=0.03)
    afm = AFMulator(use_morse=False, use_fire=False)
    afm.setup_fdbm_grid(F_total, origin, step)
    oFE, oD = _expected_2d(afm, F_total, xs, ys, hs, 0.1, 0.03)
    assert np.array_equal(FEs, oFE) and np.array_equal(tip["dx"], oD[..., 0])
    spacing = (float(xs[1] - xs[0]), float(ys[1] - ys[0]), float(hs[1] - hs[0]))
    np.testing.assert_allclose(df, O.compute_df_dir(oFE, spacing, (0., 0., 1.)), rtol=1e-6, atol=1e-9)
    # PPM mode: scan_fdbm (relaxStrokes with the radial bond) + compute_df_dir
    df2, tip2, FEs2 = AFM_utils.compose_and_relax_total(F_total, xs, ys, hs, origin, step, atomPos, K_LAT=0.03,
                                                        K_RAD=20.0, bond_length=4.0, ppm_mode=True)
    afm2 = AFMulator(use_morse=False, use_fire=True)
    afm2.setup_fdbm_grid(F_total, origin, step)
    ref, rtip = afm2.scan_fdbm(xs, ys, hs, mol_z=0.1, K_LAT=0.03, K_RAD=20.0, bond_length=4.0, ppm_mode=True)
    assert np.array_equal(FEs2, ref) and np.array_equal(tip2["dz"], rtip["dz"])
    np.testing.assert_allclose(df2, AFM.compute_df_dir(ref, spacing, (0., 0., 1.)), rtol=0, atol=0)
    with pytest.raises(NotImplementedError):
        AFM_utils.compose_and_relax_total(F_total, xs, ys, hs, origin, step, atomPos, use_gpu_relax=False)
