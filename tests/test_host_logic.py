"""Host-side logic of the drop-in API that needs no device: scan rasters,
stroke geometry, parameter parsing, oracle physics checks."""
import numpy as np
import pytest

from oracle import oracle as O
from spammm_b200 import AFM
from spammm_b200.FFparams import read_element_types


def test_raster_matches_reference_loop_order():
    """ix-major raster p0 + da*ix + db*iy (spammm/SPM/AFM.py:993-997)."""
    p0 = np.array([0.3, -1.2, 9.0], np.float32)
    da = np.array([0.1, 0.0, 0.0], np.float32)
    db = np.array([0.0, 0.1, 0.0], np.float32)
    pts = AFM._raster_points(p0, da, db, 5, 4)
    k = 0
    for ix in range(5):
        for iy in range(4):
            assert np.array_equal(pts[k, :3], p0 + da * ix + db * iy)
            k += 1
    assert np.all(pts[:, 3] == 0)
    assert np.array_equal(AFM.build_scan_xy_points_vectorized(p0, da, db, 5, 4), pts)


def test_build_scan_points_vectorized_order():
    xs, ys, hs = np.arange(3, dtype=np.float32), np.arange(2, dtype=np.float32) + 10, np.array([5, 6], np.float32)
    pts = AFM.build_scan_points_vectorized(xs, ys, hs)
    assert pts.shape == (12, 4)
    assert np.array_equal(pts[1, :3], [0, 10, 6]) and np.array_equal(pts[2, :3], [0, 11, 5])


def test_scan_fdbm_stroke_geometry():
    """Forward stroke starts at max height + mol_z + bond and descends by dh; reverse ascends (AFM.py:581-600)."""
    self = AFM.AFMulator.__new__(AFM.AFMulator)
    xs, ys = np.array([0., 0.5], np.float32), np.array([1., 2., 3.], np.float32)
    hs = np.array([3.0, 3.1, 3.2, 3.3], np.float32)
    pts, dTip = self._scan_fdbm_points(xs, ys, hs, 1.5, 3.0, np.zeros(3, np.float32), False)
    assert dTip[2] == pytest.approx(-0.1, abs=1e-6)
    assert np.all(pts[:, 2] == np.float32(float(hs.max()) + 1.5 + 3.0))
    assert np.array_equal(pts[:3, 1], ys) and np.all(pts[:3, 0] == 0)
    pts, dTip = self._scan_fdbm_points(xs, ys, hs, 1.5, 3.0, np.zeros(3, np.float32), True)
    assert dTip[2] == pytest.approx(0.1, abs=1e-6)
    assert np.all(pts[:, 2] == np.float32(float(hs.min()) + 1.5 + 3.0))


def test_stiffness_units():
    assert AFM.stiffness_Nm_to_eVA2(16.02176634) == pytest.approx(1.0)
    assert AFM.stiffness_eVA2_to_Nm(AFM.stiffness_Nm_to_eVA2(0.25)) == pytest.approx(0.25)


def test_element_table_parses():
    et = read_element_types()
    for name in ("H", "C", "N", "O", "Na", "Cl"):
        assert name in et and et[name].RvdW > 0 and et[name].EvdW > 0
    assert et["C"].iZ == 6


@pytest.mark.parametrize("kind", [0, 1])
def test_oracle_force_is_minus_energy_gradient(kind):
    rng = np.random.default_rng(3 + kind)
    atoms = np.zeros((4, 4))
    atoms[:, :3] = rng.uniform(-1, 1, (4, 3))
    atoms[:, 3] = rng.uniform(-0.3, 0.3, 4)
    if kind == 0:
        R0, E0 = rng.uniform(3.0, 3.5, 4), rng.uniform(1e-3, 3e-3, 4)
        prm = np.stack([2 * E0 * R0 ** 6, E0 * R0 ** 12], 1)
    else:
        prm = np.stack([rng.uniform(3.0, 3.5, 4), rng.uniform(1e-3, 3e-3, 4), np.full(4, -1.8), np.zeros(4)], 1)
    Qs, QZs = [-0.05, 0.1, 0, 0], [0, 1.2, 0, 0]
    q = rng.uniform(-2, 2, (8, 3)) + np.array([0, 0, 3.0])
    fe = O.pair_fe(kind, atoms, prm, q, Qs, QZs)
    h = 1e-6
    for ax in range(3):
        qp, qm = q.copy(), q.copy()
        qp[:, ax] += h
        qm[:, ax] -= h
        fd = -(O.pair_fe(kind, atoms, prm, qp, Qs, QZs)[:, 3] - O.pair_fe(kind, atoms, prm, qm, Qs, QZs)[:, 3]) / (2 * h)
        np.testing.assert_allclose(fe[:, ax], fd, rtol=1e-6, atol=1e-9)


def test_oracle_grid_cap():
    """Nodes with |E|>100 are rescaled to |E|=100 (kernels/AFM.cl:1053-1054)."""
    atoms = np.array([[0, 0, 0, 0.0]], np.float32)
    prm = np.array([[3.4, 0.003, -1.8, 0]], np.float32)
    g = O.grid_build(1, atoms, prm, (5, 5, 5), [-0.2, -0.2, -0.2, 0], [0.1, 0, 0, 0], [0, 0.1, 0, 0],
                     [0, 0, 0.1, 0], [0, 0, 0, 0], [0, 0, 0, 0])
    E = g[..., 3]
    assert np.abs(E).max() <= 100 + 1e-9
    assert np.isclose(np.abs(E).max(), 100.0)


def test_oracle_fp32_relax_is_deterministic_and_thread_independent():
    rng = np.random.default_rng(5)
    grid = (rng.standard_normal((12, 10, 9, 4)) * 0.01).astype(np.float32)
    dinv = O.dinv_axis_aligned((0.9, 1.0, 1.2), np.zeros(3, np.float32), (9, 10, 12))
    pts = np.zeros((20, 4), np.float32)
    pts[:, :3] = rng.uniform(0, 1, (20, 3))
    args = (grid, dinv, pts, 6, [0, 0, -0.05, 0], [-0.3, -0.3, -1.0, 0], [0, 0, 0, 0], [0.5, 0.1, 0, 0])
    O.set_num_threads(1)
    a = O.relax_strokes(*args)
    O.set_num_threads(4)
    b = O.relax_strokes(*args)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
