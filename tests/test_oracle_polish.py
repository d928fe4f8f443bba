"""The oracle's Newton polish (test infrastructure; CPU only).

The polish (the kernels' SPM_FLAG_POLISH, not in the reference) takes each
state FIRE stopped at |F| < 1e-5 eV/A to the equilibrium of the interpolated
field.  In FP64 that equilibrium must be the one FP64 FIRE reaches when run to
|F| < 1e-12 eV/A, and the FP32 polish must land within the 1e-4 A bar of it on
the same (FP64-built) grid values rounded to FP32.
"""
import numpy as np

from oracle import oracle as O


def _case(seed=4):
    rng = np.random.default_rng(seed)
    na = 10
    atoms = np.zeros((na, 4))
    atoms[:, :2] = rng.uniform(-2.5, 2.5, (na, 2))
    atoms[:, 2] = rng.normal(0, 0.05, na)
    atoms[:, 3] = rng.uniform(-0.3, 0.3, na)
    R0, E0 = rng.uniform(3.2, 3.5, na), rng.uniform(2e-3, 3e-3, na)
    prm = np.stack([2 * E0 * R0 ** 6, E0 * R0 ** 12], 1)
    n, step, origin = (48, 48, 44), 0.2, np.array([-4.8, -4.8, -3.0])
    p0 = np.array([*origin, 0.0])
    g64 = O.grid_build(0, atoms, prm, n, p0, [step, 0, 0, 0], [0, step, 0, 0], [0, 0, step, 0],
                       [-0.05, 0, 0, 0], [0, 0, 0, 0], prec="f64in")
    dinv = O.dinv_axis_aligned(np.array(n) * step, origin.astype(np.float32), n)
    pts = np.zeros((64, 4), np.float32)
    pts[:, :2] = rng.uniform(-2.0, 2.0, (64, 2))
    pts[:, 2] = 5.5
    return g64, dinv, pts


def test_fp64_polish_reaches_the_tight_fire_equilibrium():
    g64, dinv, pts = _case()
    kw = dict(nz=16, dTip=[0, 0, -0.1, 0], stiffness=[-0.0156, -0.0156, -1.248, 0], dpos0=[0, 0, 0, 0],
              relax=[0.5, 0.1, 0.02, 0.5])
    _, D_pol = O.relax_strokes(g64, dinv, pts, kw["nz"], kw["dTip"], kw["stiffness"], kw["dpos0"], kw["relax"],
                               1000, 1e-10, True, prec="f64", polish=True)
    _, D_loose = O.relax_strokes(g64, dinv, pts, kw["nz"], kw["dTip"], kw["stiffness"], kw["dpos0"], kw["relax"],
                                 1000, 1e-10, True, prec="f64")
    _, D_tight = O.relax_strokes(g64, dinv, pts, kw["nz"], kw["dTip"], kw["stiffness"], kw["dpos0"], kw["relax"],
                                 50000, 1e-24, True, prec="f64")
    slack = np.abs(D_loose[..., :3] - D_tight[..., :3]).max()
    err = np.abs(D_pol[..., :3] - D_tight[..., :3]).max()
    assert slack > 1e-4          # FIRE's stopping slack at |F| < 1e-5 exceeds the bar ...
    assert err < 1e-8            # ... the polish removes it
    # FP32 arithmetic on the FP32-rounded grid
    _, D32 = O.relax_strokes(g64.astype(np.float32), dinv, pts, kw["nz"], kw["dTip"], kw["stiffness"], kw["dpos0"],
                             kw["relax"], 1000, 1e-10, True, prec="f32", polish=True)
    assert np.abs(D32[..., :3] - D_tight[..., :3]).max() < 1e-4


def test_polish_keeps_out_of_range_states_unchanged():
    """A state whose cell is outside the sampler's range (a non-finite coordinate: NaN sample; every finite
    coordinate wraps into the periodic grid) is not moved by the polish."""
    g64, dinv, pts = _case()
    far = pts.copy()
    far[:, 2] = np.inf  # no texel range: NaN samples
    kw = dict(nz=2, dTip=[0, 0, -0.1, 0], stiffness=[-0.0156, -0.0156, -1.248, 0], dpos0=[0, 0, 0, 0],
              relax=[0.5, 0.1, 0.02, 0.5])
    a = O.relax_strokes(g64, dinv, far, kw["nz"], kw["dTip"], kw["stiffness"], kw["dpos0"], kw["relax"], 10, 1e-10,
                        True, prec="f64", polish=True)
    b = O.relax_strokes(g64, dinv, far, kw["nz"], kw["dTip"], kw["stiffness"], kw["dpos0"], kw["relax"], 10, 1e-10,
                        True, prec="f64")
    for x, y in zip(a, b):
        assert np.array_equal(x, y, equal_nan=True)
