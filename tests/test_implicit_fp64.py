"""The two FP64 gradient references of the grid path (tests/implicit_fp64.py)
agree with each other on a small system, on the CPU: the torch-autograd
implicit gradient at the FP64 equilibria against central finite differences of
the polished FP64 oracle pipeline, per parameter block (positions, zero-sum
charges, c6, c12, k_xy), with the error falling as h goes 1e-3 -> 1e-4 ->
1e-5 (the plateau of the reference's own gate, tests/SPM/test_afm_morse.py:
1523-1590) and within 1e-7 relative at h = 1e-5.  The GPU adjoint is compared
with both at the 38-atom workload in test_gpu_diff_config2.py.
"""
import numpy as np

import implicit_fp64 as I

KXY, KZ = 0.25 / 16.02176634, 20 / 16.02176634


def _toy(seed=5, na=8):
    rng = np.random.default_rng(seed)
    atoms = np.zeros((na, 4))
    atoms[:, :2] = rng.uniform(-2, 2, (na, 2))
    atoms[:, 2] = rng.normal(0, .05, na)
    atoms[:, 3] = rng.uniform(-.3, .3, na)
    atoms[:, 3] -= atoms[:, 3].mean()
    R0, E0 = rng.uniform(3.2, 3.5, na), rng.uniform(2e-3, 3e-3, na)
    prm = np.stack([2 * E0 * R0 ** 6, E0 * R0 ** 12], 1)
    pts = np.zeros((20, 4), np.float32)
    for k, (ix, iy) in enumerate((ix, iy) for ix in range(5) for iy in range(4)):
        pts[k, :3] = (-1.0 + 0.45 * ix, -0.8 + 0.5 * iy, 4.6)
    geom = dict(ngrid=(40, 40, 44), origin=np.array([-5., -5., -4.]), step=0.25, points=pts, nz=8, dtip=-0.1,
                tipQs=np.array([-0.05, 0, 0, 0], np.float32))
    return atoms, prm, geom, rng.normal(0, 0.02, (20, 8)), rng


def test_torch_implicit_gradient_matches_oracle_finite_differences():
    atoms, prm, geom, tgt, rng = _toy()
    stiff = np.array([-KXY, -KXY, -KZ, 0.0])
    FEs, PPs = I.oracle_forward(0, atoms, prm, stiff, geom)
    gA, gP, dk, L = I.torch_implicit_grad(0, atoms, prm, stiff, geom, PPs, tgt)
    assert abs(L - I.df_loss_np(FEs, tgt, geom["dtip"])) < 1e-15
    q = rng.normal(size=8)
    blocks = {
        "positions": (np.concatenate([rng.normal(size=(8, 3)), np.zeros((8, 1))], 1), None),
        "charges": (np.concatenate([np.zeros((8, 3)), (q - q.mean())[:, None]], 1), None),
        "c6": (None, np.stack([prm[:, 0] * rng.normal(size=8), np.zeros(8)], 1)),
        "c12": (None, np.stack([np.zeros(8), prm[:, 1] * rng.normal(size=8)], 1)),
    }
    for name, (va, vp) in blocks.items():
        va = np.zeros_like(atoms) if va is None else va
        vp = np.zeros_like(prm) if vp is None else vp
        g_dir = float((gA * va).sum() + (gP * vp).sum())
        rel = []
        for h in (1e-3, 1e-4, 1e-5):
            fd = (I.oracle_loss(0, atoms + h * va, prm + h * vp, stiff, geom, tgt) -
                  I.oracle_loss(0, atoms - h * va, prm - h * vp, stiff, geom, tgt)) / (2 * h)
            rel.append(abs(g_dir - fd) / abs(fd))
        assert rel[2] < 1e-7, (name, rel)
        assert rel[1] <= 10 * rel[0] + 1e-9 and rel[2] <= 10 * rel[1] + 1e-9, (name, rel)
    vk = np.array([-KXY, -KXY, 0.0, 0.0])  # d/dk_xy, relative step
    g_dir = float((dk * vk).sum())
    fd = (I.oracle_loss(0, atoms, prm, stiff + 1e-5 * vk, geom, tgt) -
          I.oracle_loss(0, atoms, prm, stiff - 1e-5 * vk, geom, tgt)) / 2e-5
    assert abs(g_dir - fd) / abs(fd) < 1e-7
