"""Gradients of the differentiable grid path on the 38-atom workload: the
config-0 molecule (C24 O6 H8, LJ), 200^3 grid at 0.1 A, 100x100 pixels x 40
z-steps; target df image from the molecule with positions perturbed by
N(0, 0.1 A) and charges by N(0, 0.05 e); loss = the df loss of df_loss_seed
(spammm/SPM/AFM.py:3125-3200) over the whole 100x100x40 volume; gradients with
respect to the 38x3 positions, 38 charges, 38x2 LJ parameters (c6, c12) and
k_xy.

GPU (FP32 forward with the Newton polish, FP32 implicit adjoint through the
relaxation and the grid build) against two FP64 references
(tests/implicit_fp64.py):
  * FP64 torch autograd of the implicit-function gradient at the FP64
    equilibria: relative error of each parameter block (norm of the
    difference / norm of the reference) < 1e-4;
  * central finite differences of the polished FP64 oracle pipeline along a
    random direction per block, h = 1e-3, 1e-4, 1e-5 (in A for positions, e for
    the zero-sum charge direction, relative for c6, c12 and k_xy): the
    directional derivative at the plateau (the smallest h) within 1e-4, the
    error not growing as h shrinks (the reference's gate,
    tests/SPM/test_afm_morse.py:1523-1590).
"""
import numpy as np
import pytest
import torch

import implicit_fp64 as I
from spammm_b200 import synthetic
from spammm_b200.diff import GridAFM, GridScanSpec, df_loss

pytestmark = pytest.mark.gpu

TOL = 1e-4


def _workload():
    cfg = synthetic.plain_small()
    gx, gy = np.meshgrid(cfg.scan_xs, cfg.scan_ys, indexing="ij")
    pts = np.zeros((cfg.n_pix, 4), np.float32)
    pts[:, 0], pts[:, 1], pts[:, 2] = gx.ravel(), gy.ravel(), np.float32(cfg.z_top)
    geom = dict(ngrid=cfg.ngrid, origin=np.asarray(cfg.origin, np.float64), step=cfg.step, points=pts, nz=cfg.nz,
                dtip=-cfg.dz, tipQs=cfg.tipQs)
    atoms = cfg.atoms.astype(np.float64)
    prm = cfg.params.astype(np.float64)
    stiff = cfg.stiffness.astype(np.float64)
    rng = np.random.default_rng(2026)
    pert = atoms.copy()
    pert[:, :3] += rng.normal(0, 0.1, (len(atoms), 3))
    pert[:, 3] += rng.normal(0, 0.05, len(atoms))
    FE_t, PP_t = I.oracle_forward(cfg.kind, pert, prm, stiff, geom)
    assert (PP_t[..., 3] > 0).all()
    Fz = FE_t[..., 2]
    target = np.zeros_like(Fz)
    target[:, 1:-1] = -(Fz[:, 2:] - Fz[:, :-2]) / (2 * cfg.dz)
    return cfg, geom, atoms, prm, stiff, target, rng


def _gpu_grad(cfg, geom, atoms, prm, stiff, target):
    spec = GridScanSpec(kind=cfg.kind, ngrid=cfg.ngrid, origin=np.asarray(cfg.origin), step=cfg.step,
                        points=geom["points"], nz=cfg.nz, dtip=-cfg.dz, tipQs=cfg.tipQs, max_iter=cfg.max_iter,
                        f2conv=cfg.f2conv, raster_ny=len(cfg.scan_ys), polish=True, strict=True)
    A = torch.tensor(atoms, device="cuda", requires_grad=True)
    P = torch.tensor(prm, device="cuda", requires_grad=True)
    K = torch.tensor(stiff, device="cuda", requires_grad=True)
    FEs = GridAFM.apply(A, P, K, spec)
    L = df_loss(FEs, torch.tensor(target, device="cuda"), -cfg.dz)
    L.backward()
    return A.grad.cpu().numpy(), P.grad.cpu().numpy(), K.grad.cpu().numpy(), float(L)


def _rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / np.linalg.norm(np.ravel(b)))


def test_grid_gradients_vs_fp64_autograd_and_finite_differences(cuda):
    cfg, geom, atoms, prm, stiff, target, rng = _workload()
    na = len(atoms)
    gA, gP, gK, L_gpu = _gpu_grad(cfg, geom, atoms, prm, stiff, target)
    FE64, PP64 = I.oracle_forward(cfg.kind, atoms, prm, stiff, geom)
    assert (PP64[..., 3] > 0).all()
    tA, tP, tK, L64 = I.torch_implicit_grad(cfg.kind, atoms, prm, stiff, geom, PP64, target)
    kxy = lambda k: -(k[0] + k[1])  # noqa: E731  d/dk_xy with stiffness = (-k_xy, -k_xy, -k_z, 0)
    blocks = {"positions": (gA[:, :3], tA[:, :3]), "charges": (gA[:, 3], tA[:, 3]), "c6": (gP[:, 0], tP[:, 0]),
              "c12": (gP[:, 1], tP[:, 1]), "k_xy": (kxy(gK), kxy(tK))}
    print(f"\nloss: GPU {L_gpu:.9e}  FP64 {L64:.9e}")
    errs = {}
    for name, (g, t) in blocks.items():
        errs[name] = _rel(g, t)
        print(f"{name:10s} GPU vs FP64 torch autograd: {errs[name]:.2e}")
    # finite differences of the FP64 oracle pipeline, one random direction per block
    q = rng.normal(size=na)
    zero_a, zero_p = np.zeros_like(atoms), np.zeros_like(prm)
    dirs = {
        "positions": (np.concatenate([rng.normal(size=(na, 3)), np.zeros((na, 1))], 1), zero_p, 0.0),
        "charges": (np.concatenate([np.zeros((na, 3)), (q - q.mean())[:, None]], 1), zero_p, 0.0),
        "c6": (zero_a, np.stack([prm[:, 0] * rng.normal(size=na), np.zeros(na)], 1), 0.0),
        "c12": (zero_a, np.stack([np.zeros(na), prm[:, 1] * rng.normal(size=na)], 1), 0.0),
        "k_xy": (zero_a, zero_p, 1.0),
    }
    kdir = np.array([stiff[0], stiff[0], 0.0, 0.0])  # d stiffness per relative step of k_xy
    fd_errs = {}
    for name, (va, vp, vk) in dirs.items():
        vK = vk * kdir
        g_gpu = float((gA * va).sum() + (gP * vp).sum() + (gK * vK).sum())
        g_t = float((tA * va).sum() + (tP * vp).sum() + (tK * vK).sum())
        rel = []
        for h in (1e-3, 1e-4, 1e-5):
            fd = (I.oracle_loss(cfg.kind, atoms + h * va, prm + h * vp, stiff + h * vK, geom, target) -
                  I.oracle_loss(cfg.kind, atoms - h * va, prm - h * vp, stiff - h * vK, geom, target)) / (2 * h)
            rel.append((abs(g_gpu - fd) / abs(fd), abs(g_t - fd) / abs(fd)))
        fd_errs[name] = rel
        print(f"{name:10s} directional FD (h=1e-3,1e-4,1e-5): GPU rel " +
              ", ".join(f"{r[0]:.2e}" for r in rel) + " | FP64 autograd rel " + ", ".join(f"{r[1]:.2e}" for r in rel))
    for name in blocks:
        assert errs[name] < TOL, f"{name}: GPU vs FP64 autograd {errs[name]:.2e}"
        rel = fd_errs[name]
        assert rel[2][1] < 1e-5, f"{name}: the FP64 references disagree ({rel[2][1]:.2e})"  # measured <= 1.1e-6
        assert rel[2][0] < TOL, f"{name}: GPU vs FD at h=1e-5 {rel[2][0]:.2e}"
        assert rel[1][0] <= 10 * rel[0][0] + TOL and rel[2][0] <= 10 * rel[1][0] + TOL, f"{name}: no plateau {rel}"
