"""Differentiable grid path: GPU implicit adjoint vs (1) an independent FP64
torch-autograd implementation of the implicit gradient and (2) central finite
differences of the FP64 oracle pipeline (grid build + relaxation converged to
|F| < 1e-12).  Forward relaxation bit-identical to the FP32 oracle.

Tolerances: adjoint at the FP64 equilibria vs FP64 torch autograd: 2e-4
relative per parameter block; vs finite differences (h = 1e-4, random
direction): 1e-4 relative; end to end (FP32 forward equilibria, |F|<1e-5):
1e-2 relative (the FP32 equilibrium itself moves by ~1e-5/k_xy).
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from spammm_b200 import _lib, gpu
from spammm_b200.diff import GridAFM, GridScanSpec, df_loss

pytestmark = pytest.mark.gpu

KXY = 0.25 / 16.02176634
KZ = 20.0 / 16.02176634


def _system(kind, seed=5, na=8):
    rng = np.random.default_rng(seed)
    atoms = np.zeros((na, 4))
    atoms[:, :2] = rng.uniform(-2.0, 2.0, (na, 2))
    atoms[:, 2] = rng.normal(0, 0.05, na)
    atoms[:, 3] = rng.uniform(-0.3, 0.3, na)
    atoms[:, 3] -= atoms[:, 3].mean()
    R0, E0 = rng.uniform(3.2, 3.5, na), rng.uniform(2e-3, 3e-3, na)
    if kind == 0:
        prm = np.stack([2 * E0 * R0 ** 6, E0 * R0 ** 12], 1)
    else:
        prm = np.stack([R0, E0, np.full(na, -1.8), np.zeros(na)], 1)
    return atoms.astype(np.float32).astype(np.float64), prm.astype(np.float32).astype(np.float64)


def _spec(kind, nxy=(5, 4), nz=8):
    pts = np.zeros((nxy[0] * nxy[1], 4), np.float32)
    k = 0
    for ix in range(nxy[0]):
        for iy in range(nxy[1]):
            pts[k, :3] = (-1.0 + 0.45 * ix, -0.8 + 0.5 * iy, 4.6)
            k += 1
    return GridScanSpec(kind=kind, ngrid=(40, 40, 44), origin=np.array([-5.0, -5.0, -4.0]), step=0.25, points=pts,
                        nz=nz, dtip=-0.1, raster_ny=nxy[1])


def _stiff():
    return np.array([-KXY, -KXY, -KZ, 0.0], np.float32)


def _oracle_pipeline(kind, atoms, prm, stiff, spec, prec="f64", f2conv=1e-24, max_iter=20000):
    p0, dA, dB, dC = spec.vectors()
    grid = O.grid_build(kind, atoms, prm, spec.ngrid, p0, dA, dB, dC, spec.tipQs, spec.tipQZs,
                        prec="f64in" if prec == "f64" else "f32")
    FEs, PPs = O.relax_pp(grid, spec.dinv(), spec.points, spec.nz, [1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 1, spec.dtip],
                          stiff, spec.dpos0, spec.relax_params, [0, 0, 0, 0], max_iter, f2conv, True, prec=prec)
    return grid, FEs, PPs


def _target(spec, seed=1):
    rng = np.random.default_rng(seed)
    return rng.normal(0, 0.02, (spec.points.shape[0], spec.nz))


def _loss_np(FEs, tgt, dtip):
    Fz = FEs[..., 2]
    df = np.zeros_like(Fz)
    df[:, 1:-1] = -(Fz[:, 2:] - Fz[:, :-2]) / (2 * abs(dtip))
    w = np.ones_like(Fz)
    w[:, 0] = w[:, -1] = 0
    return 0.5 * np.sum(w * (df - tgt) ** 2) / w.sum()


def _torch_implicit_grad(kind, atoms, prm, stiff, spec, PPs, u):
    """Independent FP64 implicit gradient: grid build, trilinear sampling and
    spring in torch ops; J and b by autograd; lambda by torch.linalg.solve."""
    dt = torch.float64
    A = torch.tensor(atoms, dtype=dt, requires_grad=True)
    Pm = torch.tensor(prm, dtype=dt, requires_grad=True)
    K = torch.tensor(np.asarray(stiff, np.float64), dtype=dt, requires_grad=True)
    nx, ny, nz = spec.ngrid
    p0, dA, dB, dC = spec.vectors()
    ix = torch.arange(nx, dtype=dt)
    iy = torch.arange(ny, dtype=dt)
    iz = torch.arange(nz, dtype=dt)
    Z, Y, X = torch.meshgrid(iz, iy, ix, indexing="ij")
    nodes = torch.stack([p0[0] + X * float(dA[0]), p0[1] + Y * float(dB[1]), p0[2] + Z * float(dC[2])], -1)
    dp = nodes[..., None, :] - A[:, :3]                     # (nz,ny,nx,na,3)
    r2 = (dp * dp).sum(-1) + 1e-4
    if kind == 0:
        ir2 = 1.0 / r2
        ir6 = ir2 ** 3
        E = ((Pm[:, 1] * ir6 - Pm[:, 0]) * ir6)
        s = (12 * Pm[:, 1] * ir6 - 6 * Pm[:, 0]) * ir6 * ir2
    else:
        r = torch.sqrt(r2)
        e = torch.exp(Pm[:, 2] * (r - Pm[:, 0]))
        E = Pm[:, 1] * e * (e - 2)
        s = -(2 * Pm[:, 2] * Pm[:, 1] * e * (e - 1)) / r
    F = (dp * s[..., None]).sum(-2)
    Et = E.sum(-1)
    qs = float(spec.tipQs[0]) * 14.3996448915
    ir = 1.0 / torch.sqrt(r2)
    Ec = qs * A[:, 3] * ir
    F = F + (dp * (Ec * ir * ir)[..., None]).sum(-2)
    Et = Et + Ec.sum(-1)
    grid = torch.cat([F, Et[..., None]], -1)  # (nz,ny,nx,4) uncapped; the states touch no capped node
    dinv = spec.dinv()
    q = torch.tensor(PPs[:, :3], dtype=dt, requires_grad=True)

    def sample(qq):
        out = []
        idx = []
        for d, n in zip(range(3), (nx, ny, nz)):
            uu = qq[:, d] * float(dinv[d][d]) + float(dinv[d][3])
            ss = uu - torch.floor(uu)
            t = ss * n - 0.5
            fi = torch.floor(t)
            a = t - fi
            i0 = fi.long() % n
            idx.append((i0, (i0 + 1) % n))
            out.append(a)
        (x0, x1), (y0, y1), (z0, z1) = idx
        ax, ay, az = [v[:, None] for v in out]
        c00 = grid[z0, y0, x0] * (1 - ax) + grid[z0, y0, x1] * ax
        c10 = grid[z0, y1, x0] * (1 - ax) + grid[z0, y1, x1] * ax
        c01 = grid[z1, y0, x0] * (1 - ax) + grid[z1, y0, x1] * ax
        c11 = grid[z1, y1, x0] * (1 - ax) + grid[z1, y1, x1] * ax
        return (c00 * (1 - ay) + c10 * ay) * (1 - az) + (c01 * (1 - ay) + c11 * ay) * az

    n_scan = spec.points.shape[0]
    tips = torch.tensor(spec.points[:, :3], dtype=dt).repeat_interleave(spec.nz, 0)
    tips = tips + torch.arange(spec.nz, dtype=dt).repeat(n_scan)[:, None] * torch.tensor([0, 0, spec.dtip], dtype=dt)

    def G_of(qq, KK):
        fe = sample(qq)
        return fe[:, :3] + (qq - tips) * KK[:3], fe

    Gq, fe = G_of(q, K)
    U = torch.tensor(u, dtype=dt)
    J = torch.zeros((q.shape[0], 3, 3), dtype=dt)
    for i in range(3):
        (gi,) = torch.autograd.grad(Gq[:, i].sum(), q, retain_graph=True)
        J[:, i, :] = gi
    (bvec,) = torch.autograd.grad((fe * U).sum(), q, retain_graph=True)
    lam = torch.linalg.solve(J.transpose(1, 2), bvec[..., None])[..., 0].detach()
    S = (fe * U).sum() - (lam * Gq).sum()
    gA, gP, gK = torch.autograd.grad(S, [A, Pm, K])
    return gA.numpy(), gP.numpy(), gK.numpy()


def _gpu_grads(kind, atoms, prm, stiff, spec, PPs=None, u=None):
    """GPU adjoint; with PPs/u given, evaluated at those equilibria (bypassing the forward)."""
    p0, dA, dB, dC = spec.vectors()
    a32 = torch.tensor(atoms, dtype=torch.float32, device="cuda")
    p32 = torch.tensor(prm, dtype=torch.float32, device="cuda")
    grid = gpu.grid_build(kind, a32, p32, spec.ngrid, p0, dA, dB, dC, spec.tipQs, spec.tipQZs)
    P = spec.scan_params(stiff)
    pts = torch.tensor(spec.points, device="cuda")
    PPs_t = torch.tensor(np.asarray(PPs, np.float32).reshape(-1, 4), device="cuda")
    u_t = torch.tensor(np.asarray(u, np.float32).reshape(-1, 4), device="cuda")
    ubar, dk, diag = gpu.adjoint_grid_state(grid, P, pts, PPs_t, u_t)
    assert int((diag[:, 3] != 0).sum()) == 0, diag[diag[:, 3] != 0][:4]
    g, dks = gpu.adjoint_grid_params(kind, a32, p32, p0, dA, dB, dC, spec.tipQs, spec.tipQZs, grid, P, PPs_t, ubar,
                                     dk)
    g = g.cpu().numpy()
    gA = np.zeros_like(atoms)
    gA[:, :3] = g[:, :3]
    gA[:, 3] = g[:, 5]
    gP = np.zeros_like(prm)
    gP[:, 0], gP[:, 1] = g[:, 3], g[:, 4]
    return gA, gP, dks.cpu().numpy()


def _rel(a, b):
    return np.abs(a - b).max() / (np.abs(b).max() + 1e-300)


@pytest.mark.parametrize("kind", [0, 1])
def test_grid_pp_forward_bit_exact(cuda, kind):
    atoms, prm = _system(kind)
    spec = _spec(kind)
    stiff = _stiff()
    p0, dA, dB, dC = spec.vectors()
    grid = gpu.grid_build(kind, atoms.astype(np.float32), prm.astype(np.float32), spec.ngrid, p0, dA, dB, dC,
                          spec.tipQs, spec.tipQZs)
    P = spec.scan_params(stiff)
    FEs, PPs = gpu.relax_pp(grid, P, torch.tensor(spec.points, device="cuda"))
    oFE, oPP = O.relax_pp(grid.cpu().numpy(), spec.dinv(), spec.points, spec.nz, [1, 0, 0, 0], [0, 1, 0, 0],
                          [0, 0, 1, spec.dtip], stiff, spec.dpos0, spec.relax_params, [0, 0, 0, 0], spec.max_iter,
                          spec.f2conv, True)
    assert np.array_equal(FEs.cpu().numpy(), oFE) and np.array_equal(PPs.cpu().numpy(), oPP)
    assert (oPP[..., 3] > 0).all()


@pytest.mark.parametrize("kind", [0, 1])
def test_grid_adjoint_matches_fp64_autograd_and_finite_differences(cuda, kind):
    atoms, prm = _system(kind, seed=11 + kind)
    spec = _spec(kind)
    stiff = _stiff().astype(np.float64)
    tgt = _target(spec)
    grid64, FEs, PPs = _oracle_pipeline(kind, atoms, prm, stiff, spec)
    assert (PPs[..., 3] > 0).all()
    FEs = FEs.reshape(-1, spec.nz, 4)
    # u = dL/dFEs of the df loss (torch autograd of the same loss formula)
    F_t = torch.tensor(FEs, requires_grad=True)
    L = df_loss(F_t, torch.tensor(tgt), spec.dtip)
    (u,) = torch.autograd.grad(L, F_t)
    u = u.numpy().reshape(-1, 4)
    PPf = PPs.reshape(-1, 4)
    tA, tP, tK = _torch_implicit_grad(kind, atoms, prm, stiff, spec, PPf, u)
    gA, gP, gK = _gpu_grads(kind, atoms, prm, stiff, spec, PPs=PPf, u=u)
    assert _rel(gA[:, :3], tA[:, :3]) < 2e-4, (gA[:, :3], tA[:, :3])
    assert _rel(gA[:, 3], tA[:, 3]) < 2e-4
    assert _rel(gP[:, :2], tP[:, :2]) < 2e-4
    assert _rel(gK[:3], tK[:3]) < 2e-4
    # central finite differences of the FP64 oracle pipeline along a random direction
    rng = np.random.default_rng(7)
    va = rng.normal(0, 1, atoms.shape)
    vp = rng.normal(0, 1, prm.shape) * np.abs(prm) * 1e-2
    if kind == 1:
        vp[:, 2:] = 0
    vk = np.array([1.0, 1.0, 0.0, 0.0]) * 1e-2 * KXY
    h = 1e-4

    def L_at(s):
        _, F, _ = _oracle_pipeline(kind, atoms + s * va, prm + s * vp, stiff + s * vk, spec)
        return _loss_np(F.reshape(-1, spec.nz, 4), tgt, spec.dtip)

    fd = (L_at(h) - L_at(-h)) / (2 * h)
    dirg = float((gA * va).sum() + (gP * vp).sum() + (gK * vk).sum())
    dirt = float((tA * va).sum() + (tP * vp).sum() + (tK * vk).sum())
    assert abs(dirt - fd) / abs(fd) < 1e-4, (dirt, fd)
    assert abs(dirg - fd) / abs(fd) < 1e-4, (dirg, fd)


def test_grid_afm_autograd_end_to_end(cuda):
    """torch.autograd through GridAFM (FP32 forward equilibria) vs FP64 finite differences."""
    kind = 0
    atoms, prm = _system(kind, seed=21)
    spec = _spec(kind)
    tgt = _target(spec, seed=3)
    A = torch.tensor(atoms, dtype=torch.float32, device="cuda", requires_grad=True)
    Pm = torch.tensor(prm, dtype=torch.float32, device="cuda", requires_grad=True)
    kxy = torch.tensor(KXY, dtype=torch.float64, device="cuda", requires_grad=True)
    stiff = torch.stack([-kxy, -kxy, torch.tensor(-KZ, dtype=torch.float64, device="cuda"),
                         torch.tensor(0.0, dtype=torch.float64, device="cuda")])
    FEs = GridAFM.apply(A, Pm, stiff, spec)
    L = df_loss(FEs, torch.tensor(tgt, device="cuda"), spec.dtip)
    L.backward()
    gA = A.grad.double().cpu().numpy()
    gk = float(kxy.grad)
    rng = np.random.default_rng(9)
    va = rng.normal(0, 1, atoms.shape)
    h = 1e-4

    def L_at(s, dk=0.0):
        st = np.array([-(KXY + dk), -(KXY + dk), -KZ, 0.0])
        _, F, _ = _oracle_pipeline(kind, atoms + s * va, prm, st, spec)
        return _loss_np(F.reshape(-1, spec.nz, 4), tgt, spec.dtip)

    fd = (L_at(h) - L_at(-h)) / (2 * h)
    assert abs(float((gA * va).sum()) - fd) / abs(fd) < 1e-2
    hk = 1e-5 * KXY
    fdk = (L_at(0.0, hk) - L_at(0.0, -hk)) / (2 * hk)
    assert abs(gk - fdk) / abs(fdk) < 1e-2, (gk, fdk)
