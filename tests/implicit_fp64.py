"""Test infrastructure: two FP64 references for the gradient of the grid
path's df loss, independent of the CUDA adjoint.

* ``oracle_loss``: the FP64 oracle pipeline -- grid build from FP64 atoms,
  FIRE relaxation with the direct path's bookkeeping (convergence tested before
  each update) stopped at |F| < 1e-5 eV/A and Newton-polished to the
  equilibrium of the interpolated field, df loss -- for central finite
  differences.
* ``torch_implicit_grad``: the implicit-function gradient at the FP64
  equilibria in FP64 torch autograd.  Grid values only at the cell corners the
  states touch (g(theta) evaluated from the pair laws), trilinear sample and
  spring as torch functions of (q, theta); dL/dq|theta and J = dG/dq by
  autograd, J^T lambda = dL/dq by torch.linalg.solve, and
  dL/dtheta = dL/dtheta|q - lambda . dG/dtheta|q by autograd through the grid
  values (chunked over nodes).  No FIRE trajectory is differentiated.

The loss is the reference's df_loss_seed (spammm/SPM/AFM.py:3125-3200):
df = -(Fz[iz+1] - Fz[iz-1]) / (2|dtip|) inside each stroke,
L = 0.5 sum(w (df - t)^2) / sum(w), w = 1 inside and 0 on each stroke's first
and last z-step.  Strokes are z-strokes with an identity probe frame and an
axis-aligned grid; the probe carries one charge site at the probe position.
"""
import numpy as np
import torch

from oracle import oracle as O

COULOMB = 14.3996448915


def df_loss_np(FEs, target, dtip):
    Fz = FEs[..., 2].astype(np.float64)
    df = np.zeros_like(Fz)
    df[:, 1:-1] = -(Fz[:, 2:] - Fz[:, :-2]) / (2 * abs(dtip))
    w = np.ones_like(Fz)
    w[:, 0] = w[:, -1] = 0
    return 0.5 * np.sum(w * (df - target) ** 2) / w.sum()


def dinv_of(ngrid, origin, step):
    L = np.array(ngrid, dtype=np.float64) * step
    o = np.asarray(origin, np.float32)
    return (np.array([1. / L[0], 0., 0., -o[0] / L[0] + 0.5 / ngrid[0]], np.float32),
            np.array([0., 1. / L[1], 0., -o[1] / L[1] + 0.5 / ngrid[1]], np.float32),
            np.array([0., 0., 1. / L[2], -o[2] / L[2] + 0.5 / ngrid[2]], np.float32))


def oracle_forward(kind, atoms, params, stiff, geom, max_iter=1000, f2conv=1e-10):
    """FP64 grid + FP64 polished PP relaxation -> FEs, PPs (n_scan, nz, 4) float64."""
    ngrid, origin, step, pts, nz, dtip, Qs = (geom[k] for k in ("ngrid", "origin", "step", "points", "nz", "dtip",
                                                                "tipQs"))
    p0 = np.array([origin[0], origin[1], origin[2], 0.0])
    g = O.grid_build(kind, atoms, params, ngrid, p0, [step, 0, 0, 0], [0, step, 0, 0], [0, 0, step, 0], Qs,
                     [0, 0, 0, 0], prec="f64in")
    return O.relax_pp(g, dinv_of(ngrid, origin, step), pts, nz, [1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 1, dtip], stiff,
                      [0, 0, 0, 0], [0.5, 0.1, 0.02, 0.5], [0, 0, 0, 0], max_iter, f2conv, True, prec="f64",
                      polish=True)


def oracle_loss(kind, atoms, params, stiff, geom, target):
    FEs, PPs = oracle_forward(kind, atoms, params, stiff, geom)
    assert (PPs[..., 3] > 0).all(), "FP64 oracle: a state did not converge"
    return df_loss_np(FEs, target, geom["dtip"])


def _pair_values(kind, nodes, A, P, qs):
    """(n, 4) grid values (F, E) at FP64 node positions from atoms A (na,4) and params P: the pair law plus
    the probe charge qs * COULOMB at the node, uncapped (the states used touch no capped node)."""
    dp = nodes[:, None, :] - A[None, :, :3]
    r2 = (dp * dp).sum(-1) + 1e-4
    if kind == 0:
        ir2 = 1.0 / r2
        ir6 = ir2 ** 3
        E = (P[:, 1] * ir6 - P[:, 0]) * ir6
        s = (12 * P[:, 1] * ir6 - 6 * P[:, 0]) * ir6 * ir2
    else:
        r = torch.sqrt(r2)
        e = torch.exp(P[:, 2] * (r - P[:, 0]))
        E = P[:, 1] * e * (e - 2)
        s = -(2 * P[:, 2] * P[:, 1] * e * (e - 1)) / r
    ir = torch.rsqrt(r2)
    Ec = (qs * COULOMB) * A[:, 3] * ir
    s = s + Ec * ir * ir
    F = (dp * s[..., None]).sum(1)
    return torch.cat([F, (E + Ec).sum(1, keepdim=True)], 1)


def torch_implicit_grad(kind, atoms, params, stiff, geom, PPs, target, chunk=20000):
    """dL/d(atoms (na,4), params (na,2|4), stiffness (4,)) in FP64 at the equilibria PPs (n_scan, nz, 4)."""
    dt = torch.float64
    ngrid, origin, step, nz, dtip, pts = (geom[k] for k in ("ngrid", "origin", "step", "nz", "dtip", "points"))
    qs = float(geom["tipQs"][0])
    nx, ny, nzg = ngrid
    dinv = dinv_of(ngrid, origin, step)
    q = PPs[..., :3].reshape(-1, 3).astype(np.float64)
    n_state = q.shape[0]
    # texel coordinates of the REPEAT/LINEAR sampler and the cell corners of every state
    Tn = np.array([nx, ny, nzg], np.float64)
    u = np.stack([q[:, d] * float(dinv[d][d]) + float(dinv[d][3]) for d in range(3)], 1)
    t = (u - np.floor(u)) * Tn - 0.5
    i0 = np.floor(t).astype(np.int64)
    corner_idx = []
    for k in range(2):
        for j in range(2):
            for i in range(2):
                cx, cy, cz = (i0[:, 0] + i) % nx, (i0[:, 1] + j) % ny, (i0[:, 2] + k) % nzg
                corner_idx.append((cz * ny + cy) * nx + cx)
    corner_idx = np.stack(corner_idx, 1)                      # (n_state, 8): corner x_i y_j z_k at 4k+2j+i
    uniq, inv = np.unique(corner_idx, return_inverse=True)
    inv = inv.reshape(n_state, 8)
    iz_, iy_, ix_ = uniq // (nx * ny), (uniq // nx) % ny, uniq % nx
    nodes = torch.tensor(np.stack([origin[0] + ix_ * step, origin[1] + iy_ * step, origin[2] + iz_ * step], 1),
                         dtype=dt)
    A = torch.tensor(np.asarray(atoms, np.float64), dtype=dt)
    P = torch.tensor(np.asarray(params, np.float64), dtype=dt)
    with torch.no_grad():
        gvals = torch.cat([_pair_values(kind, nodes[c:c + chunk], A, P, qs) for c in range(0, len(uniq), chunk)])
    # states as torch functions of q (grid values fixed): FE = trilinear sample, G = F + spring
    qt = torch.tensor(q, dtype=dt, requires_grad=True)
    s_list = [qt[:, d] * float(dinv[d][d]) + float(dinv[d][3]) for d in range(3)]
    tt = torch.stack([(s - torch.floor(s.detach())) * float(Tn[d]) - 0.5 for d, s in enumerate(s_list)], 1)
    a = tt - torch.floor(tt.detach())                          # the lerp weights, differentiable in q
    invt = torch.tensor(inv)
    corners = gvals[invt]                                      # (n_state, 8, 4)
    wts = []
    for k in range(2):
        for j in range(2):
            for i in range(2):
                wx = a[:, 0] if i else 1 - a[:, 0]
                wy = a[:, 1] if j else 1 - a[:, 1]
                wz = a[:, 2] if k else 1 - a[:, 2]
                wts.append(wx * wy * wz)
    W = torch.stack(wts, 1)                                    # (n_state, 8)
    FE = (W[..., None] * corners).sum(1)                       # (n_state, 4)
    kk = torch.tensor(np.asarray(stiff, np.float64), dtype=dt)
    iz = torch.arange(nz, dtype=dt).repeat(pts.shape[0])
    tip = torch.tensor(np.repeat(pts[:, :3].astype(np.float64), nz, 0), dtype=dt)
    tip = tip.clone()
    tip[:, 2] = tip[:, 2] + iz * dtip
    G = FE[:, :3] + (qt - tip) * kk[:3]
    # dL/dFE from the df loss at the equilibria
    FEv = FE.detach().clone().requires_grad_(True)
    Fz = FEv[:, 2].reshape(-1, nz)
    df = torch.zeros_like(Fz)
    df[:, 1:-1] = -(Fz[:, 2:] - Fz[:, :-2]) / (2 * abs(dtip))
    w = torch.ones_like(Fz)
    w[:, 0] = 0
    w[:, -1] = 0
    L = 0.5 * (w * (df - torch.tensor(target, dtype=dt)) ** 2).sum() / w.sum()
    uFE, = torch.autograd.grad(L, FEv)
    # dL/dq at fixed theta, and J = dG/dq (states independent: one backward pass per row)
    dLdq, = torch.autograd.grad(FE, qt, uFE, retain_graph=True)
    J = torch.zeros((n_state, 3, 3), dtype=dt)
    for r in range(3):
        e = torch.zeros_like(G)
        e[:, r] = 1.0
        J[:, r, :], = torch.autograd.grad(G, qt, e, retain_graph=True)
    lam = torch.linalg.solve(J.transpose(1, 2), dLdq.unsqueeze(-1)).squeeze(-1)     # J^T lambda = dL/dq
    # dL/dg at each node: W (u_FE - (lambda, 0)); dL/dk = -lambda . dG/dk
    ubar = uFE.clone()
    ubar[:, :3] -= lam
    gbar = torch.zeros_like(gvals)
    gbar.index_add_(0, invt.reshape(-1), (W[..., None] * ubar[:, None, :]).reshape(-1, 4).detach())
    dk = torch.zeros(4, dtype=dt)
    dk[:3] = -(lam * (qt.detach() - tip)).sum(0)
    # through the grid build, chunk by chunk
    A.requires_grad_(True)
    P.requires_grad_(True)
    gA = torch.zeros_like(A)
    gP = torch.zeros_like(P)
    for c in range(0, len(uniq), chunk):
        vals = _pair_values(kind, nodes[c:c + chunk], A, P, qs)
        da, dp = torch.autograd.grad(vals, (A, P), gbar[c:c + chunk])
        gA += da
        gP += dp
    return gA.numpy(), gP.numpy(), dk.numpy(), float(L.detach())
