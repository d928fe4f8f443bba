"""Differentiable AFM images: torch.autograd.Function over the CUDA kernels.

Two differentiable paths:

* ``GridAFM``: force-grid build + relaxation on the grid (the plain path).
  Forward: spm_grid_build -> spm_relax_ex(SPM_RELAX_PP).  Backward: the
  implicit-function adjoint at each converged state (spm_adjoint_grid_state)
  and the atomics-free gather through the grid build
  (spm_adjoint_grid_params).  Gradients: atom positions and charges, LJ
  (c6, c12) or Morse (R0, E0) parameters, the four spring constants.
* ``DirectMorseAFM``: the reference's grid-free Morse path
  (relaxStrokesTiltedMorseDirect + morseDirect* adjoint, kernels/AFM.cl:1419-2029).

No FIRE trajectory is stored: the adjoint only needs the equilibria.  Both
Functions return the tip-frame sample FE volume (n_scan, nz, 4); any torch loss
on it (e.g. ``df_loss``) back-propagates through them.
"""
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib, gpu


@dataclass
class GridScanSpec:
    """Geometry of one differentiable grid scan."""
    kind: int                 # 0 LJ, 1 Morse
    ngrid: tuple              # (nx, ny, nz) nodes
    origin: np.ndarray        # (3,) grid origin [A]
    step: float               # node spacing [A]
    points: np.ndarray        # (n_scan, 4) tip start positions (ix-major raster)
    nz: int                   # z-steps
    dtip: float               # z step (< 0: approach)
    tipQs: np.ndarray = field(default_factory=lambda: np.array([-0.05, 0, 0, 0], np.float32))
    tipQZs: np.ndarray = field(default_factory=lambda: np.zeros(4, np.float32))
    dpos0: np.ndarray = field(default_factory=lambda: np.zeros(4, np.float32))
    relax_params: np.ndarray = field(default_factory=lambda: np.array([0.5, 0.1, 0.02, 0.5], np.float32))
    max_iter: int = 1000
    f2conv: float = 1e-10
    raster_ny: int = 0
    strict: bool = True       # raise if any state fails the adjoint gates (else those states are masked)
    polish: bool = False      # Newton-polish every equilibrium (SPM_FLAG_POLISH): the forward and the
                              # adjoint then sit at the equilibrium of the interpolated field, not at
                              # FIRE's stopping point

    def vectors(self):
        o, s = self.origin, float(self.step)
        return (np.array([o[0], o[1], o[2], 0], np.float32), np.array([s, 0, 0, 0], np.float32),
                np.array([0, s, 0, 0], np.float32), np.array([0, 0, s, 0], np.float32))

    def dinv(self):
        L = np.array(self.ngrid, dtype=np.float64) * self.step
        n = self.ngrid
        o = np.asarray(self.origin, np.float32)
        return (np.array([1. / L[0], 0., 0., -o[0] / L[0] + 0.5 / n[0]], np.float32),
                np.array([0., 1. / L[1], 0., -o[1] / L[1] + 0.5 / n[1]], np.float32),
                np.array([0., 0., 1. / L[2], -o[2] / L[2] + 0.5 / n[2]], np.float32))

    def scan_params(self, stiffness):
        return _lib.make_scan_params(dinv=self.dinv(), tipC=[0, 0, 1, self.dtip],
                                     stiffness=np.asarray(stiffness, np.float32), dpos0=self.dpos0,
                                     relax_params=self.relax_params, nz=self.nz, max_iter=self.max_iter,
                                     f2conv=self.f2conv, fire=True, raster_ny=self.raster_ny, polish=self.polish)


class AdjointFailure(RuntimeError):
    pass


def _check_diag(diag, what):
    st = diag[:, 3]
    bad = st != 0
    if bool(bad.any()):
        i = int(torch.nonzero(bad)[0])
        d = diag[i].tolist()
        raise AdjointFailure(f"{what}: adjoint failed at state {i}: status={int(d[3])} residual={d[0]:.3e} "
                             f"lambda_min={d[1]:.3e} cond={d[2]:.3e} ({int(bad.sum())} states)")


class GridAFM(torch.autograd.Function):
    """FEs = GridAFM.apply(atoms (na,4)[x,y,z,Q], params (na,2|4), stiffness (4,), spec)."""

    @staticmethod
    def forward(ctx, atoms, params, stiffness, spec):
        dev = atoms.device
        atoms_c = atoms.detach().to(torch.float32).contiguous()
        params_c = params.detach().to(torch.float32).contiguous()
        k = stiffness.detach().to(torch.float32).cpu().numpy()
        p0, dA, dB, dC = spec.vectors()
        grid = gpu.grid_build(spec.kind, atoms_c, params_c, spec.ngrid, p0, dA, dB, dC, spec.tipQs, spec.tipQZs)
        P = spec.scan_params(k)
        pts = torch.as_tensor(spec.points, dtype=torch.float32, device=dev)
        FEs, PPs = gpu.relax_pp(grid, P, pts)
        ctx.spec = spec
        ctx.k = k
        ctx.save_for_backward(atoms_c, params_c, grid, PPs, pts)
        ctx.n_fail = int((PPs[..., 3] <= 0).sum().item())
        if spec.strict and ctx.n_fail:
            raise AdjointFailure(f"GridAFM: {ctx.n_fail} states did not converge (max_iter={spec.max_iter})")
        ctx.dtypes = (atoms.dtype, params.dtype, stiffness.dtype, stiffness.device)
        return FEs

    @staticmethod
    def backward(ctx, gFEs):
        atoms_c, params_c, grid, PPs, pts = ctx.saved_tensors
        spec = ctx.spec
        P = spec.scan_params(ctx.k)
        ubar, dk, diag = gpu.adjoint_grid_state(grid, P, pts, PPs, gFEs.contiguous())
        if spec.strict:
            _check_diag(diag, "GridAFM.backward")
        p0, dA, dB, dC = spec.vectors()
        grad, dk_sum = gpu.adjoint_grid_params(spec.kind, atoms_c, params_c, p0, dA, dB, dC, spec.tipQs,
                                               spec.tipQZs, grid, P, PPs, ubar, dk)
        g_atoms = torch.zeros_like(atoms_c, dtype=torch.float64)
        g_atoms[:, :3] = grad[:, :3]
        g_atoms[:, 3] = grad[:, 5]
        g_params = torch.zeros_like(params_c, dtype=torch.float64)
        g_params[:, 0] = grad[:, 3]
        g_params[:, 1] = grad[:, 4]
        da, dp, dkt, kdev = ctx.dtypes
        return g_atoms.to(da), g_params.to(dp), dk_sum.to(device=kdev, dtype=dkt), None


def grid_afm(atoms, params, stiffness, spec):
    """Tip-frame FE volume (n_scan, nz, 4), differentiable in atoms, params and stiffness."""
    return GridAFM.apply(atoms, params, stiffness, spec)


def df_loss(FEs, target_df, dtip, weights=None):
    """Central-difference df loss of df_loss_seed (spammm/SPM/AFM.py:3125-3200) in torch ops:
    df = -(Fz[iz+1] - Fz[iz-1]) / (2|dtip|) inside, L = 0.5 sum(w (df - t)^2) / sum(w)."""
    Fz = FEs[..., 2].to(torch.float64)
    dz = abs(float(dtip))
    df = torch.zeros_like(Fz)
    df[..., 1:-1] = -(Fz[..., 2:] - Fz[..., :-2]) / (2.0 * dz)
    if weights is None:
        w = torch.ones_like(Fz)
        w[..., 0] = 0.0
        w[..., -1] = 0.0
    else:
        w = weights.to(torch.float64)
    diff = df - target_df.to(torch.float64)
    return 0.5 * (w * diff * diff).sum() / w.sum()


class DirectMorseAFM(torch.autograd.Function):
    """FEs, PPs = DirectMorseAFM.apply(atoms (na,4), cMs (na,4), spec) on the grid-free Morse path."""

    @staticmethod
    def forward(ctx, atoms, cMs, spec):
        atoms_c = atoms.detach().to(torch.float32).contiguous()
        cMs_c = cMs.detach().to(torch.float32).contiguous()
        P = spec.scan_params(spec.stiffness)
        pts = torch.as_tensor(spec.points, dtype=torch.float32, device=atoms.device)
        FEs, PPs = gpu.relax_direct_morse(atoms_c, cMs_c, pts, P, spec.tipQs, spec.tipQZs)
        ctx.spec = spec
        ctx.save_for_backward(atoms_c, cMs_c, pts, PPs)
        return FEs

    @staticmethod
    def backward(ctx, gFEs):
        atoms_c, cMs_c, pts, PPs = ctx.saved_tensors
        spec = ctx.spec
        P = spec.scan_params(spec.stiffness)
        lam, diag = gpu.adjoint_direct_state(atoms_c, cMs_c, pts, P, spec.tipQs, spec.tipQZs, PPs,
                                             gFEs.contiguous())
        if spec.strict:
            _check_diag(diag, "DirectMorseAFM.backward")
        g = gpu.adjoint_direct_params(atoms_c, cMs_c, pts, P, spec.tipQs, spec.tipQZs, PPs, gFEs.contiguous(), lam)
        g_atoms = torch.zeros_like(atoms_c)
        g_atoms[:, :3] = g[:, :3]
        g_atoms[:, 3] = g[:, 5]
        g_cMs = torch.zeros_like(cMs_c)
        g_cMs[:, 0] = g[:, 3]
        g_cMs[:, 1] = g[:, 4]
        return g_atoms, g_cMs, None


@dataclass
class DirectScanSpec:
    """Geometry of one differentiable direct (grid-free) Morse scan."""
    points: np.ndarray
    nz: int
    dtip: float
    stiffness: np.ndarray = field(default_factory=lambda: np.array([-0.03, -0.03, -0.03, -1.0], np.float32))
    dpos0: np.ndarray = field(default_factory=lambda: np.array([0., 0., -4.0, 4.0], np.float32))
    tipQs: np.ndarray = field(default_factory=lambda: np.array([0., -0.1, 0.1, 0.], np.float32))
    tipQZs: np.ndarray = field(default_factory=lambda: np.array([0., 1.8, 3.6, 0.], np.float32))
    relax_params: np.ndarray = field(default_factory=lambda: np.array([0.5, 0.1, 0.02, 0.5], np.float32))
    max_iter: int = 128
    f2conv: float = 1e-8
    raster_ny: int = 0
    strict: bool = True

    def scan_params(self, stiffness):
        return _lib.make_scan_params(tipC=[0, 0, 1, self.dtip], stiffness=np.asarray(stiffness, np.float32),
                                     dpos0=self.dpos0, relax_params=self.relax_params, nz=self.nz,
                                     max_iter=self.max_iter, f2conv=self.f2conv, fire=True,
                                     raster_ny=self.raster_ny)
