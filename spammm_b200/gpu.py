"""Tensor-level calls into libspmb200.so.

Each function validates shapes/dtypes, allocates its outputs with torch on the
current CUDA device (unless ``out`` tensors are passed) and launches the
corresponding C ABI entry point on ``torch.cuda.current_stream()``.  Nothing
here computes on the host; a missing library raises.
"""
import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import check, hostvec, hptr, lib, ptr, stream_ptr

F32 = torch.float32
F64 = torch.float64


def to_host(t):
    """A tensor as a NumPy array.  Device tensors are copied through pinned host
    memory (torch's caching host allocator): a pageable device-to-host copy
    runs at a few GB/s on the B200 boxes, a pinned one at PCIe speed (50 GB/s).
    The array keeps its pinned buffer alive; freed buffers are reused."""
    if not t.is_cuda:
        return t.numpy()
    t = t.contiguous()
    h = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
    h.copy_(t, non_blocking=True)
    torch.cuda.current_stream().synchronize()
    return h.numpy()


def _dev():
    _lib.require_cuda()
    return torch.device("cuda", torch.cuda.current_device())


def _as_dev(x, dtype, shape_tail=None, name="array"):
    """Contiguous CUDA tensor of dtype (copies from numpy / host if needed)."""
    if isinstance(x, torch.Tensor):
        t = x
        if not t.is_cuda:
            t = t.to(_dev())
        if t.dtype != dtype:
            t = t.to(dtype)
    else:
        t = torch.as_tensor(np.ascontiguousarray(x), dtype=dtype, device=_dev())
    t = t.contiguous()
    if shape_tail is not None and tuple(t.shape[-len(shape_tail):]) != tuple(shape_tail):
        raise ValueError(f"{name}: expected trailing shape {shape_tail}, got {tuple(t.shape)}")
    return t


# ---------------------------------------------------------------- stage (a)
def grid_build(kind, atoms, params, n, p0, dA, dB, dC, Qs, QZs, out=None):
    """Force grid (nz,ny,nx,4) float32 of the LJ (kind 0) or Morse (kind 1) +
    point-charge Coulomb law.  atoms (na,4), params (na,2) LJ / (na,4) Morse."""
    nx, ny, nz = (int(v) for v in n)
    atoms = _as_dev(atoms, F32, (4,), "atoms")
    pcols = 2 if kind == _lib.SPM_KIND_LJ else 4
    params = _as_dev(params, F32, (pcols,), "params")
    na = atoms.shape[0]
    if params.shape[0] != na:
        raise ValueError(f"params has {params.shape[0]} rows for {na} atoms")
    if out is None:
        out = torch.empty((nz, ny, nx, 4), dtype=F32, device=atoms.device)
    elif tuple(out.shape) != (nz, ny, nx, 4) or out.dtype != F32 or not out.is_contiguous():
        raise ValueError(f"grid out must be contiguous float32 {(nz, ny, nx, 4)}")
    hv = [hostvec(v) for v in (p0, dA, dB, dC, Qs, QZs)]
    rc = lib().spm_grid_build(int(kind), na, ptr(atoms) if na else None, ptr(params) if na else None, ptr(out),
                              nx, ny, nz, *[hptr(h) for h in hv], stream_ptr())
    check(rc, "spm_grid_build")
    return out


# ---------------------------------------------------------------- stage (b)
def _grid_dims(grid):
    if grid.dim() != 4 or grid.shape[3] != 4 or grid.dtype != F32 or not grid.is_cuda:
        raise ValueError("grid must be a CUDA float32 tensor (nz,ny,nx,4)")
    nz, ny, nx = grid.shape[:3]
    return int(nx), int(ny), int(nz)


def _workspace(device):
    """A fresh relaxation workspace (the pixel counter); per call, so concurrent
    launches on different streams never share one."""
    n = int(lib().spm_relax_workspace_bytes())
    return torch.empty(((n + 3) // 4,), dtype=torch.int32, device=device)


def relax_strokes(grid, params, points, FEs=None, disps=None, iter_count=None, dynamic=True):
    """relaxStrokes over (n_scan,4) points -> FEs, disps (n_scan,nz,4).

    iter_count: optional int32 CUDA tensor (n_scan,) receiving per-pixel step
    totals; dynamic: lanes draw pixels from a device counter (same results)."""
    nx, ny, nz = _grid_dims(grid)
    points = _as_dev(points, F32, (4,), "points")
    n_scan = points.shape[0]
    shape = (n_scan, params.nz, 4)
    FEs = torch.empty(shape, dtype=F32, device=points.device) if FEs is None else FEs
    disps = torch.empty(shape, dtype=F32, device=points.device) if disps is None else disps
    if iter_count is not None and (iter_count.dtype != torch.int32 or iter_count.numel() < n_scan):
        raise ValueError("iter_count must be an int32 tensor with n_scan entries")
    ws = _workspace(points.device) if dynamic else None
    rc = lib().spm_relax_ex(_lib.SPM_RELAX_STROKES, ptr(grid), nx, ny, nz, ptr(points), n_scan, ctypes.byref(params),
                            ptr(FEs), ptr(disps), ptr(iter_count), ptr(ws), stream_ptr())
    check(rc, "spm_relax_strokes")
    return FEs, disps


def relax_strokes_tilted(grid, params, points, FEs=None, dynamic=True):
    nx, ny, nz = _grid_dims(grid)
    points = _as_dev(points, F32, (4,), "points")
    n_scan = points.shape[0]
    FEs = torch.empty((n_scan, params.nz, 4), dtype=F32, device=points.device) if FEs is None else FEs
    ws = _workspace(points.device) if dynamic else None
    rc = lib().spm_relax_ex(_lib.SPM_RELAX_TILTED, ptr(grid), nx, ny, nz, ptr(points), n_scan, ctypes.byref(params),
                            ptr(FEs), None, None, ptr(ws), stream_ptr())
    check(rc, "spm_relax_strokes_tilted")
    return FEs


def relax_pp(grid, params, points, FEs=None, PPs=None, iter_count=None, dynamic=True):
    """Grid relaxation with equilibrium bookkeeping (SPM_RELAX_PP) -> FEs, PPs (n_scan,nz,4).

    FEs: tip-frame sample FE at the stored position; PPs = (pos, +iters / -iters)."""
    nx, ny, nz = _grid_dims(grid)
    points = _as_dev(points, F32, (4,), "points")
    n_scan = points.shape[0]
    shape = (n_scan, params.nz, 4)
    FEs = torch.empty(shape, dtype=F32, device=points.device) if FEs is None else FEs
    PPs = torch.empty(shape, dtype=F32, device=points.device) if PPs is None else PPs
    ws = _workspace(points.device) if dynamic else None
    rc = lib().spm_relax_ex(_lib.SPM_RELAX_PP, ptr(grid), nx, ny, nz, ptr(points), n_scan, ctypes.byref(params),
                            ptr(FEs), ptr(PPs), ptr(iter_count), ptr(ws), stream_ptr())
    check(rc, "spm_relax_ex(PP)")
    return FEs, PPs


def relax_2d(grid, params, points, FEs=None, disps=None, iter_count=None, dynamic=True):
    """relaxStrokes2D (SPM_RELAX_2D) over (n_scan,4) anchors -> FEs, disps (n_scan,nz,4).
    params: stiffness[0] = K_lat, relax_params = (dt, damp), dTip[2] = -dh."""
    nx, ny, nz = _grid_dims(grid)
    points = _as_dev(points, F32, (4,), "points")
    n_scan = points.shape[0]
    shape = (n_scan, params.nz, 4)
    FEs = torch.empty(shape, dtype=F32, device=points.device) if FEs is None else FEs
    disps = torch.empty(shape, dtype=F32, device=points.device) if disps is None else disps
    ws = _workspace(points.device) if dynamic else None
    rc = lib().spm_relax_ex(_lib.SPM_RELAX_2D, ptr(grid), nx, ny, nz, ptr(points), n_scan, ctypes.byref(params),
                            ptr(FEs), ptr(disps), ptr(iter_count), ptr(ws), stream_ptr())
    check(rc, "spm_relax_ex(2D)")
    return FEs, disps


def adjoint_grid_state(grid, params, points, PPs, dL_dFEs):
    """Per-state implicit adjoint on the grid -> ubar, dk, diag (n_state,4)."""
    nx, ny, nz = _grid_dims(grid)
    points = _as_dev(points, F32, (4,), "points")
    PPs = _as_dev(PPs, F32, (4,), "PPs").reshape(-1, 4)
    dL = _as_dev(dL_dFEs, F32, (4,), "dL_dFEs").reshape(-1, 4)
    n_scan = points.shape[0]
    if PPs.shape[0] != n_scan * params.nz or dL.shape[0] != PPs.shape[0]:
        raise ValueError("PPs/dL_dFEs must hold n_scan*nz states")
    ubar, dk, diag = torch.empty_like(PPs), torch.empty_like(PPs), torch.empty_like(PPs)
    rc = lib().spm_adjoint_grid_state(ptr(grid), nx, ny, nz, ptr(points), n_scan, ctypes.byref(params), ptr(PPs),
                                      ptr(dL), ptr(ubar), ptr(dk), ptr(diag), stream_ptr())
    check(rc, "spm_adjoint_grid_state")
    return ubar, dk, diag


def adjoint_grid_params(kind, atoms, params_atoms, p0, dA, dB, dC, Qs, QZs, grid, scan_params, PPs, ubar, dk):
    """Atom and spring gradients of the grid path -> grad (na,6) f64 (x,y,z,P1,P2,Q), dk (4,) f64."""
    nx, ny, nz = _grid_dims(grid)
    atoms = _as_dev(atoms, F32, (4,), "atoms")
    pcols = 2 if kind == _lib.SPM_KIND_LJ else 4
    prm = _as_dev(params_atoms, F32, (pcols,), "params")
    PPs = _as_dev(PPs, F32, (4,), "PPs").reshape(-1, 4)
    ubar = _as_dev(ubar, F32, (4,), "ubar").reshape(-1, 4)
    dk = _as_dev(dk, F32, (4,), "dk").reshape(-1, 4)
    na, n_state = int(atoms.shape[0]), int(PPs.shape[0])
    grad = torch.empty((na, 6), dtype=F64, device=atoms.device)
    dk_sum = torch.empty((4,), dtype=F64, device=atoms.device)
    nbytes = int(lib().spm_adjoint_grid_scratch_bytes(na, n_state))
    scratch = torch.empty((max(nbytes, 8) + 7) // 8, dtype=F64, device=atoms.device)
    hv = [hostvec(v) for v in (p0, dA, dB, dC, Qs, QZs)]
    rc = lib().spm_adjoint_grid_params(int(kind), na, ptr(atoms) if na else None, ptr(prm) if na else None,
                                       *[hptr(h) for h in hv], ptr(grid), nx, ny, nz, ctypes.byref(scan_params),
                                       ptr(PPs), ptr(ubar), ptr(dk), n_state, ptr(grad), ptr(dk_sum), ptr(scratch),
                                       stream_ptr())
    check(rc, "spm_adjoint_grid_params")
    return grad, dk_sum


def fe_in_strokes_tilted(grid, params, points, FEs=None):
    nx, ny, nz = _grid_dims(grid)
    points = _as_dev(points, F32, (4,), "points")
    n_scan = points.shape[0]
    FEs = torch.empty((n_scan, params.nz, 4), dtype=F32, device=points.device) if FEs is None else FEs
    rc = lib().spm_fe_in_strokes_tilted(ptr(grid), nx, ny, nz, ptr(points), n_scan, ctypes.byref(params), ptr(FEs),
                                        stream_ptr())
    check(rc, "spm_fe_in_strokes_tilted")
    return FEs


# ---------------------------------------------------------------- stage (c)
def _dir_spacing(spacing, osc_dir):
    """Normalised direction and per-axis spacing (AFM.py:3091-3103 contract)."""
    n = np.asarray(osc_dir, dtype=np.float64)
    if n.shape != (3,) or not np.isfinite(n).all():
        raise ValueError(f"osc_dir must contain three finite components, got {osc_dir!r}")
    norm = float(np.linalg.norm(n))
    if norm <= 0.0:
        raise ValueError(f"osc_dir must be non-zero, got {osc_dir!r}")
    n = n / norm
    dr = (np.full(3, abs(float(spacing)), dtype=np.float64) if np.ndim(spacing) == 0
          else np.abs(np.asarray(spacing, dtype=np.float64)))
    if dr.shape != (3,) or not np.isfinite(dr).all() or np.any(dr <= 0.0):
        raise ValueError(f"spacing must be a positive scalar or (dx,dy,dz), got {spacing!r}")
    return np.ascontiguousarray(n), np.ascontiguousarray(dr)


def _fes_volume(FEs):
    """(nx,ny,nz,4) CUDA volume kept in float64 when given float64, else float32."""
    is64 = (FEs.dtype == torch.float64) if isinstance(FEs, torch.Tensor) else (np.asarray(FEs).dtype == np.float64)
    FEs = _as_dev(FEs, F64 if is64 else F32)
    if FEs.dim() != 4 or FEs.shape[-1] != 4:
        raise ValueError(f"FEs must have shape (nx,ny,nz,4), got {tuple(FEs.shape)}")
    return FEs


def _dt(t):
    return _lib.SPM_F64 if t.dtype == F64 else _lib.SPM_F32


def df_amp_dir(FEs, spacing, osc_dir=(0., 0., 1.), amp=1.0, out_iz=None):
    """compute_df_amp_dir on the device -> (nx,ny,n_out) float32."""
    FEs = _fes_volume(FEs)
    nx, ny, nz = (int(s) for s in FEs.shape[:3])
    n, dr = _dir_spacing(spacing, osc_dir)
    for ia in np.flatnonzero(np.abs(n) > 1e-15):
        if FEs.shape[ia] < 2:
            raise ValueError(f"FEs axis {ia} needs at least 2 samples for osc_dir={tuple(n)}")
    iz_t = None
    n_out = nz
    if out_iz is not None:
        iz_t = torch.as_tensor(np.asarray(out_iz, dtype=np.int32), device=FEs.device)
        n_out = int(iz_t.numel())
    df = torch.empty((nx, ny, n_out), dtype=F32, device=FEs.device)
    rc = lib().spm_df_amp_dir(ptr(FEs), _dt(FEs), nx, ny, nz, hptr(n), hptr(dr), float(amp), ptr(iz_t), n_out, ptr(df),
                              stream_ptr())
    check(rc, "spm_df_amp_dir")
    return df


def df_dir(FEs, spacing, osc_dir=(0., 0., 1.)):
    """compute_df_dir on the device -> (nx,ny,nz) float64."""
    FEs = _fes_volume(FEs)
    nx, ny, nz = (int(s) for s in FEs.shape[:3])
    n, dr = _dir_spacing(spacing, osc_dir)
    for ia in np.flatnonzero(np.abs(n) > 1e-15):
        if FEs.shape[ia] < 2:
            raise ValueError(f"FEs axis {ia} needs at least 2 samples for osc_dir={tuple(n)}")
    df = torch.empty((nx, ny, nz), dtype=F64, device=FEs.device)
    check(lib().spm_df_dir(ptr(FEs), _dt(FEs), nx, ny, nz, hptr(n), hptr(dr), ptr(df), stream_ptr()), "spm_df_dir")
    return df


def pair_fe_points(kind, atoms, params, queries, Qs, QZs):
    """Uncapped pair sums (F, E) at (n,3) query points -> (n,4) float32 CUDA tensor."""
    q = _as_dev(queries, F32, (3,), "queries")
    dev = q.device
    a = torch.as_tensor(np.ascontiguousarray(atoms, np.float32), device=dev).reshape(-1, 4).contiguous()
    pstride = 4 if kind == _lib.SPM_KIND_MORSE else 2
    prm = torch.as_tensor(np.ascontiguousarray(params, np.float32), device=dev).reshape(-1, pstride).contiguous()
    out = torch.empty((q.shape[0], 4), dtype=F32, device=dev)
    rc = lib().spm_pair_fe_points(int(kind), a.shape[0], ptr(a), ptr(prm), ptr(q), q.shape[0], hptr(hostvec(Qs)),
                                  hptr(hostvec(QZs)), ptr(out), stream_ptr())
    check(rc, "spm_pair_fe_points")
    return out


def _diss_lists(h_scan, h_df, amp, osc_dir, dev):
    """compute_dissipation's integration windows (AFM.py:3266-3273): for every output height, the scan
    heights within +-amp*|n_z| (all of them when fewer than two) -> (n, h, off, idx) for the kernels."""
    h_scan = np.asarray(h_scan, dtype=np.float64)
    nz = h_scan.shape[0]
    n = np.asarray(osc_dir, dtype=np.float64)
    n = np.ascontiguousarray(n / np.linalg.norm(n))
    amp_z = float(amp) * abs(n[2])
    off = [0]
    idx = []
    for h in np.asarray(h_df, dtype=np.float64):
        mask = (h_scan >= h - amp_z) & (h_scan <= h + amp_z)
        if mask.sum() < 2:
            mask = np.ones(nz, dtype=bool)
        idx.extend(np.flatnonzero(mask).tolist())
        off.append(len(idx))
    return (n, torch.as_tensor(h_scan, dtype=F64, device=dev), torch.as_tensor(np.asarray(off, np.int32), device=dev),
            torch.as_tensor(np.asarray(idx if idx else [0], np.int32), device=dev))


def relax_pair_dissipation(grid, params, points, h_scan, h_df, amp, osc_dir=(0., 0., 1.), iter_count=None):
    """Forward + backward strokes (SPM_FLAG_PAIRED in params) and their dissipation in one launch ->
    FEs, disps (n_scan,nz,4), E_diss (n_scan/2, len(h_df)) float32; h_scan in the stored z order."""
    nx, ny, nz = _grid_dims(grid)
    points = _as_dev(points, F32, (4,), "points")
    n_scan = points.shape[0]
    shape = (n_scan, params.nz, 4)
    dev = points.device
    FEs = torch.empty(shape, dtype=F32, device=dev)
    disps = torch.empty(shape, dtype=F32, device=dev)
    if len(np.asarray(h_scan)) != params.nz:
        raise ValueError(f"h_scan must have {params.nz} entries")
    n, h_t, off_t, idx_t = _diss_lists(h_scan, h_df, amp, osc_dir, dev)
    n_out = len(np.asarray(h_df))
    E = torch.empty((n_scan // 2, n_out), dtype=F32, device=dev)
    ws = torch.empty(((int(lib().spm_relax_pair_workspace_bytes(n_scan)) + 15) // 16, 4), dtype=torch.int32,
                     device=dev)
    rc = lib().spm_relax_pair_dissipation(ptr(grid), nx, ny, nz, ptr(points), n_scan, ctypes.byref(params), ptr(FEs),
                                          ptr(disps), ptr(iter_count), hptr(n), ptr(h_t), ptr(off_t), ptr(idx_t),
                                          n_out, ptr(E), ptr(ws), stream_ptr())
    check(rc, "spm_relax_pair_dissipation")
    return FEs, disps, E


def dissipation(FEs_fwd, FEs_bwd, h_scan, h_df, amp, osc_dir=(0., 0., 1.)):
    """compute_dissipation on the device -> (nx,ny,nz_df) float32."""
    Ff = _fes_volume(FEs_fwd)
    Fb = _fes_volume(FEs_bwd)
    if Ff.dtype != Fb.dtype:
        Ff, Fb = Ff.to(F64), Fb.to(F64)
    if Ff.shape != Fb.shape:
        raise ValueError(f"forward/backward volumes differ: {tuple(Ff.shape)} vs {tuple(Fb.shape)}")
    nx, ny, nz = (int(s) for s in Ff.shape[:3])
    h_scan = np.asarray(h_scan, dtype=np.float64)
    h_df = np.asarray(h_df, dtype=np.float64)
    if h_scan.shape != (nz,):
        raise ValueError(f"h_scan must have {nz} entries, got {h_scan.shape}")
    dev = Ff.device
    n, h_t, off_t, idx_t = _diss_lists(h_scan, h_df, amp, osc_dir, dev)
    E = torch.empty((nx, ny, len(h_df)), dtype=F32, device=dev)
    rc = lib().spm_dissipation(ptr(Ff), ptr(Fb), _dt(Ff), nx, ny, nz, hptr(n), ptr(h_t), ptr(off_t), ptr(idx_t), len(h_df),
                               ptr(E), stream_ptr())
    check(rc, "spm_dissipation")
    return E


def convolve_z(FEs, weights, nz_out):
    """convolveZ (kernels/AFM.cl:666-701) on every z-column of FEs (..., nz_in, 4)
    float32: out[..., izo, :] = sum_jz FEs[..., izo + jz, :] * weights[jz],
    len(weights) = nz_in - nz_out -> (..., nz_out, 4) float32."""
    FEs = _as_dev(FEs, F32, None, "FEs")
    if FEs.dim() < 2 or FEs.shape[-1] != 4:
        raise ValueError(f"FEs must be (..., nz, 4), got {tuple(FEs.shape)}")
    FEs = FEs.contiguous()
    nz_in = int(FEs.shape[-2])
    w = _as_dev(np.asarray(weights, np.float32).ravel() if not isinstance(weights, torch.Tensor) else weights, F32,
                None, "weights").reshape(-1).contiguous()
    if int(w.numel()) != nz_in - int(nz_out):
        raise ValueError(f"{w.numel()} weights for nz_in={nz_in}, nz_out={nz_out}: need nz_in - nz_out")
    n_col = int(FEs.numel() // (4 * nz_in)) if nz_in else 0
    out = torch.empty(tuple(FEs.shape[:-2]) + (int(nz_out), 4), dtype=F32, device=FEs.device)
    check(lib().spm_convolve_z(ptr(FEs), n_col, nz_in, int(nz_out), ptr(w), ptr(out), stream_ptr()), "spm_convolve_z")
    return out


def izo_z(FEs, iso):
    """izoZ (kernels/AFM.cl:705-723): per z-column of FEs (..., nz, 4) float32
    the first iz >= 1 with Fz > iso, as iz + the linear fraction from iz-1
    (-1 when Fz never exceeds iso) -> (...) float32."""
    FEs = _as_dev(FEs, F32, None, "FEs")
    if FEs.dim() < 2 or FEs.shape[-1] != 4:
        raise ValueError(f"FEs must be (..., nz, 4), got {tuple(FEs.shape)}")
    FEs = FEs.contiguous()
    nz = int(FEs.shape[-2])
    out = torch.empty(tuple(FEs.shape[:-2]), dtype=F32, device=FEs.device)
    n_col = int(out.numel())
    check(lib().spm_izo_z(ptr(FEs), n_col, nz, float(iso), ptr(out), stream_ptr()), "spm_izo_z")
    return out


def df_loss_seed(FEs, target_df, dtip, weights=None):
    """df_loss_seed on the device -> (loss (1,) f64, df (nx,ny,nz) f64, dL_dFEs (nx,ny,nz,4) f32)."""
    FEs = _fes_volume(FEs)
    nx, ny, nz = (int(s) for s in FEs.shape[:3])
    dtip = float(dtip)
    if dtip >= 0.0:
        raise ValueError(f"df_loss_seed: dtip must be <0, got dtip={dtip}")
    if nz < 3:
        raise ValueError(f"df_loss_seed: need nz>=3 for central difference, got nz={nz}")
    tgt = _as_dev(target_df, F64)
    if tuple(tgt.shape) != (nx, ny, nz):
        raise ValueError(f"df_loss_seed: target_df must be ({nx},{ny},{nz}), got {tuple(tgt.shape)}")
    w = None
    if weights is not None:
        w = _as_dev(weights, F64)
        if tuple(w.shape) != (nx, ny, nz):
            raise ValueError(f"df_loss_seed: weights must be ({nx},{ny},{nz}), got {tuple(w.shape)}")
    dev = FEs.device
    df = torch.empty((nx, ny, nz), dtype=F64, device=dev)
    dL = torch.empty((nx, ny, nz, 4), dtype=F32, device=dev)
    loss = torch.empty((1,), dtype=F64, device=dev)
    nbytes = int(lib().spm_df_loss_scratch_bytes(nx, ny, nz))
    scratch = torch.empty((max(nbytes, 8) + 7) // 8, dtype=F64, device=dev)
    rc = lib().spm_df_loss_seed(ptr(FEs), _dt(FEs), ptr(tgt), ptr(w), nx, ny, nz, dtip, ptr(df), ptr(dL), ptr(loss),
                                ptr(scratch), stream_ptr())
    check(rc, "spm_df_loss_seed")
    return loss, df, dL


def fp32_peak_flops(iters=1 << 16):
    out = ctypes.c_double(0.0)
    check(lib().spm_fp32_peak_probe(int(iters), ctypes.byref(out), stream_ptr()), "spm_fp32_peak_probe")
    return out.value


# ---------------------------------------------------------------- direct Morse path
def relax_direct_morse(atoms, cMs, points, params, Qs, QZs):
    """relaxStrokesTiltedMorseDirect -> FEs, PPs (n_scan,nz,4)."""
    atoms = _as_dev(atoms, F32, (4,), "atoms")
    cMs = _as_dev(cMs, F32, (4,), "cMs")
    points = _as_dev(points, F32, (4,), "points")
    n_scan = points.shape[0]
    shape = (n_scan, params.nz, 4)
    FEs = torch.empty(shape, dtype=F32, device=points.device)
    PPs = torch.empty(shape, dtype=F32, device=points.device)
    q, qz = hostvec(Qs), hostvec(QZs)
    rc = lib().spm_relax_direct_morse(int(atoms.shape[0]), ptr(atoms), ptr(cMs), ptr(points), n_scan,
                                      ctypes.byref(params), hptr(q), hptr(qz), ptr(FEs), ptr(PPs), stream_ptr())
    check(rc, "spm_relax_direct_morse")
    return FEs, PPs


def adjoint_direct_state(atoms, cMs, points, params, Qs, QZs, PPs, dL_dFEs):
    """morseDirectStateAdjoint -> lambdas, diag (n_state,4)."""
    atoms = _as_dev(atoms, F32, (4,), "atoms")
    cMs = _as_dev(cMs, F32, (4,), "cMs")
    points = _as_dev(points, F32, (4,), "points")
    PPs = _as_dev(PPs, F32, (4,), "PPs").reshape(-1, 4)
    dL = _as_dev(dL_dFEs, F32, (4,), "dL_dFEs").reshape(-1, 4)
    n_scan = points.shape[0]
    if PPs.shape[0] != n_scan * params.nz or dL.shape[0] != PPs.shape[0]:
        raise ValueError("PPs/dL_dFEs must hold n_scan*nz states")
    lam = torch.empty_like(PPs)
    diag = torch.empty_like(PPs)
    q, qz = hostvec(Qs), hostvec(QZs)
    rc = lib().spm_adjoint_direct_state(int(atoms.shape[0]), ptr(atoms), ptr(cMs), ptr(points), n_scan,
                                        ctypes.byref(params), hptr(q), hptr(qz), ptr(PPs), ptr(dL), ptr(lam),
                                        ptr(diag), stream_ptr())
    check(rc, "spm_adjoint_direct_state")
    return lam, diag


def adjoint_direct_params(atoms, cMs, points, params, Qs, QZs, PPs, dL_dFEs, lambdas, scratch=None):
    """morseDirectParamPartials + reduce -> grad (n_atoms,6) float32 (x,y,z,R0,E0,Q)."""
    atoms = _as_dev(atoms, F32, (4,), "atoms")
    cMs = _as_dev(cMs, F32, (4,), "cMs")
    points = _as_dev(points, F32, (4,), "points")
    PPs = _as_dev(PPs, F32, (4,), "PPs").reshape(-1, 4)
    dL = _as_dev(dL_dFEs, F32, (4,), "dL_dFEs").reshape(-1, 4)
    lam = _as_dev(lambdas, F32, (4,), "lambdas").reshape(-1, 4)
    na, n_scan = int(atoms.shape[0]), int(points.shape[0])
    grad = torch.empty((na, 6), dtype=F32, device=atoms.device)
    nbytes = int(lib().spm_adjoint_direct_scratch_bytes(na, n_scan))
    if scratch is None:
        scratch = torch.empty((max(nbytes, 4) + 3) // 4, dtype=F32, device=atoms.device)
    elif scratch.numel() * scratch.element_size() < nbytes:
        raise ValueError(f"scratch holds {scratch.numel() * scratch.element_size()} bytes, needs {nbytes}")
    q, qz = hostvec(Qs), hostvec(QZs)
    rc = lib().spm_adjoint_direct_params(na, ptr(atoms), ptr(cMs), ptr(points), n_scan, ctypes.byref(params),
                                         hptr(q), hptr(qz), ptr(PPs), ptr(dL), ptr(lam), ptr(grad), ptr(scratch),
                                         stream_ptr())
    check(rc, "spm_adjoint_direct_params")
    return grad
