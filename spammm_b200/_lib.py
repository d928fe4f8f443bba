"""ctypes binding of libspmb200.so (the C ABI declared in include/spm_b200.h).

The library is the only compute path of this package: every public function
raises ``RuntimeError`` when it is missing or cannot run -- there is no CPU or
PyTorch fallback.  Device buffers are torch CUDA tensors; calls are issued on
``torch.cuda.current_stream()``.
"""
import ctypes
import os

import numpy as np
import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libspmb200.so")

SPM_OK = 0
SPM_ERR_ARG = 1
SPM_ERR_CUDA = 2
SPM_ERR_UNSUPPORTED = 3
SPM_ERR_TIMEOUT = 4

SPM_KIND_LJ = 0
SPM_KIND_MORSE = 1
SPM_F32 = 0
SPM_F64 = 1
SPM_FLAG_FIRE = 1
SPM_RELAX_STROKES = 0
SPM_RELAX_TILTED = 1
SPM_RELAX_PP = 2
SPM_RELAX_2D = 3
SPM_FLAG_FLIP_Z = 2
SPM_FLAG_PAIRED = 4
# Newton polish of every relaxed state (not in the reference): after FIRE stops, up to four Newton
# steps on the total force of the interpolated grid and the spring; outputs at the polished position
SPM_FLAG_POLISH = 8
# batched relaxation: start each z-step from the previous call's equilibrium (PPs read and written)
SPM_FLAG_WARM = 16
SPM_ADJ_PAIR_PARAMS = 1
SPM_ADJ_STATE_MAXIMA = 2

_f4 = ctypes.c_float * 4


class ScanParams(ctypes.Structure):
    """Mirror of ``spm_scan_params``."""
    _fields_ = [
        ("dinvA", _f4), ("dinvB", _f4), ("dinvC", _f4),
        ("tipA", _f4), ("tipB", _f4), ("tipC", _f4),
        ("dTip", _f4), ("stiffness", _f4), ("dpos0", _f4),
        ("relax_params", _f4), ("surfFF", _f4),
        ("nz", ctypes.c_int), ("max_iter", ctypes.c_int),
        ("f2conv", ctypes.c_float), ("flags", ctypes.c_int),
        ("raster_ny", ctypes.c_int),
    ]


def f4(v):
    """float[4] from any 3- or 4-vector (missing .w = 0)."""
    a = np.zeros(4, dtype=np.float32)
    v = np.asarray(v, dtype=np.float32).ravel()
    a[: min(4, v.size)] = v[:4]
    return _f4(*a.tolist())


def make_scan_params(*, dinv=None, tipA=None, tipB=None, tipC=None, dTip=None, stiffness=None,
                     dpos0=None, relax_params=None, surfFF=None, nz=1, max_iter=128, f2conv=1e-8,
                     fire=True, flip_z=False, raster_ny=0, paired=False, polish=False, warm=False):
    p = ScanParams()
    z4 = np.zeros(4, np.float32)
    if dinv is not None:
        p.dinvA, p.dinvB, p.dinvC = f4(dinv[0]), f4(dinv[1]), f4(dinv[2])
    p.tipA = f4(tipA if tipA is not None else [1, 0, 0, 0])
    p.tipB = f4(tipB if tipB is not None else [0, 1, 0, 0])
    p.tipC = f4(tipC if tipC is not None else [0, 0, 1, 0])
    p.dTip = f4(dTip if dTip is not None else z4)
    p.stiffness = f4(stiffness if stiffness is not None else z4)
    p.dpos0 = f4(dpos0 if dpos0 is not None else z4)
    p.relax_params = f4(relax_params if relax_params is not None else z4)
    p.surfFF = f4(surfFF if surfFF is not None else z4)
    p.nz = int(nz)
    p.max_iter = int(max_iter)
    p.f2conv = float(f2conv)
    p.flags = ((SPM_FLAG_FIRE if fire else 0) | (SPM_FLAG_FLIP_Z if flip_z else 0) | (SPM_FLAG_PAIRED if paired else 0)
               | (SPM_FLAG_POLISH if polish else 0) | (SPM_FLAG_WARM if warm else 0))
    p.raster_ny = int(raster_ny)
    return p


class BatchMol(ctypes.Structure):
    """Mirror of ``spm_batch_mol`` (one molecule of a batch)."""
    _fields_ = [
        ("grid_off", ctypes.c_longlong), ("state_off", ctypes.c_longlong),
        ("tile_off", ctypes.c_longlong), ("slot_off", ctypes.c_longlong),
        ("unit_off", ctypes.c_longlong), ("chunk_off", ctypes.c_longlong),
        ("row_off", ctypes.c_longlong),
        ("atom_off", ctypes.c_int), ("n_atoms", ctypes.c_int),
        ("pix_off", ctypes.c_int), ("n_scan", ctypes.c_int),
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("z_lo", ctypes.c_int), ("nz_slab", ctypes.c_int),
        ("nz_steps", ctypes.c_int), ("raster_ny", ctypes.c_int),
        ("x_lo", ctypes.c_int), ("nx_slab", ctypes.c_int), ("y_lo", ctypes.c_int), ("ny_slab", ctypes.c_int),
        ("reserved", ctypes.c_int),
        ("p0", _f4), ("dA", _f4), ("dB", _f4), ("dC", _f4),
        ("dinvA", _f4), ("dinvB", _f4), ("dinvC", _f4),
    ]


class BatchShape(ctypes.Structure):
    """Mirror of ``spm_batch_shape`` (launch shapes of the batched kernels)."""
    _fields_ = [
        ("gb_ty", ctypes.c_int), ("gb_zb", ctypes.c_int), ("rx_threads", ctypes.c_int),
        ("rx_tile_h", ctypes.c_int), ("rx_ctas_per_sm", ctypes.c_int), ("adj_chunk", ctypes.c_int),
        ("rx_regs", ctypes.c_int), ("grid_layout", ctypes.c_int), ("rx_sync", ctypes.c_int),
        ("adj_ilp", ctypes.c_int), ("adj_agg", ctypes.c_int), ("adj_stage", ctypes.c_int),
    ]

    def key(self):
        return tuple(getattr(self, f) for f, _ in self._fields_)

    def __repr__(self):
        return "BatchShape(" + ", ".join(f"{f}={getattr(self, f)}" for f, _ in self._fields_) + ")"


_lib = None
_load_error = None

_vp = ctypes.c_void_p
_i = ctypes.c_int
_d = ctypes.c_double
_ll = ctypes.c_longlong
_P = ctypes.POINTER(ScanParams)
_BS = ctypes.POINTER(BatchShape)
_LLP = ctypes.POINTER(ctypes.c_longlong)
SPM_BATCH_TOTALS = 9

_SIGNATURES = {
    "spm_abi_version": (_i, []),
    "spm_last_error": (ctypes.c_char_p, []),
    "spm_grid_build": (_i, [_i, _i, _vp, _vp, _vp, _i, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "spm_pair_fe_points": (_i, [_i, _i, _vp, _vp, _vp, _i, _vp, _vp, _vp, _vp]),
    "spm_relax_strokes": (_i, [_vp, _i, _i, _i, _vp, _i, _P, _vp, _vp, _vp]),
    "spm_relax_ex": (_i, [_i, _vp, _i, _i, _i, _vp, _i, _P, _vp, _vp, _vp, _vp, _vp]),
    "spm_relax_workspace_bytes": (_ll, []),
    "spm_relax_strokes_tilted": (_i, [_vp, _i, _i, _i, _vp, _i, _P, _vp, _vp]),
    "spm_fe_in_strokes_tilted": (_i, [_vp, _i, _i, _i, _vp, _i, _P, _vp, _vp]),
    "spm_df_amp_dir": (_i, [_vp, _i, _i, _i, _i, _vp, _vp, _d, _vp, _i, _vp, _vp]),
    "spm_df_dir": (_i, [_vp, _i, _i, _i, _i, _vp, _vp, _vp, _vp]),
    "spm_dissipation": (_i, [_vp, _vp, _i, _i, _i, _i, _vp, _vp, _vp, _vp, _i, _vp, _vp]),
    "spm_relax_pair_dissipation": (_i, [_vp, _i, _i, _i, _vp, _i, _P, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i, _vp,
                                        _vp, _vp]),
    "spm_relax_pair_workspace_bytes": (_ll, [_i]),
    "spm_convolve_z": (_i, [_vp, _i, _i, _i, _vp, _vp, _vp]),
    "spm_izo_z": (_i, [_vp, _i, _i, ctypes.c_float, _vp, _vp]),
    "spm_df_loss_seed": (_i, [_vp, _i, _vp, _vp, _i, _i, _i, _d, _vp, _vp, _vp, _vp, _vp]),
    "spm_df_loss_scratch_bytes": (_ll, [_i, _i, _i]),
    "spm_df_loss_seed_noalloc": (_i, [_vp, _i, _vp, _vp, _i, _i, _i, _d, _vp, _vp, _vp, _vp]),
    "spm_relax_direct_morse": (_i, [_i, _vp, _vp, _vp, _i, _P, _vp, _vp, _vp, _vp, _vp]),
    "spm_adjoint_direct_state": (_i, [_i, _vp, _vp, _vp, _i, _P, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "spm_adjoint_direct_params": (_i, [_i, _vp, _vp, _vp, _i, _P, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "spm_adjoint_direct_scratch_bytes": (_ll, [_i, _i]),
    "spm_fp32_peak_probe": (_i, [_i, ctypes.POINTER(ctypes.c_double), _vp]),
    "spm_adjoint_grid_state": (_i, [_vp, _i, _i, _i, _vp, _i, _P, _vp, _vp, _vp, _vp, _vp, _vp]),
    "spm_adjoint_grid_params": (_i, [_i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i, _i, _i, _P, _vp, _vp,
                                     _vp, _ll, _vp, _vp, _vp, _vp]),
    "spm_adjoint_grid_scratch_bytes": (_ll, [_i, _ll]),
    "spm_batch_default_shape": (BatchShape, []),
    "spm_batch_prepare": (_i, [ctypes.POINTER(BatchMol), _i, _BS, _LLP]),
    "spm_batch_grid_build": (_i, [_i, _i, _vp, _ll, _BS, _vp, _vp, _vp, _vp, _vp, _vp]),
    "spm_batch_relax": (_i, [_i, _vp, _ll, _BS, _vp, _vp, _P, _vp, _vp, _vp, _vp, _ll, _vp]),
    "spm_batch_relax_workspace_bytes": (_ll, [_ll, _BS]),
    "spm_batch_df_amp": (_i, [_i, _vp, _ll, _vp, _d, _d, _vp, _vp]),
    "spm_batch_df_loss_seed": (_i, [_i, _vp, _ll, _vp, _vp, _vp, _d, _vp, _vp, _vp, _vp, _vp]),
    "spm_batch_loss_scratch_bytes": (_ll, [_ll, _i]),
    "spm_batch_failure_mask": (_i, [_ll, _vp, _vp, _vp, _vp]),
    "spm_batch_adam_step": (_i, [_ll, _vp, _vp, _vp, _vp, _vp, _d, _d, _d, _d, _i, _vp]),
    "spm_batch_adjoint_state": (_i, [_i, _vp, _ll, _BS, _vp, _vp, _P, _vp, _vp, _vp, _vp, _vp, _LLP, _vp, _vp]),
    "spm_batch_adjoint_params": (_i, [_i, _i, _vp, _LLP, _BS, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i,
                                      _vp, _vp]),
    "spm_batch_adjoint_scratch_bytes": (_ll, [_LLP, _i]),
}


def lib():
    """The loaded library; raises RuntimeError (no fallback) when unavailable."""
    global _lib, _load_error
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"libspmb200.so not found at {LIB_PATH}: build it with "
                           "`python -m spammm_b200.build` (nvcc, sm_100a); there is no CPU fallback")
    try:
        L = ctypes.CDLL(LIB_PATH)
    except OSError as e:
        _load_error = str(e)
        raise RuntimeError(f"cannot load {LIB_PATH}: {e}") from e
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(L, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def exported_symbols():
    """Names of the C ABI functions this binding knows about."""
    return list(_SIGNATURES)


def check(rc, what):
    if rc != SPM_OK:
        msg = lib().spm_last_error().decode(errors="replace")
        if rc == SPM_ERR_ARG:
            raise ValueError(f"{what}: {msg}")
        raise RuntimeError(f"{what} failed (status {rc}): {msg}")


def require_cuda():
    if not torch.cuda.is_available():
        raise RuntimeError("spammm_b200 needs a CUDA device (sm_100a); there is no CPU fallback")
    lib()


def stream_ptr():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def ptr(t):
    """Device pointer of a contiguous CUDA tensor (None -> NULL)."""
    if t is None:
        return None
    if not t.is_cuda:
        raise ValueError("expected a CUDA tensor")
    if not t.is_contiguous():
        raise ValueError("expected a contiguous tensor")
    return ctypes.c_void_p(t.data_ptr())


def hostvec(v, n=4, dtype=np.float32):
    a = np.zeros(n, dtype=dtype)
    v = np.asarray(v, dtype=dtype).ravel()
    a[: min(n, v.size)] = v[:n]
    return a


def hptr(a):
    """Host pointer of a contiguous numpy array (kept alive by the caller)."""
    return a.ctypes.data_as(ctypes.c_void_p)
