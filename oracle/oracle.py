"""TEST INFRASTRUCTURE ONLY -- the oracle for the probe-particle AFM hot path.

Loaded by tests/, bench.py's CPU-baseline leg and __graft_entry__.smoke() as
the checker; the product (spammm_b200) never imports it.

Two parts:
  * ctypes access to libspm_oracle.so, the C restatement of SPAMMM's OpenCL
    kernels (kernels/AFM.cl; see ora_core.h for per-function citations), in
    canonical FP32 (bit-identical to the CUDA relaxation paths) and FP64;
  * NumPy restatements of the reference's host-side stage (c) and loss code:
      compute_df            spammm/SPM/AFM.py:3048-3050
      compute_df_amp        spammm/SPM/AFM.py:3052-3089
      compute_df_dir        spammm/SPM/AFM.py:3105-3123
      compute_df_amp_dir    spammm/SPM/AFM.py:3203-3236
      df_loss_seed          spammm/SPM/AFM.py:3125-3200
      compute_dissipation   spammm/SPM/AFM.py:3238-3277
    The linear interpolation of scipy.ndimage.map_coordinates(order=1,
    mode='nearest') is restated here (weights (1-t, t) at floor(c), indices
    clamped to the array), so the oracle does not depend on SciPy; it is
    pinned against fixtures produced by the reference itself
    (tests/golden/gen_golden.py).
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libspm_oracle.so")
COULOMB_CONST = 14.3996448915

_lib = None
_vp = ctypes.c_void_p
_i = ctypes.c_int
_f = ctypes.c_float
_d = ctypes.c_double
_ll = ctypes.c_longlong


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        build()
    try:
        L = ctypes.CDLL(LIB_PATH)
    except OSError:
        build()
        L = ctypes.CDLL(LIB_PATH)
    sig = {
        "ora_num_threads": (_i, []),
        "ora_set_num_threads": (None, [_i]),
        "ora_grid_build_d": (None, [_i, _i, _vp, _vp, _i, _i, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _ll, _ll, _vp]),
        "ora_grid_build_f": (None, [_i, _i, _vp, _vp, _i, _i, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _ll, _ll, _vp]),
        "ora_grid_build_d64": (None, [_i, _i, _vp, _vp, _i, _i, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _ll, _ll,
                                      _vp]),
        "ora_pair_fe_d": (None, [_i, _i, _vp, _vp, _i, _vp, _i, _vp, _vp, _vp]),
        "ora_pair_fe_abs_d": (None, [_i, _i, _vp, _vp, _i, _vp, _i, _vp, _vp, _vp]),
        "ora_relax_strokes_f": (None, [_vp, _i, _i, _i, _vp, _vp, _vp, _vp, _i, _i, _vp, _vp, _vp, _vp, _i, _f, _i,
                                       _i, _i, _vp, _vp]),
        "ora_relax_strokes_d": (None, [_vp, _i, _i, _i, _vp, _vp, _vp, _vp, _i, _i, _vp, _vp, _vp, _vp, _i, _d, _i,
                                       _i, _i, _vp, _vp]),
        "ora_relax_tilted_f": (None, [_vp, _i, _i, _i, _vp, _vp, _vp, _vp, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                      _i, _f, _i, _i, _vp]),
        "ora_relax_2d_f": (None, [_vp, _i, _i, _i, _vp, _vp, _vp, _vp, _i, _i, _f, _f, _f, _f, _i, _f, _i, _vp,
                                  _vp]),
        "ora_relax_tilted_d": (None, [_vp, _i, _i, _i, _vp, _vp, _vp, _vp, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                      _i, _d, _i, _i, _vp]),
        "ora_raw_tilted_f": (None, [_vp, _i, _i, _i, _vp, _vp, _vp, _vp, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp]),
        "ora_raw_tilted_d": (None, [_vp, _i, _i, _i, _vp, _vp, _vp, _vp, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp]),
        "ora_relax_direct_d": (None, [_i, _vp, _vp, _vp, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _i,
                                      _d, _i, _vp, _vp]),
        "ora_relax_pp_f": (None, [_vp, _i, _i, _i, _vp, _vp, _vp, _vp, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                  _i, _f, _i, _i, _vp, _vp]),
        "ora_relax_pp_d": (None, [_vp, _i, _i, _i, _vp, _vp, _vp, _vp, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                  _i, _d, _i, _i, _vp, _vp]),
        "ora_convolve_z_f": (None, [_vp, _i, _i, _i, _vp, _vp]),
        "ora_izo_z_f": (None, [_vp, _i, _i, _f, _vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _v4(v, dtype=np.float32):
    a = np.zeros(4, dtype=dtype)
    v = np.asarray(v, dtype=dtype).ravel()
    a[: min(4, v.size)] = v[:4]
    return a


def num_threads():
    return lib().ora_num_threads()


def set_num_threads(n):
    lib().ora_set_num_threads(int(n))


# ---------------------------------------------------------------- stage (a)
def grid_build(kind, atoms, params, n, p0, dA, dB, dC, Qs, QZs, prec="f64", node0=0, nnodes=None):
    """Force grid (nz,ny,nx,4) (or a flattened node slice when nnodes is given).

    prec: 'f32' (FP32 arithmetic), 'f64' (FP64 arithmetic on float32 inputs, as
    the reference kernel receives them) or 'f64in' (FP64 arithmetic and inputs)."""
    atoms_in, params_in = atoms, params
    nx, ny, nz = (int(v) for v in n)
    atoms = np.ascontiguousarray(atoms, dtype=np.float32).reshape(-1, 4)
    pstride = 2 if kind == 0 else 4
    params = np.ascontiguousarray(params, dtype=np.float32).reshape(-1, pstride)
    total = nx * ny * nz
    full = nnodes is None
    if full:
        node0, nnodes = 0, total
    dt = np.float64 if prec in ("f64", "f64in") else np.float32
    out = np.zeros((nnodes, 4), dtype=dt)
    if prec == "f64in":  # FP64 inputs as given (no float32 rounding of atoms / parameters)
        atoms = np.ascontiguousarray(atoms_in, dtype=np.float64).reshape(-1, 4)
        params = np.ascontiguousarray(params_in, dtype=np.float64).reshape(-1, pstride)
        vs = [_v4(v, np.float64) for v in (p0, dA, dB, dC, Qs, QZs)]
        fn = lib().ora_grid_build_d64
    else:
        vs = [_v4(v) for v in (p0, dA, dB, dC, Qs, QZs)]
        fn = lib().ora_grid_build_d if prec == "f64" else lib().ora_grid_build_f
    fn(int(kind), atoms.shape[0], _p(atoms), _p(params), pstride, nx, ny, nz, *[_p(v) for v in vs], int(node0),
       int(nnodes), _p(out))
    return out.reshape(nz, ny, nx, 4) if full else out


def pair_fe(kind, atoms, params, queries, Qs, QZs):
    """Uncapped direct pair FE at (n,3) query points, FP64 -> (n,4)."""
    atoms = np.ascontiguousarray(atoms, dtype=np.float64).reshape(-1, 4)
    pstride = 2 if kind == 0 else 4
    params = np.ascontiguousarray(params, dtype=np.float64).reshape(-1, pstride)
    q = np.ascontiguousarray(queries, dtype=np.float64).reshape(-1, 3)
    out = np.zeros((q.shape[0], 4), dtype=np.float64)
    qs, qz = _v4(Qs, np.float64), _v4(QZs, np.float64)
    lib().ora_pair_fe_d(int(kind), atoms.shape[0], _p(atoms), _p(params), pstride, _p(q), q.shape[0], _p(qs),
                        _p(qz), _p(out))
    return out


def pair_fe_abs(kind, atoms, params, queries, Qs, QZs):
    """Per channel, the sum over atoms and tip-charge sites of |contribution| at (n,3) query points
    (FP64, uncapped) -> (n,4): the cancellation scale of a grid value."""
    atoms = np.ascontiguousarray(atoms, dtype=np.float64).reshape(-1, 4)
    pstride = 2 if kind == 0 else 4
    params = np.ascontiguousarray(params, dtype=np.float64).reshape(-1, pstride)
    q = np.ascontiguousarray(queries, dtype=np.float64).reshape(-1, 3)
    out = np.zeros((q.shape[0], 4), dtype=np.float64)
    qs, qz = _v4(Qs, np.float64), _v4(QZs, np.float64)
    lib().ora_pair_fe_abs_d(int(kind), atoms.shape[0], _p(atoms), _p(params), pstride, _p(q), q.shape[0], _p(qs),
                            _p(qz), _p(out))
    return out


# ---------------------------------------------------------------- stage (b)
def _grid_args(grid):
    nz, ny, nx = grid.shape[:3]
    return int(nx), int(ny), int(nz)


def relax_strokes(grid, dinv, pts, nz, dTip, stiffness, dpos0, relax, max_iter=128, f2conv=1e-8, use_fire=True,
                  flip=False, prec="f32", polish=False):
    """relaxStrokes -> FEs, disps (n_scan,nz,4). prec 'f32' (bit-exact canon) or 'f64'.
    polish: Newton-polish each z-step's equilibrium (the kernels' SPM_FLAG_POLISH)."""
    dt = np.float32 if prec == "f32" else np.float64
    g = np.ascontiguousarray(grid, dtype=dt)
    pts = np.ascontiguousarray(pts, dtype=np.float32).reshape(-1, 4)
    n_scan = pts.shape[0]
    FEs = np.zeros((n_scan, nz, 4), dtype=dt)
    disps = np.zeros((n_scan, nz, 4), dtype=dt)
    vs = [_v4(v) for v in (dinv[0], dinv[1], dinv[2])]
    ps = [_v4(v) for v in (dTip, stiffness, dpos0, relax)]
    fn = lib().ora_relax_strokes_f if prec == "f32" else lib().ora_relax_strokes_d
    fn(_p(g), *_grid_args(g), *[_p(v) for v in vs], _p(pts), n_scan, int(nz), *[_p(v) for v in ps], int(max_iter),
       float(f2conv), int(bool(use_fire)), int(bool(flip)), int(bool(polish)), _p(FEs), _p(disps))
    return FEs, disps


def relax_2d(grid, dinv, pts, nz, K_lat, dh, dt, damp, max_iter=128, f2conv=1e-8, flip=False):
    """relaxStrokes2D (kernels/AFM.cl:410-450) -> FEs, disps (n_scan,nz,4), canonical FP32."""
    g = np.ascontiguousarray(grid, dtype=np.float32)
    pts = np.ascontiguousarray(pts, dtype=np.float32).reshape(-1, 4)
    n_scan = pts.shape[0]
    FEs = np.zeros((n_scan, nz, 4), dtype=np.float32)
    disps = np.zeros((n_scan, nz, 4), dtype=np.float32)
    vs = [_v4(v) for v in (dinv[0], dinv[1], dinv[2])]
    lib().ora_relax_2d_f(_p(g), *_grid_args(g), *[_p(v) for v in vs], _p(pts), n_scan, int(nz), float(K_lat),
                         float(dh), float(dt), float(damp), int(max_iter), float(f2conv), int(bool(flip)), _p(FEs),
                         _p(disps))
    return FEs, disps


def relax_tilted(grid, dinv, pts, nz, tipA, tipB, tipC, stiffness, dpos0, relax, surfFF, max_iter=128, f2conv=1e-8,
                 use_fire=True, prec="f32", polish=False):
    dt = np.float32 if prec == "f32" else np.float64
    g = np.ascontiguousarray(grid, dtype=dt)
    pts = np.ascontiguousarray(pts, dtype=np.float32).reshape(-1, 4)
    n_scan = pts.shape[0]
    FEs = np.zeros((n_scan, nz, 4), dtype=dt)
    vs = [_v4(v) for v in (dinv[0], dinv[1], dinv[2])]
    ps = [_v4(v) for v in (tipA, tipB, tipC, stiffness, dpos0, relax, surfFF)]
    fn = lib().ora_relax_tilted_f if prec == "f32" else lib().ora_relax_tilted_d
    fn(_p(g), *_grid_args(g), *[_p(v) for v in vs], _p(pts), n_scan, int(nz), *[_p(v) for v in ps], int(max_iter),
       float(f2conv), int(bool(use_fire)), int(bool(polish)), _p(FEs))
    return FEs


def relax_pp(grid, dinv, pts, nz, tipA, tipB, tipC, stiffness, dpos0, relax, surfFF, max_iter=128, f2conv=1e-8,
             use_fire=True, prec="f32", polish=False):
    """Grid relaxation with equilibrium bookkeeping -> FEs, PPs (n_scan,nz,4)."""
    dt = np.float32 if prec == "f32" else np.float64
    g = np.ascontiguousarray(grid, dtype=dt)
    pts = np.ascontiguousarray(pts, dtype=np.float32).reshape(-1, 4)
    n_scan = pts.shape[0]
    FEs = np.zeros((n_scan, nz, 4), dtype=dt)
    PPs = np.zeros((n_scan, nz, 4), dtype=dt)
    vs = [_v4(v, dt) for v in (dinv[0], dinv[1], dinv[2])]
    ps = [_v4(v, dt) for v in (tipA, tipB, tipC, stiffness, dpos0, relax, surfFF)]
    fn = lib().ora_relax_pp_f if prec == "f32" else lib().ora_relax_pp_d
    fn(_p(g), *_grid_args(g), *[_p(v) for v in vs], _p(pts), n_scan, int(nz), *[_p(v) for v in ps], int(max_iter),
       float(f2conv), int(bool(use_fire)), int(bool(polish)), _p(FEs), _p(PPs))
    return FEs, PPs


def raw_tilted(grid, dinv, pts, nz, tipA, tipB, tipC, dTip, dpos0, prec="f32"):
    dt = np.float32 if prec == "f32" else np.float64
    g = np.ascontiguousarray(grid, dtype=dt)
    pts = np.ascontiguousarray(pts, dtype=np.float32).reshape(-1, 4)
    n_scan = pts.shape[0]
    FEs = np.zeros((n_scan, nz, 4), dtype=dt)
    vs = [_v4(v) for v in (dinv[0], dinv[1], dinv[2])]
    ps = [_v4(v) for v in (tipA, tipB, tipC, dTip, dpos0)]
    fn = lib().ora_raw_tilted_f if prec == "f32" else lib().ora_raw_tilted_d
    fn(_p(g), *_grid_args(g), *[_p(v) for v in vs], _p(pts), n_scan, int(nz), *[_p(v) for v in ps], _p(FEs))
    return FEs


def relax_direct(atoms, cMs, pts, nz, tipA, tipB, tipC, stiffness, dpos0, relax, surfFF, Qs, QZs, max_iter=128,
                 f2conv=1e-8, test_oracle_loop=False):
    """relaxStrokesTiltedMorseDirect in FP64 -> FEs, PPs (n_scan,nz,4).

    test_oracle_loop=True reproduces the loop structure of the reference's
    FP64 test oracle _cpu_relax_direct (tests/SPM/test_afm_morse.py:548-604),
    which keeps v across z-steps and threads (dt, damp) through the scan
    points, unlike the kernel (kernels/AFM.cl:1441-1466)."""
    atoms = np.ascontiguousarray(atoms, dtype=np.float64).reshape(-1, 4)
    cMs = np.ascontiguousarray(cMs, dtype=np.float64).reshape(-1, 4)
    pts = np.ascontiguousarray(pts, dtype=np.float32).reshape(-1, 4)
    n_scan = pts.shape[0]
    FEs = np.zeros((n_scan, nz, 4), dtype=np.float64)
    PPs = np.zeros((n_scan, nz, 4), dtype=np.float64)
    ps = [_v4(v) for v in (tipA, tipB, tipC, stiffness, dpos0, relax, surfFF, Qs, QZs)]
    lib().ora_relax_direct_d(atoms.shape[0], _p(atoms), _p(cMs), _p(pts), n_scan, int(nz), *[_p(v) for v in ps],
                             int(max_iter), float(f2conv), 3 if test_oracle_loop else 0, _p(FEs), _p(PPs))
    return FEs, PPs


# ---------------------------------------------------------------- stage (c), NumPy
def _dir_spacing(spacing, osc_dir):
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
    return n, dr


def _linear_nearest(F, coords):
    """Linear interpolation of the 3-D array F at coords (3,...) with clamped indices."""
    acc = np.zeros(coords.shape[1:], dtype=np.float64)
    i0, w = [], []
    for d in range(3):
        fl = np.floor(coords[d])
        t = coords[d] - fl
        i0.append(fl.astype(np.int64))
        w.append((1.0 - t, t))
    for a0 in (0, 1):
        for a1 in (0, 1):
            for a2 in (0, 1):
                ii = [np.clip(i0[d] + a, 0, F.shape[d] - 1) for d, a in zip(range(3), (a0, a1, a2))]
                acc += ((F[ii[0], ii[1], ii[2]] * w[0][a0]) * w[1][a1]) * w[2][a2]
    return acc


def _gradient(f, h, axis):
    """numpy.gradient semantics: central inside, one-sided (edge_order=1) at the ends."""
    f = np.moveaxis(f, axis, 0)
    out = np.empty_like(f)
    out[1:-1] = (f[2:] - f[:-2]) / (2.0 * h)
    out[0] = (f[1] - f[0]) / h
    out[-1] = (f[-1] - f[-2]) / h
    return np.moveaxis(out, 0, axis)


QUAD_N = 9


def quad_nodes():
    k = np.arange(QUAD_N)
    return np.cos((2 * k + 1) / (2 * QUAD_N) * np.pi), np.full(QUAD_N, 1.0 / QUAD_N)


def compute_df_dir(FEs, spacing, osc_dir=(0., 0., 1.)):
    FEs = np.asarray(FEs)
    n, dr = _dir_spacing(spacing, osc_dir)
    F_n = FEs[..., 0] * n[0] + FEs[..., 1] * n[1] + FEs[..., 2] * n[2]
    df = np.zeros(F_n.shape, dtype=np.float64)
    for ia in np.flatnonzero(np.abs(n) > 1e-15):
        df -= n[ia] * _gradient(F_n.astype(np.float64), dr[ia], ia)
    return df


def compute_df_amp_dir(FEs, spacing, osc_dir=(0., 0., 1.), amp=1.0):
    FEs = np.asarray(FEs)
    n, dr = _dir_spacing(spacing, osc_dir)
    F_n = (FEs[..., 0] * n[0] + FEs[..., 1] * n[1] + FEs[..., 2] * n[2]).astype(np.float64)
    active = np.flatnonzero(np.abs(n) > 1e-15)
    u_k, w_k = quad_nodes()
    df = np.zeros(F_n.shape, dtype=np.float64)
    coords0 = np.indices(F_n.shape, dtype=np.float64)
    shift = (float(amp) * n / dr).reshape(3, 1, 1, 1)
    for uk, wk in zip(u_k, w_k):
        S = _linear_nearest(F_n, coords0 + uk * shift)
        for ia in active:
            df -= wk * n[ia] * _gradient(S, dr[ia], ia)
    return df.astype(np.float32)


def compute_df(Fz, dz):
    FEs = np.zeros(np.shape(Fz) + (4,))
    FEs[..., 2] = Fz
    return -_gradient(np.asarray(Fz, dtype=np.float64), abs(dz), 2)


def compute_df_amp(Fz, dz, amp=1.0):
    FEs = np.zeros(np.shape(Fz) + (4,))
    FEs[..., 2] = Fz
    return compute_df_amp_dir(FEs, (1.0, 1.0, abs(dz)), (0., 0., 1.), amp)


def df_loss_seed(FEs, target_df, dtip, weights=None):
    FEs = np.asarray(FEs)
    target = np.asarray(target_df, dtype=np.float64)
    nx, ny, nz = FEs.shape[:3]
    if weights is None:
        w = np.ones((nx, ny, nz))
        w[:, :, 0] = 0.0
        w[:, :, -1] = 0.0
    else:
        w = np.asarray(weights, dtype=np.float64)
    Fz = FEs[..., 2].astype(np.float64)
    dz = abs(float(dtip))
    df = np.zeros((nx, ny, nz))
    df[:, :, 1:-1] = -(Fz[:, :, 2:] - Fz[:, :, :-2]) / (2.0 * dz)
    diff = df - target
    wsum = float(w.sum())
    loss = 0.5 * float(np.sum(w * diff ** 2)) / wsum
    g = w * diff / wsum
    c = 1.0 / (2.0 * dz)
    dFz = np.zeros((nx, ny, nz))
    dFz[:, :, 1:-1] = (g[:, :, 2:] - g[:, :, :-2]) * c
    dFz[:, :, 0] = g[:, :, 1] * c
    dFz[:, :, -1] = -g[:, :, -2] * c
    dL = np.zeros((nx, ny, nz, 4))
    dL[..., 2] = dFz
    return loss, df, dL


def compute_dissipation(FEs_fwd, FEs_bwd, h_scan, h_df, amp, osc_dir=(0., 0., 1.)):
    Ff = np.asarray(FEs_fwd, dtype=np.float64)
    Fb = np.asarray(FEs_bwd, dtype=np.float64)
    h_scan = np.asarray(h_scan, dtype=np.float64)
    n = np.asarray(osc_dir, dtype=np.float64)
    n = n / np.linalg.norm(n)
    amp_z = float(amp) * abs(n[2])
    dF = (Ff[..., 0] * n[0] + Ff[..., 1] * n[1] + Ff[..., 2] * n[2]) - \
         (Fb[..., 0] * n[0] + Fb[..., 1] * n[1] + Fb[..., 2] * n[2])
    nz = dF.shape[2]
    out = np.zeros(dF.shape[:2] + (len(h_df),), dtype=np.float32)
    for i, h in enumerate(np.asarray(h_df, dtype=np.float64)):
        mask = (h_scan >= h - amp_z) & (h_scan <= h + amp_z)
        if mask.sum() < 2:
            mask = np.ones(nz, dtype=bool)
        x = h_scan[mask]
        y = dF[:, :, mask]
        out[:, :, i] = np.abs(np.sum(np.diff(x) * (y[:, :, 1:] + y[:, :, :-1]) / 2.0, axis=2))
    return out


def convolve_z(FEs, weights, nz_out):
    """convolveZ (kernels/AFM.cl:666-701) on the z-columns of FEs (..., nz_in, 4), canonical FP32."""
    F = np.ascontiguousarray(FEs, dtype=np.float32)
    nz_in = F.shape[-2]
    w = np.ascontiguousarray(weights, dtype=np.float32).ravel()
    assert w.size == nz_in - nz_out
    out = np.zeros(F.shape[:-2] + (nz_out, 4), np.float32)
    ncol = int(np.prod(F.shape[:-2]))
    lib().ora_convolve_z_f(_p(F), ncol, int(nz_in), int(nz_out), _p(w), _p(out))
    return out


def izo_z(FEs, iso):
    """izoZ (kernels/AFM.cl:705-723) on the z-columns of FEs (..., nz, 4), canonical FP32."""
    F = np.ascontiguousarray(FEs, dtype=np.float32)
    out = np.zeros(F.shape[:-2], np.float32)
    lib().ora_izo_z_f(_p(F), int(out.size), int(F.shape[-2]), float(iso), _p(out))
    return out


def dinv_axis_aligned(L, origin, n):
    """(dinvA,dinvB,dinvC) with the half-texel offset (spammm/SPM/AFM.py:274-285)."""
    nx, ny, nz = n
    return (np.array([1. / L[0], 0., 0., -origin[0] / L[0] + 0.5 / nx], dtype=np.float32),
            np.array([0., 1. / L[1], 0., -origin[1] / L[1] + 0.5 / ny], dtype=np.float32),
            np.array([0., 0., 1. / L[2], -origin[2] / L[2] + 0.5 / nz], dtype=np.float32))
