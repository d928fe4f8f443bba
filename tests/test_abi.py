"""The C ABI library loads, exports every symbol include/spm_b200.h declares,
and rejects bad arguments before touching the device (no GPU needed)."""
import ctypes
import os
import re

import numpy as np
import pytest

from spammm_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "spm_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(spm_\w+)\s*\(", src, flags=re.M)))


def test_header_declares_the_boundary():
    names = declared_functions()
    for must in ("spm_grid_build", "spm_relax_strokes", "spm_relax_strokes_tilted", "spm_fe_in_strokes_tilted",
                 "spm_df_amp_dir", "spm_df_dir", "spm_dissipation", "spm_df_loss_seed", "spm_relax_direct_morse",
                 "spm_adjoint_direct_state", "spm_adjoint_direct_params", "spm_last_error", "spm_abi_version"):
        assert must in names


def test_library_exports_every_declared_symbol():
    L = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_binding_covers_every_declared_symbol():
    assert set(declared_functions()) <= set(_lib.exported_symbols())


def test_abi_version_and_error_text():
    L = _lib.lib()
    assert L.spm_abi_version() == 4
    assert L.spm_last_error() == b""


def test_scan_params_layout():
    # 11 float[4] + nz, max_iter, f2conv, flags, raster_ny
    assert ctypes.sizeof(_lib.ScanParams) == 11 * 16 + 5 * 4
    p = _lib.make_scan_params(nz=7, max_iter=1000, f2conv=1e-10, fire=True, flip_z=True, raster_ny=5)
    assert p.flags == _lib.SPM_FLAG_FIRE | _lib.SPM_FLAG_FLIP_Z
    assert (p.nz, p.max_iter, p.raster_ny) == (7, 1000, 5)


def test_argument_errors_are_reported_without_a_device():
    L = _lib.lib()
    v = np.zeros(4, np.float32)
    hp = v.ctypes.data_as(ctypes.c_void_p)
    rc = L.spm_grid_build(7, 0, None, None, None, 4, 4, 4, hp, hp, hp, hp, hp, hp, None)
    assert rc == _lib.SPM_ERR_ARG and b"kind" in L.spm_last_error()
    rc = L.spm_grid_build(0, 0, None, None, None, 0, 4, 4, hp, hp, hp, hp, hp, hp, None)
    assert rc == _lib.SPM_ERR_ARG and b"positive" in L.spm_last_error()
    P = _lib.make_scan_params(nz=3)
    rc = L.spm_relax_strokes(None, 4, 4, 4, None, 1, ctypes.byref(P), None, None, None)
    assert rc == _lib.SPM_ERR_ARG
    rc = L.spm_relax_direct_morse(0, ctypes.c_void_p(16), ctypes.c_void_p(16), ctypes.c_void_p(16), 1,
                                  ctypes.byref(P), hp, hp, ctypes.c_void_p(16), ctypes.c_void_p(16), None)
    assert rc == _lib.SPM_ERR_UNSUPPORTED and b"n_atoms" in L.spm_last_error()
    rc = L.spm_df_loss_seed(None, 0, None, None, 2, 2, 2, -0.1, None, None, None, None, None)
    assert rc == _lib.SPM_ERR_ARG


def test_adam_step_arguments_are_checked_before_any_launch():
    """spm_batch_adam_step refuses bad arguments with an error code and text; nothing is launched,
    so the (never dereferenced) buffer addresses need no device."""
    L = _lib.lib()
    p = ctypes.c_void_p(256)
    ok = (0.01, 0.9, 0.999, 1e-8, 15)
    rc = L.spm_batch_adam_step(4, None, p, p, p, p, *ok, None)
    assert rc == _lib.SPM_ERR_ARG and b"null" in L.spm_last_error()
    rc = L.spm_batch_adam_step(4, p, ctypes.c_void_p(260), p, p, p, *ok, None)
    assert rc == _lib.SPM_ERR_ARG and b"aligned" in L.spm_last_error()
    rc = L.spm_batch_adam_step(4, p, p, p, p, p, 0.01, 1.0, 0.999, 1e-8, 15, None)
    assert rc == _lib.SPM_ERR_ARG and b"beta1" in L.spm_last_error()
    rc = L.spm_batch_adam_step(4, p, p, p, p, p, 0.01, 0.9, 0.999, 0.0, 15, None)
    assert rc == _lib.SPM_ERR_ARG and b"eps" in L.spm_last_error()
    rc = L.spm_batch_adam_step(4, p, p, p, p, p, 0.01, 0.9, 0.999, 1e-8, 16, None)
    assert rc == _lib.SPM_ERR_ARG and b"cols" in L.spm_last_error()
    rc = L.spm_batch_adam_step(-1, p, p, p, p, p, *ok, None)
    assert rc == _lib.SPM_ERR_ARG and b"n_atoms" in L.spm_last_error()


def test_check_raises_value_error_for_argument_errors():
    L = _lib.lib()
    v = np.zeros(4, np.float32)
    hp = v.ctypes.data_as(ctypes.c_void_p)
    rc = L.spm_grid_build(5, 0, None, None, None, 4, 4, 4, hp, hp, hp, hp, hp, hp, None)
    with pytest.raises(ValueError):
        _lib.check(rc, "spm_grid_build")
