"""The allocation-free df loss seed (spm_df_loss_seed_noalloc) against the
regular entry point (spm_df_loss_seed with caller scratch).

That entry point exists for callers that cannot allocate device memory around
the call: it keeps its partial sums in a fixed device array inside the
library.  This file is collected last so that a run stopping at the first
failure has run every other test already; it also passes alone in a fresh
process (the first call on the device resolves the array's address).
"""
import ctypes

import numpy as np
import pytest
import torch

from spammm_b200 import _lib, gpu

pytestmark = pytest.mark.gpu

MAX_ELEMS = 16777216  # SPM_DF_LOSS_NOALLOC_MAX_ELEMS


def _noalloc(FEs, target, dtip, weights=None):
    """Calls spm_df_loss_seed_noalloc through the C ABI; outputs are torch-allocated here."""
    nx, ny, nz = (int(s) for s in FEs.shape[:3])
    df = torch.empty((nx, ny, nz), dtype=torch.float64, device=FEs.device)
    dL = torch.empty((nx, ny, nz, 4), dtype=torch.float32, device=FEs.device)
    loss = torch.empty((1,), dtype=torch.float64, device=FEs.device)
    dt = _lib.SPM_F64 if FEs.dtype == torch.float64 else _lib.SPM_F32
    rc = _lib.lib().spm_df_loss_seed_noalloc(_lib.ptr(FEs), dt, _lib.ptr(target), _lib.ptr(weights), nx, ny, nz,
                                             float(dtip), _lib.ptr(df), _lib.ptr(dL), _lib.ptr(loss),
                                             _lib.stream_ptr())
    _lib.check(rc, "spm_df_loss_seed_noalloc")
    return loss, df, dL


def test_noalloc_loss_seed_matches_regular_entry_point_twice(cuda):
    rng = np.random.default_rng(2026)
    cases = [((37, 29, 41), torch.float32, -0.1, False), ((64, 50, 60), torch.float64, -0.15, True)]
    for shape, dt, dtip, weighted in cases:  # two calls in a row, different sizes and inputs
        FEs = torch.from_numpy(rng.standard_normal(shape + (4,))).to(dt).cuda()
        tgt = torch.from_numpy(rng.standard_normal(shape)).cuda()
        w = None
        if weighted:
            w = torch.from_numpy(rng.uniform(0.1, 1.0, shape)).cuda()
        l1, d1, g1 = _noalloc(FEs, tgt, dtip, w)
        l2, d2, g2 = gpu.df_loss_seed(FEs, tgt, dtip, w)
        torch.cuda.synchronize()
        assert float(l1) == pytest.approx(float(l2), rel=1e-12)
        assert torch.allclose(d1, d2, rtol=1e-12, atol=1e-12)
        assert torch.allclose(g1, g2, rtol=1e-6, atol=1e-7 * float(g2.abs().max()))


def test_noalloc_loss_seed_at_exactly_the_fixed_limit(cuda):
    """A 256^3 volume fills the fixed array exactly (65536 block partials, the final sums in the last two
    slots): it must agree with the regular entry point, twice in a row."""
    n = 256
    assert n ** 3 == MAX_ELEMS
    g = torch.Generator(device="cuda").manual_seed(7)
    for dtip in (-0.1, -0.2):
        FEs = torch.randn((n, n, n, 4), generator=g, device="cuda", dtype=torch.float32)
        tgt = torch.randn((n, n, n), generator=g, device="cuda", dtype=torch.float64)
        l1, d1, g1 = _noalloc(FEs, tgt, dtip)
        l2, d2, g2 = gpu.df_loss_seed(FEs, tgt, dtip)
        torch.cuda.synchronize()
        assert float(l1) == pytest.approx(float(l2), rel=1e-12)
        assert torch.allclose(d1, d2, rtol=1e-12, atol=1e-12)
        assert torch.allclose(g1, g2, rtol=1e-6, atol=1e-7 * float(g2.abs().max()))
        del FEs, tgt, d1, d2, g1, g2


def test_noalloc_rejects_volumes_above_the_fixed_limit(cuda):
    L = _lib.lib()
    dummy = ctypes.c_void_p(256)
    # exactly one element past the limit (2^24 + 1 = 257 * 65281) and far past it; both are rejected on the
    # host before any launch, so the dummy pointers are never dereferenced
    for nx, ny, nz in ((1, 257, 65281), (4096, 4097, 3)):
        assert nx * ny * nz > MAX_ELEMS
        rc = L.spm_df_loss_seed_noalloc(dummy, _lib.SPM_F32, dummy, None, nx, ny, nz, -0.1, dummy, dummy, dummy, None)
        assert rc == _lib.SPM_ERR_UNSUPPORTED
        assert b"fixed scratch limit" in L.spm_last_error()
