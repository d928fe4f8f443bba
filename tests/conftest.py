"""Shared test plumbing: repo on sys.path, golden fixtures, the gpu marker.

Tests marked ``gpu`` need a CUDA device and the in-tree libspmb200.so; they
fail (not skip) when either is missing, so a GPU run can never pass on a
fallback.  Everything else runs on the CPU.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: longer-running case")


def load_golden(name):
    return dict(np.load(os.path.join(GOLDEN, name), allow_pickle=False))


@pytest.fixture(scope="session")
def golden():
    cache = {}

    def get(name):
        if name not in cache:
            cache[name] = load_golden(name)
        return cache[name]

    return get


@pytest.fixture(scope="session")
def cuda():
    import torch
    assert torch.cuda.is_available(), "GPU test run without a CUDA device"
    from spammm_b200 import _lib
    _lib.lib()  # raises if the in-tree library is missing
    return torch.device("cuda", 0)
