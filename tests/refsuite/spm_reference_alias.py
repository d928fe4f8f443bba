"""pytest plugin for running the SPAMMM reference's own hot-path tests against
this drop-in (tests/refsuite/run_reference_suite.py loads it with -p).

It makes the reference's import paths resolve to the drop-in before the test
modules are collected:

  spammm.SPM.AFM        -> spammm_b200.AFM
  spammm.SPM.AFM_utils  -> spammm_b200.AFM_utils

and supplies the two third-party modules the reference's test files import but
this image lacks:

  pyopencl    only enqueue_copy(queue, host, image, origin, region) is used by
              the tests (to read back AFMulator.img_FF); here it synchronises
              and copies the CUDA grid's bytes into the host buffer in the
              order an OpenCL image read writes them (x fastest), which is
              this grid's memory order;
  matplotlib  an inert stand-in (the helpers import it for plotting only).
"""
import importlib
import sys
import types


def _stub_pyopencl():
    cl = types.ModuleType("pyopencl")

    def enqueue_copy(queue, dest, src, origin=None, region=None, **kw):
        import numpy as np
        import torch
        if isinstance(src, torch.Tensor):
            torch.cuda.synchronize()
            host = src.detach().contiguous().cpu().numpy()
            flat = np.asarray(dest).reshape(-1)
            flat[:host.size] = host.reshape(-1).astype(flat.dtype, copy=False)
            return None
        raise NotImplementedError("pyopencl stand-in: only device-grid -> host copies are provided")

    cl.enqueue_copy = enqueue_copy
    return cl


class _Inert:
    """A figure, axes or artist that accepts every call and draws nothing."""

    def __getattr__(self, name):
        return self

    def __call__(self, *a, **k):
        return self


def _stub_matplotlib():
    mpl = types.ModuleType("matplotlib")
    mpl.use = lambda *a, **k: None
    mpl.__path__ = []
    plt = types.ModuleType("matplotlib.pyplot")

    def subplots(nrows=1, ncols=1, **kw):
        import numpy as np
        axes = np.empty((nrows, ncols), dtype=object)
        for i in range(nrows):
            for j in range(ncols):
                axes[i, j] = _Inert()
        if kw.get("squeeze", True):
            axes = axes[0, 0] if nrows == ncols == 1 else (axes.ravel() if 1 in (nrows, ncols) else axes)
        return _Inert(), axes

    plt.subplots = subplots
    plt.__getattr__ = lambda name: _Inert()
    mpl.pyplot = plt
    return mpl, plt


def pytest_load_initial_conftests(early_config, parser, args):
    _install()


def _install():
    afm = importlib.import_module("spammm_b200.AFM")
    utils = importlib.import_module("spammm_b200.AFM_utils")
    pkg = sys.modules.get("spammm") or types.ModuleType("spammm")
    if not hasattr(pkg, "__path__"):
        pkg.__path__ = []
    spm = types.ModuleType("spammm.SPM")
    spm.__path__ = []
    spm.AFM, spm.AFM_utils = afm, utils
    pkg.SPM = spm
    sys.modules.update({"spammm": pkg, "spammm.SPM": spm, "spammm.SPM.AFM": afm, "spammm.SPM.AFM_utils": utils})
    try:
        import pyopencl  # noqa: F401
    except ImportError:
        sys.modules["pyopencl"] = _stub_pyopencl()
    try:
        import matplotlib  # noqa: F401
    except ImportError:
        mpl, plt = _stub_matplotlib()
        sys.modules.update({"matplotlib": mpl, "matplotlib.pyplot": plt})
