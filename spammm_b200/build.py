"""Builds libspmb200.so in-tree with nvcc for sm_100a.

Each translation unit is compiled with its own flags: the relaxation and df
kernels use ``-fmad=false`` (explicit fused multiply-adds only, so results are
a pure function of the inputs); the grid build keeps FMA contraction.  The
build is incremental on source/header modification times.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libspmb200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I" + INCLUDE, "-I" + CSRC,
          "--expt-relaxed-constexpr"]
# per-file extra flags
UNITS = {
    "capi.cu": [],
    "grid_build.cu": [],
    "relax.cu": ["-fmad=false"],
    "df.cu": ["-fmad=false"],
    "direct.cu": [],
    "adjoint_grid.cu": [],
    "batched.cu": [],
    "zmaps.cu": ["-fmad=false"],
}


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _mtime(p):
    try:
        return os.path.getmtime(p)
    except OSError:
        return 0.0


def build(verbose=False, force=False):
    """Compile every CUDA unit present in csrc/ and link libspmb200.so."""
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(INCLUDE, "spm_b200.h"))
    hdr_t = max(_mtime(h) for h in headers)
    nvcc = _nvcc()
    objs = []
    for unit, extra in UNITS.items():
        src = os.path.join(CSRC, unit)
        if not os.path.exists(src):
            continue
        obj = os.path.join(BUILD, unit.replace(".cu", ".o"))
        objs.append(obj)
        if not force and _mtime(obj) > max(_mtime(src), hdr_t, _mtime(__file__)):
            continue
        cmd = [nvcc] + ARCH + COMMON + extra + ["-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    if force or not os.path.exists(LIB) or _mtime(LIB) < max(_mtime(o) for o in objs):
        cmd = [nvcc] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart_static"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
