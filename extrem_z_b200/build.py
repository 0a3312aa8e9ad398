"""Build the libraries in-tree: extrem_z_b200/libextremz.so (the CUDA library,
sm_100a) and extrem_z_b200/libExtreMz.so (the reference host API
include/api/ExtreM.h over it, compat/extrem_api.cpp)."""

from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libextremz.so")
COMPAT_LIB = os.path.join(PKG, "libExtreMz.so")
COMPAT_SOURCES = [os.path.join(PKG, "compat", "extrem_api.cpp"),
                  os.path.join(PKG, "compat", "extrem_api.h")]

SOURCES = ["extremz_engine.cu"]
HEADERS = ["extremz_common.cuh", "extremz_kernels.cuh", "extremz_batch.cuh", "extremz_encode.cuh",
           "extremz_topo.cuh", "extremz_lut.h"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-fmad=false",            # no contraction: float updates match the oracle bit for bit
    "-Xcompiler", "-fPIC", "-shared",
    "--expt-relaxed-constexpr",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(ROOT, "include", "extremz.h"))
    deps.append(__file__)
    return any(os.path.getmtime(p) > t for p in deps if os.path.exists(p))


def build(force: bool = False, verbose: bool = False, extra=()) -> str:
    if not force and not _stale():
        build_compat()
        return LIB
    tmp = LIB + ".tmp"
    cmd = [nvcc(), *NVCC_FLAGS, *extra, "-I", os.path.join(ROOT, "include"),
           *[os.path.join(CSRC, s) for s in SOURCES], "-o", tmp]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    build_compat(force=True, verbose=verbose)
    return LIB


def build_compat(force: bool = False, verbose: bool = False) -> str:
    """libExtreMz.so: the reference's host API over libextremz.so (found next
    to it at run time)."""
    if not force and os.path.exists(COMPAT_LIB) and all(
            os.path.getmtime(p) <= os.path.getmtime(COMPAT_LIB) for p in COMPAT_SOURCES + [LIB]):
        return COMPAT_LIB
    tmp = COMPAT_LIB + ".tmp"
    cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-O2",
           "-Xcompiler", "-fPIC", "-shared",
           "-I", os.path.join(ROOT, "include"), COMPAT_SOURCES[0], "-o", tmp,
           "-L", PKG, "-lextremz", "-Xlinker", "-rpath", "-Xlinker", "$ORIGIN"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(tmp, COMPAT_LIB)
    return COMPAT_LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas-v" in sys.argv else [])
    print(LIB)
