"""Builds libmfista_b200.so in-tree with nvcc for sm_100a, and
libmfista_b200_cpp.so (the reference's C++-build names, forwarding to it).

    python -m sparseimaging_b200.build

The library links the CUDA runtime statically, so it depends only on the
driver (libcuda.so) at run time.
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libmfista_b200.so")
CPP_LIB = os.path.join(PKG, "libmfista_b200_cpp.so")
INCLUDE = os.path.abspath(os.path.join(PKG, "..", "include"))
SOURCES = ["mfista_b200.cu", "nufft_noalloc.cu", "unet.cu"]
HEADERS = ["common.cuh", "fft_smem.cuh", "nufft_ops.cuh", "fftvar_ops.cuh", "dft_ops.cuh",
           "mfista_ops.cuh", "fgp.cuh", "solver.cuh", "looe.cuh", "dft_tc.cuh", "cpp_nufft.cuh"]

NVCC_FLAGS = ["-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
              "-Xcompiler", "-fPIC", "-shared", "-cudart", "static"]


def _stale():
    if not os.path.exists(LIB) or not os.path.exists(CPP_LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS + ["cpp_build_abi.c"]]
    deps += [os.path.join(INCLUDE, h) for h in ("mfista_b200.h", "mfista_b200_cpp.h")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force=False, verbose=True):
    if not force and not _stale():
        return LIB
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [nvcc] + NVCC_FLAGS + ["-o", LIB] + [os.path.join(CSRC, s) for s in SOURCES]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    # the C++ build's exported names: a plain C library over LIB
    cc = os.environ.get("CC", "gcc")
    cmd = [cc, "-O2", "-fPIC", "-shared", "-Wall", "-Werror", f"-I{INCLUDE}", "-o", CPP_LIB,
           os.path.join(CSRC, "cpp_build_abi.c"), f"-L{PKG}", f"-l:{os.path.basename(LIB)}", "-Wl,-rpath,$ORIGIN"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv)
