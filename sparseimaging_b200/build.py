"""Builds libmfista_b200.so in-tree with nvcc for sm_100a.

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
SOURCES = ["mfista_b200.cu", "nufft_noalloc.cu", "unet.cu"]
HEADERS = ["common.cuh", "fft_smem.cuh", "nufft_ops.cuh", "fftvar_ops.cuh", "dft_ops.cuh",
           "mfista_ops.cuh", "fgp.cuh", "solver.cuh", "looe.cuh", "dft_tc.cuh", "cpp_nufft.cuh"]

NVCC_FLAGS = ["-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo",
              "-Xcompiler", "-fPIC", "-shared", "-cudart", "static"]


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(PKG, "..", "include", "mfista_b200.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force=False, verbose=True):
    if not force and not _stale():
        return LIB
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [nvcc] + NVCC_FLAGS + ["-o", LIB] + [os.path.join(CSRC, s) for s in SOURCES]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv)
