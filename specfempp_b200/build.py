"""Build libsfg.so in-tree for sm_100a (nvcc; no JIT cache)."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SOURCES = ["csrc/sfg.cu", "csrc/sfg3d.cu", "csrc/host2d.cpp"]
HEADERS = ["csrc/kernels2d.cuh", "csrc/kernels2d_batched.cuh", "csrc/kernels2d_adjoint.cuh", "csrc/kernels2d_tma.cuh", "csrc/kernels2d_tile.cuh", "csrc/kernels2d_tile_batched.cuh", "csrc/kernels2d_row.cuh", "csrc/kernels2d_btile.cuh", "csrc/kernels3d.cuh", "csrc/host2d.hpp", "../include/sfg.h", "../include/sfg3d.h"]
# -fmad=false: products and sums are rounded separately unless a kernel asks
# for an FMA explicitly, so every launch shape of a kernel (and the CPU oracle,
# built with contraction off) performs the same rounding steps.
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
              "-fmad=false", "-Xcompiler", "-fPIC,-O3,-fopenmp", "-shared", "-lgomp"]


def nvcc() -> str:
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def build(force: bool = False, verbose: bool = False) -> str:
    out = os.path.join(HERE, "libsfg.so")
    deps = [os.path.join(HERE, s) for s in SOURCES + HEADERS]
    if not force and os.path.exists(out) and all(os.path.getmtime(out) >= os.path.getmtime(d) for d in deps):
        return out
    cmd = [nvcc(), *NVCC_FLAGS, "-o", out, *[os.path.join(HERE, s) for s in SOURCES]]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return out


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
