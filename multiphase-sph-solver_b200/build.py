"""Build libsphgpu.so (the engine) in-tree for sm_100a.

    python multiphase-sph-solver_b200/build.py

nvcc compiles the kernels and the C-ABI host code into one shared library next
to this file.  -fmad=false keeps every FP64 multiply and add separately
rounded (no contraction into fused multiply-adds), as the reference's x86-64
build rounds them; the engine's results therefore follow the reference's
arithmetic operation for operation.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libsphgpu.so")
SOURCES = ["sph_kernels.cu", "sph_capi.cu", "sph_noalloc.cu"]
HEADERS = ["sph_device.cuh", "sph_constitutive.cuh", os.path.join("..", "..", "include", "sphgpu.h")]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-fmad=false",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
    "-shared",
]


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, s) for s in SOURCES + HEADERS] + [__file__]
    return any(os.path.getmtime(p) > t for p in deps if os.path.exists(p))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [nvcc] + NVCC_FLAGS + ["-o", LIB] + [os.path.join(CSRC, s) for s in SOURCES]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
