"""Build libsphgpu.so (the engine) in-tree for sm_100a.

    python multiphase-sph-solver_b200/build.py

nvcc compiles the kernels and the C-ABI host code into one shared library next
to this file.  -fmad=false keeps every FP64 multiply and add separately
rounded (no contraction into fused multiply-adds), as the reference's x86-64
build rounds them; the FP64 drop-in form therefore follows the reference's
arithmetic operation for operation.  The FP32-bulk form
(sph_kernels_bulk32.cu) is compiled with contraction allowed.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libsphgpu.so")
# the bounds-checked build (SPHGPU_CHECK=1): the same sources with an index
# check after the neighbour search that sets an error code instead of trapping
LIB_CHECK = os.path.join(HERE, "libsphgpu_check.so")
SOURCES = ["sph_kernels.cu", "sph_capi.cu", "sph_noalloc.cu", "sph_kernels_bulk32.cu", "sph_kl.cu", "sph_kl_tc.cu",
           "sph_rf.cu", "sph_peaks.cu"]
# per-source flags on top of NVCC_FLAGS
SOURCE_FLAGS = {"sph_kernels_bulk32.cu": ["-fmad=true"]}
HEADERS = ["sph_device.cuh", "sph_constitutive.cuh", os.path.join("..", "..", "include", "sphgpu.h")]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
]


def _stale(lib: str = LIB) -> bool:
    if not os.path.exists(lib):
        return True
    t = os.path.getmtime(lib)
    deps = [os.path.join(CSRC, s) for s in SOURCES + HEADERS] + [__file__]
    return any(os.path.getmtime(p) > t for p in deps if os.path.exists(p))


def build(force: bool = False, verbose: bool = False, check: bool = False) -> str:
    lib = LIB_CHECK if check else LIB
    if not force and not _stale(lib):
        return lib
    nvcc = os.environ.get("NVCC", "nvcc")
    objdir = os.path.join(HERE, "_build_check" if check else "_build")
    os.makedirs(objdir, exist_ok=True)
    procs, objs = [], []
    for src in SOURCES:
        obj = os.path.join(objdir, os.path.splitext(src)[0] + ".o")
        flags = SOURCE_FLAGS.get(src, ["-fmad=false"]) + (["-DSPHGPU_CHECK=1"] if check else [])
        cmd = [nvcc] + NVCC_FLAGS + flags + ["-c", "-o", obj, os.path.join(CSRC, src)]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
            print(" ".join(cmd))
        procs.append(subprocess.Popen(cmd))
        objs.append(obj)
    for p in procs:
        if p.wait() != 0:
            raise subprocess.CalledProcessError(p.returncode, "nvcc")
    subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", lib] + objs, check=True)
    return lib


if __name__ == "__main__":
    check = "--check" in sys.argv
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv, check=check))
