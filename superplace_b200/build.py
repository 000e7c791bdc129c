"""Builds superplace_b200/libspgpu.so (the C-ABI engine) for sm_100a with nvcc.

Usage: python -m superplace_b200.build [--force]

Host code is compiled with -ffp-contract=off so the host-side float arithmetic (grid
set-up, footprints, clamp boxes) matches the reference's un-contracted expressions.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libspgpu.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

SOURCES = ["engine.cu", "density.cu", "wirelength.cu", "optimizer.cu", "poisson.cu",
           "poisson_tc.cu", "poisson_static.cu", "filler_order.cu", "bookshelf.cpp", "qp.cpp", "qp_device.cu"]
# host sources parallelised with OpenMP
OPENMP = {"qp.cpp"}


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    deps = srcs + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    deps.append(os.path.join(ROOT, "include", "spgpu.h"))
    if not force and not _stale(LIB, deps):
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    base = [NVCC, "-std=c++17", "-O3", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC",
            "-Xcompiler", "-ffp-contract=off", "-I", os.path.join(ROOT, "include"), "-I", CSRC,
            "--expt-relaxed-constexpr", "-ccbin", "/usr/bin/g++"]
    if verbose:
        base += ["-Xptxas", "-v"]
    for src in srcs:
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        if force or _stale(obj, [src] + deps):
            omp = ["-Xcompiler", "-fopenmp"] if os.path.basename(src) in OPENMP else []
            cmd = base + omp + ["-c", src, "-o", obj]
            subprocess.run(cmd, check=True)
        objs.append(obj)
    tmp = LIB + ".tmp"
    subprocess.run([NVCC, *ARCH, "-shared", "-o", tmp, *objs, "-ccbin", "/usr/bin/g++",
                    "-lcudart_static", "-lgomp", "-lrt", "-lpthread", "-ldl"], check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
