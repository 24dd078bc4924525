"""Builds the benchmark's comparison arm libsdx_plain_fp64.so (sm_100a) in-tree with nvcc.

The plain FP64 PCG (cuSPARSE + cuBLAS, the structure of the reference's krylov::CudaPCG) is not part of
libsdx_b200.so: the benchmark plugs it into sdx_step through sdx_set_linear_solver.
Run: python -m bench_arms.build
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libsdx_plain_fp64.so")
SRC = os.path.join(HERE, "plain_fp64.cu")
HEADER = os.path.join(HERE, "..", "include", "sdx_b200.h")


def build(force: bool = False) -> str:
    from project_superdex_b200.build import ARCH, nvcc
    if not force and os.path.exists(LIB) and all(os.path.getmtime(d) < os.path.getmtime(LIB) for d in (SRC, HEADER)):
        return LIB
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler", "-fPIC", "-ccbin",
           "/usr/bin/g++", "-o", LIB + ".tmp", SRC, "-lcusparse", "-lcublas", "-Xlinker", "--no-undefined"]
    subprocess.check_call(cmd)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    sys.path.insert(0, os.path.join(HERE, ".."))
    print(build(force="--force" in sys.argv))
