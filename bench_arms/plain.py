"""The plain FP64 comparison solver (libsdx_plain_fp64.so) plugged into a SoftBodyWorld's Newton solves.

It restates the reference's CUDA solver path (krylov::CudaPCG: cuSPARSE bsrmv, cuBLAS, graph bursts
with a host convergence check, one env after the other) and is used by the benchmark's `plain_fp64` arm
and its test; libsdx_b200.so itself has one solver.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsdx_plain_fp64.so")
_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `python -m bench_arms.build`")
        from project_superdex_b200 import capi
        capi.lib()  # the hook's types come from libsdx_b200.so's header; load it first
        L = C.CDLL(LIB_PATH)
        L.sdx_plain_fp64_create.restype = C.c_void_p
        L.sdx_plain_fp64_destroy.argtypes = [C.c_void_p]
        _lib = L
    return _lib


class PlainFp64:
    """One plain solver instance attached to one world (its structure is built on the first solve)."""

    def __init__(self, world):
        L = lib()
        self._h = L.sdx_plain_fp64_create()
        self._world = world
        world.set_linear_solver(C.cast(L.sdx_plain_fp64_solve, C.c_void_p), self._h)

    def close(self):
        if self._h:
            if getattr(self._world, "_ctx", None):
                self._world.set_linear_solver(None, None)
            lib().sdx_plain_fp64_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()
