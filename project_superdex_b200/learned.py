"""Learned CG warm start: data generation from the plain solver, GPU training, evaluation.

The network (sdx_mlp.cu) maps per-vertex, 1-ring-averaged features — displacement, dt * velocity, the last
Newton update, the previous step's update at the same Newton iteration (the temporal warm start) and the
Jacobi-preconditioned Newton gradient, each group divided by the env's RMS of it — to the Newton update
in the same units. Training pairs are (features before a Newton linear
solve, its converged solution) recorded while the plain solver (zero initial guess, the reference's
behaviour at mochi_core/src/solvers/newton_solver.cpp:746) steps seeded episodes. The prediction is only
ever an initial guess: every solve still runs to the same residual tolerance.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np

from . import capi
from .soft_body import SoftBodyWorld


class Mlp:
    """Parameter handle bound to a context (a SoftBodyWorld's, or a standalone one)."""

    def __init__(self, ctx):
        self.ctx = ctx

    def init(self, seed: int = 0):
        capi.check(capi.lib().sdx_mlp_init(self.ctx, seed))

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, np.float32)
        capi.check(capi.lib().sdx_mlp_set_params(self.ctx, p.ctypes.data_as(C.POINTER(C.c_float)), p.size))

    def get_params(self) -> np.ndarray:
        p = np.zeros(capi.SDX_MLP_PARAMS, np.float32)
        capi.check(capi.lib().sdx_mlp_get_params(self.ctx, p.ctypes.data_as(C.POINTER(C.c_float)), p.size))
        return p

    def forward(self, X: np.ndarray) -> np.ndarray:
        X = np.ascontiguousarray(X, np.float32)
        Y = np.zeros((X.shape[0], 3), np.float32)
        capi.check(capi.lib().sdx_mlp_forward(self.ctx, X.ctypes.data_as(C.POINTER(C.c_float)), X.shape[0],
                                              Y.ctypes.data_as(C.POINTER(C.c_float))))
        return Y

    def gradients(self, X: np.ndarray, T: np.ndarray):
        X = np.ascontiguousarray(X, np.float32)
        T = np.ascontiguousarray(T, np.float32)
        g = np.zeros(capi.SDX_MLP_PARAMS, np.float32)
        loss = C.c_double()
        capi.check(capi.lib().sdx_mlp_gradients(self.ctx, X.ctypes.data_as(C.POINTER(C.c_float)),
                                                T.ctypes.data_as(C.POINTER(C.c_float)), X.shape[0],
                                                g.ctypes.data_as(C.POINTER(C.c_float)), C.byref(loss)))
        return loss.value, g

    def train(self, X: np.ndarray, T: np.ndarray, batch: int = 4096, epochs: int = 20, lr: float = 1e-3,
              seed: int = 0) -> np.ndarray:
        X = np.ascontiguousarray(X, np.float32)
        T = np.ascontiguousarray(T, np.float32)
        losses = np.zeros(epochs)
        capi.check(capi.lib().sdx_mlp_train(self.ctx, X.ctypes.data_as(C.POINTER(C.c_float)),
                                            T.ctypes.data_as(C.POINTER(C.c_float)), X.shape[0], batch, epochs,
                                            lr, seed, capi.ptr(losses)))
        return losses


def collect(world: SoftBodyWorld, steps: int, samples_per_solve: int, capacity: int, seed: int = 0):
    """Step `world` with the plain solver and return the recorded (X, T) samples."""
    L = capi.lib()
    capi.check(L.sdx_collect_training(world._ctx, samples_per_solve, capacity, seed))
    world.set_params(warm_start=capi.SDX_WARM_ZERO)
    for _ in range(steps):
        world.step(1)
        n = C.c_int64()
        capi.check(L.sdx_get_training_data(world._ctx, None, None, 0, C.byref(n)))
        if n.value >= capacity:
            break
    n = C.c_int64()
    capi.check(L.sdx_get_training_data(world._ctx, None, None, 0, C.byref(n)))
    m = min(n.value, capacity)
    X = np.zeros((m, 16), np.float32)
    T = np.zeros((m, 3), np.float32)
    capi.check(L.sdx_get_training_data(world._ctx, X.ctypes.data_as(C.POINTER(C.c_float)),
                                       T.ctypes.data_as(C.POINTER(C.c_float)), m, C.byref(n)))
    capi.check(L.sdx_collect_training(world._ctx, 0, 0, 0))
    return X, T


def cg_iterations(world: SoftBodyWorld, steps: int, warm_start: int, params: Optional[np.ndarray] = None):
    """CG iterations per step and Newton iterations per step of `steps` steps with the given warm start."""
    if params is not None:
        Mlp(world._ctx).set_params(params)
    world.set_params(warm_start=warm_start)
    cg, nw = [], []
    for _ in range(steps):
        world.step(1)
        st = world.stats()
        cg.append(sum(s["cg_iters"] for s in st))
        nw.append(sum(s["newton_iters"] for s in st))
    return np.asarray(cg), np.asarray(nw)
