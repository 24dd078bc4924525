"""Batched soft-body executor: the state boundary between a Python environment loop and the
device-resident envs of one SoftBodyWorld.

Mirrors the contract of the reference's SceneBatchExecutorV2 (mochi_physics/pybind/src/
scene_batch_executor_v2.cpp:55-1275): `write_state` with per-DoF write masks, `step(time_step_sec,
generalized_forces, qpos_out, qvel_out, link_state_out, contact_out, diverged_out, readback_mask)` that
fills only the caller's buffers the readback mask selects (and refuses buffers it does not select),
`close` / context-manager use, and the Scene state snapshots the Lab environments take around every
environment step (`capture_state`, `restore_state(handle, release_immediately)`, superdex_lab/superdex/
lab/gym/envs/mochi_env.py:786-821), here device-resident.

The soft envs differ from the reference's articulated slots in two ways: the DoFs are the nodal
displacements (qpos) and velocities (qvel) of every body, concatenated env after env in node order
(`scene_dof_offsets`, ragged: uneven bodies have different DoF counts); and there is no generalized force
input (the reference's soft actors do not read external DoF forces), so `generalized_forces` must be None
or zero. `contact_out[s]` is the number of active (sample, collider) pairs of scene s at its last assembly,
`diverged_out[s]` is 1 when its Newton solve diverged.
"""
from __future__ import annotations

import ctypes as C
import math
from typing import Optional

import numpy as np

from . import capi
from .soft_body import SoftBodyWorld

READ_QPOS = 1 << 0
READ_QVEL = 1 << 1
READ_LINKS = 1 << 2
READ_CONTACTS = 1 << 3
READ_DIVERGED = 1 << 4
READ_ALL = READ_QPOS | READ_QVEL | READ_LINKS | READ_CONTACTS | READ_DIVERGED


def validate_time_step(name: str, value: float) -> float:
    """A finite, positive step (backward Euler divides by it; the reference also allows 0 for its
    articulated slots, which a soft step cannot take)."""
    v = float(value)
    if not math.isfinite(v) or v <= 0.0:
        raise ValueError(f"{name} requires a finite, positive time_step_sec")
    return v


def validate_readback(readback_mask: int, n_dofs: int, n_scenes: int, qpos_out, qvel_out, link_state_out,
                      contact_out, diverged_out):
    """The reference's ValidateReadback (scene_batch_executor_v2.cpp:672-745): unknown bits are refused;
    a selected output needs a C-contiguous buffer of the right size and dtype, an unselected one must
    be None. Links do not exist for soft envs."""
    if readback_mask & ~READ_ALL:
        raise ValueError("readback_mask has unknown bits")

    def check(flag, buf, size, dtype, name):
        if not (readback_mask & flag):
            if buf is not None:
                raise ValueError(f"{name} given but not selected by readback_mask")
            return
        if buf is None:
            raise ValueError(f"readback_mask selects {name} but it is None")
        if not isinstance(buf, np.ndarray) or buf.dtype != dtype or not buf.flags.c_contiguous or buf.size != size:
            raise ValueError(f"{name} must be a C-contiguous {np.dtype(dtype).name} array of {size} entries")

    check(READ_QPOS, qpos_out, n_dofs, np.float64, "qpos_out")
    check(READ_QVEL, qvel_out, n_dofs, np.float64, "qvel_out")
    if readback_mask & READ_LINKS or link_state_out is not None:
        raise ValueError("soft envs have no links: READ_LINKS and link_state_out are not supported")
    check(READ_CONTACTS, contact_out, n_scenes, np.float64, "contact_out")
    check(READ_DIVERGED, diverged_out, n_scenes, np.uint8, "diverged_out")


class SoftSceneBatchExecutor:
    """One device-resident batch of soft envs behind the executor contract (see the module docstring)."""

    abi_version = 2

    def __init__(self, world: SoftBodyWorld):
        self._w = world
        self._closed = False
        self._dt = float(world.params.dt)
        counts = 3 * np.diff(np.asarray(world.node_off, np.int64))
        self.scene_dof_counts = counts
        self.scene_dof_offsets = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)

    # layout -------------------------------------------------------------------------------------
    @property
    def num_scenes(self) -> int:
        return self._w.n_envs

    @property
    def num_actors(self) -> int:
        return 1  # one soft body per scene

    @property
    def num_dofs(self) -> int:
        return 3 * self._w.n_nodes

    @property
    def num_links(self) -> int:
        return 0

    @property
    def closed(self) -> bool:
        return self._closed

    @property
    def world(self) -> SoftBodyWorld:
        return self._w

    def _live(self):
        if self._closed:
            raise RuntimeError("SoftSceneBatchExecutor is closed")

    # state ------------------------------------------------------------------------------------
    def write_state(self, qpos=None, qvel=None, qpos_write_mask=None, qvel_write_mask=None):
        self._live()
        if (qpos is None) != (qpos_write_mask is None) or (qvel is None) != (qvel_write_mask is None):
            raise ValueError("values and their write mask are given together")  # RequireWritePayload
        self._w.write_state(qpos, qvel, qpos_write_mask, qvel_write_mask)

    def step(self, time_step_sec: float, generalized_forces=None, qpos_out: Optional[np.ndarray] = None,
             qvel_out: Optional[np.ndarray] = None, link_state_out=None, contact_out: Optional[np.ndarray] = None,
             diverged_out: Optional[np.ndarray] = None, readback_mask: int = READ_QPOS | READ_QVEL):
        self._live()
        dt = validate_time_step("step", time_step_sec)
        if generalized_forces is not None and np.any(np.asarray(generalized_forces) != 0):
            raise ValueError("soft envs take no generalized forces")
        validate_readback(readback_mask, self.num_dofs, self.num_scenes, qpos_out, qvel_out, link_state_out,
                          contact_out, diverged_out)
        if dt != self._dt:
            self._w.set_params(dt=dt)
            self._dt = dt
        self._w.step(1)
        if readback_mask & (READ_QPOS | READ_QVEL):  # only the selected vectors cross to the host
            t = C.c_double()
            qp = qpos_out if readback_mask & READ_QPOS else None
            qv = qvel_out if readback_mask & READ_QVEL else None
            capi.check(capi.lib().sdx_get_state(self._w._ctx, capi.ptr(qp), capi.ptr(qv), C.byref(t)))
        if readback_mask & (READ_CONTACTS | READ_DIVERGED):
            st = self._w.stats()
            if readback_mask & READ_CONTACTS:
                contact_out[:] = [s["n_contacts"] for s in st]
            if readback_mask & READ_DIVERGED:
                diverged_out[:] = [1 if s["convergence"] == 3 else 0 for s in st]

    # snapshots (Scene.capture_state / restore_state) ---------------------------------------------
    def capture_state(self) -> int:
        self._live()
        return self._w.capture_state()

    def restore_state(self, handle: int, release_immediately: bool = False, env_mask=None):
        self._live()
        self._w.restore_state(handle, release_immediately, env_mask)

    def release_state(self, handle: int):
        self._w.release_state(handle)

    # lifetime ---------------------------------------------------------------------------------
    def close(self):
        if not self._closed:
            self._closed = True
            self._w.release_all_states()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
