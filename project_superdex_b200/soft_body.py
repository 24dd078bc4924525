"""Batched soft-body world on the GPU: the reference's FEM-body and island-Newton boundary.

A `SoftBodyWorld` holds many independent soft bodies (environments) in one device-resident batch and
advances all of them with `step()`, the analogue of Scene::Step for soft actors
(mochi_physics/src/mochi_scene.cpp:594 -> solver::StepIslandNewtonAsync, mochi_solve.cpp:1090; one
island per env). `assemble()` exposes the FEM-body assembly (AssembleObjResDRes + MakeBatchedBodyOp +
async contact, mochi_soft.cpp:202-474) for parity checks.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np

from . import capi
from .scenes import Body, SceneConfig, concat_bodies


class SoftBodyWorld:
    def __init__(self, bodies: Sequence[Body], cfg: SceneConfig, device: int = 0, **overrides):
        L = capi.lib()
        self.bodies = list(bodies)
        self.cfg = cfg
        self._ctx = L.sdx_create(device)
        if not self._ctx:
            raise capi.SdxError(L.sdx_last_error().decode())
        node_off, tet_off, X, tets = concat_bodies(self.bodies)
        lam = np.concatenate([b.lame()[0] for b in self.bodies])
        mu = np.concatenate([b.lame()[1] for b in self.bodies])
        rho = np.concatenate([b.rho for b in self.bodies]).astype(np.float64)
        pin = np.concatenate([b.pin for b in self.bodies]).astype(np.uint8)
        self.node_off, self.tet_off = node_off, tet_off
        self.n_envs = len(self.bodies)
        self.n_nodes = int(node_off[-1])
        capi.check(L.sdx_upload_bodies(self._ctx, self.n_envs, capi.ptr(node_off, capi._lp),
                                       capi.ptr(tet_off, capi._lp), capi.ptr(np.ascontiguousarray(X)),
                                       capi.ptr(np.ascontiguousarray(tets), capi._ip),
                                       capi.ptr(np.ascontiguousarray(lam)), capi.ptr(np.ascontiguousarray(mu)),
                                       capi.ptr(rho), capi.ptr(pin, capi._up)))
        rows, envs = [], []
        for e, b in enumerate(self.bodies):
            for c in b.colliders:
                rows.append(c.as_row())
                envs.append(e)
        self.n_colliders = len(rows)
        mats = np.asarray([int(getattr(b, "material", 0)) for b in self.bodies], np.int32)
        if np.any(mats != 0):
            capi.check(L.sdx_set_materials(self._ctx, self.n_envs, capi.ptr(mats, capi._ip)))
        if rows:
            R = np.ascontiguousarray(np.stack(rows))
            E = np.asarray(envs, np.int32)
            capi.check(L.sdx_set_colliders(self._ctx, len(rows), capi.ptr(E, capi._ip), capi.ptr(R)))
        self.params = capi.default_step_params()
        self.params.dt = cfg.dt
        for k in range(3):
            self.params.gravity[k] = cfg.gravity[k]
        self.params.k_contact, self.params.t_half = cfg.k_contact, cfg.t_half
        self.params.thr, self.params.max_align = cfg.thr, cfg.max_align
        self.params.mass_damping = float(getattr(cfg, "mass_damping", 0.0))
        self.params.stiffness_damping = float(getattr(cfg, "stiffness_damping", 0.0))
        self.params.stiffness_damping_geometric = int(bool(getattr(cfg, "stiffness_damping_geometric", False)))
        for name in ("friction_coulomb", "friction_falloff_vel", "friction_viscous", "contact_normal_damping"):
            if hasattr(cfg, name):
                setattr(self.params, name, float(getattr(cfg, name)))
        for name in ("friction_model", "friction_fitted_hessian", "friction_fade", "friction_collider_normal",
                     "contact_explicit_normals", "contact_implicit_normal_force"):
            if hasattr(cfg, name):
                setattr(self.params, name, int(getattr(cfg, name)))
        for k, v in overrides.items():
            if k.startswith("linear_"):
                setattr(self.params.linear, k[len("linear_"):], v)
            else:
                setattr(self.params, k, v)
        capi.check(L.sdx_set_params(self._ctx, C.byref(self.params)))
        sizes = [C.c_int64() for _ in range(4)]
        capi.check(L.sdx_get_sizes(self._ctx, *[C.byref(s) for s in sizes]))
        self.n_tets, self.nnzb, self.n_faces = sizes[1].value, sizes[2].value, sizes[3].value

    def set_linear_solver(self, fn, user=None):
        """Hand every Newton solve of step() to an external solver: fn is the address of a C function of
        type sdx_linear_solve_fn (None: this library's PCG)."""
        capi.check(capi.lib().sdx_set_linear_solver(self._ctx, fn, user))

    def close(self):
        if getattr(self, "_ctx", None):
            capi.lib().sdx_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        self.close()

    def set_params(self, **kw):
        for k, v in kw.items():
            if k.startswith("linear_"):
                setattr(self.params.linear, k[len("linear_"):], v)
            else:
                setattr(self.params, k, v)
        capi.check(capi.lib().sdx_set_params(self._ctx, C.byref(self.params)))

    # state -------------------------------------------------------------------------------------
    def set_state(self, u: Optional[np.ndarray], v: Optional[np.ndarray], time: float = 0.0):
        u = None if u is None else np.ascontiguousarray(u, np.float64).reshape(-1)
        v = None if v is None else np.ascontiguousarray(v, np.float64).reshape(-1)
        capi.check(capi.lib().sdx_set_state(self._ctx, capi.ptr(u), capi.ptr(v), time))

    def get_state(self, u_out: Optional[np.ndarray] = None, v_out: Optional[np.ndarray] = None):
        u = np.empty(3 * self.n_nodes) if u_out is None else u_out
        v = np.empty(3 * self.n_nodes) if v_out is None else v_out
        t = C.c_double()
        capi.check(capi.lib().sdx_get_state(self._ctx, capi.ptr(u), capi.ptr(v), C.byref(t)))
        return u, v, t.value

    def write_state(self, qpos: Optional[np.ndarray] = None, qvel: Optional[np.ndarray] = None,
                    qpos_write_mask: Optional[np.ndarray] = None, qvel_write_mask: Optional[np.ndarray] = None):
        """Masked write of displacement (qpos) and velocity (qvel) DoFs in node order: DoF i is written where
        its mask is nonzero, every DoF when the mask is None (SceneBatchExecutorV2.write_state)."""
        n3 = 3 * self.n_nodes

        def vec(a, dt):
            if a is None:
                return None
            a = np.ascontiguousarray(a, dt).reshape(-1)
            if a.size != n3:
                raise ValueError(f"expected {n3} DoFs, got {a.size}")
            return a
        u, v = vec(qpos, np.float64), vec(qvel, np.float64)
        mu, mv = vec(qpos_write_mask, np.uint8), vec(qvel_write_mask, np.uint8)
        capi.check(capi.lib().sdx_write_state_masked(self._ctx, capi.ptr(u), capi.ptr(v), capi.ptr(mu, capi._up),
                                                     capi.ptr(mv, capi._up)))

    # state snapshots (Scene.capture_state / restore_state / ... of the reference) ---------------------
    def capture_state(self) -> int:
        h = C.c_uint64()
        capi.check(capi.lib().sdx_capture_state(self._ctx, C.byref(h)))
        return h.value

    def restore_state(self, handle: int, release_immediately: bool = False, env_mask: Optional[np.ndarray] = None):
        m = None if env_mask is None else np.ascontiguousarray(env_mask, np.uint8).reshape(-1)
        if m is not None and m.size != self.n_envs:
            raise ValueError(f"env_mask needs {self.n_envs} entries")
        capi.check(capi.lib().sdx_restore_state(self._ctx, int(handle), int(bool(release_immediately)),
                                                capi.ptr(m, capi._up)))

    def release_state(self, handle: int):
        capi.check(capi.lib().sdx_release_state(self._ctx, int(handle)))

    def release_all_states(self):
        capi.check(capi.lib().sdx_release_all_states(self._ctx))

    def is_equal_state(self, a: int, b: int) -> bool:
        eq = C.c_int()
        capi.check(capi.lib().sdx_is_equal_state(self._ctx, int(a), int(b), C.byref(eq)))
        return bool(eq.value)

    def capture_state_to_bytes(self) -> bytes:
        n = C.c_int64()
        capi.check(capi.lib().sdx_capture_state_to_bytes(self._ctx, None, 0, C.byref(n)))
        buf = (C.c_uint8 * n.value)()
        capi.check(capi.lib().sdx_capture_state_to_bytes(self._ctx, buf, n.value, C.byref(n)))
        return bytes(buf)

    def restore_state_from_bytes(self, data: bytes):
        b = (C.c_uint8 * len(data)).from_buffer_copy(data)
        capi.check(capi.lib().sdx_restore_state_from_bytes(self._ctx, b, len(data)))

    # stepping ------------------------------------------------------------------------------------
    def step(self, n: int = 1):
        capi.check(capi.lib().sdx_step(self._ctx, int(n)))

    def stats(self):
        arr = (capi.EnvStats * self.n_envs)()
        capi.check(capi.lib().sdx_get_stats(self._ctx, arr))
        return [dict(newton_iters=s.newton_iters, cg_iters=s.cg_iters, ls_iters=s.ls_iters,
                     convergence=s.convergence, res_norm0=s.res_norm0, res_norm=s.res_norm,
                     n_contacts=s.n_contacts) for s in arr]

    def kernel_launches(self) -> int:
        return int(capi.lib().sdx_kernel_launches(self._ctx))

    # parity ----------------------------------------------------------------------------------------
    def pattern(self):
        rp = np.zeros(self.n_nodes + 1, np.int64)
        col = np.zeros(self.nnzb, np.int32)
        capi.check(capi.lib().sdx_get_pattern(self._ctx, capi.ptr(rp, capi._lp), capi.ptr(col, capi._ip)))
        return rp, col

    def faces(self):
        fn = np.zeros(3 * self.n_faces, np.int32)
        ft = np.zeros(self.n_faces, np.int32)
        fa = np.zeros(self.n_faces)
        capi.check(capi.lib().sdx_get_faces(self._ctx, capi.ptr(fn, capi._ip), capi.ptr(ft, capi._ip),
                                            capi.ptr(fa)))
        return fn, ft, fa

    def assemble(self, u: Optional[np.ndarray] = None, t: float = 0.0, hess: bool = True, psd: bool = True,
                 obj: bool = True):
        flags = capi.SDX_ASM_RES | (capi.SDX_ASM_OBJ if obj else 0) | (capi.SDX_ASM_PSD if psd else 0)
        o = np.zeros(self.n_envs)
        g = np.zeros(3 * self.n_nodes)
        H = np.zeros(9 * self.nnzb, np.float32) if hess else None
        npairs = np.zeros(self.n_envs, np.int64)
        uu = None if u is None else np.ascontiguousarray(u, np.float64).reshape(-1)
        capi.check(capi.lib().sdx_assemble(self._ctx, capi.ptr(uu), t, flags, capi.ptr(o), capi.ptr(g),
                                           capi.ptr(H, capi._fp), capi.ptr(npairs, capi._lp)))
        return {"obj": o, "g": g, "H": None if H is None else H.reshape(-1, 3, 3), "n_pairs": npairs}

    def contact_pairs(self) -> np.ndarray:
        n = C.c_int64()
        capi.check(capi.lib().sdx_get_contact_pairs(self._ctx, None, 0, C.byref(n)))
        out = np.zeros(max(1, n.value), np.int64)
        capi.check(capi.lib().sdx_get_contact_pairs(self._ctx, capi.ptr(out, capi._lp), out.size, C.byref(n)))
        return out[: n.value]

    def stream_handle(self) -> int:
        h = C.c_void_p()
        capi.check(capi.lib().sdx_get_stream(self._ctx, C.byref(h)))
        return int(h.value or 0)

    def pcg_cta_profile(self, n_cta: int) -> np.ndarray:
        """Per-CTA PCG phase times [n_cta, 4] in SM clock cycles since profiling was enabled with cta=True
        (SpMV phase, barrier wait, update phase, barrier wait)."""
        out = np.zeros(4 * int(n_cta))
        capi.check(capi.lib().sdx_get_pcg_cta_profile(self._ctx, int(n_cta), capi.ptr(out)))
        return out.reshape(int(n_cta), 4)

    def set_profiling(self, enable: bool = True, cta: bool = False):
        """Per-kernel event timing; with cta=True also the per-CTA PCG phase timers."""
        capi.check(capi.lib().sdx_set_profiling(self._ctx, (2 if cta else 1) if enable else 0))

    def profile(self) -> dict:
        p = capi.Profile()
        capi.check(capi.lib().sdx_get_profile(self._ctx, C.byref(p)))
        return {f: getattr(p, f) for f, _ in capi.Profile._fields_}

    def bench_spmv(self, reps: int = 20):
        ms, by = C.c_double(), C.c_double()
        capi.check(capi.lib().sdx_bench_spmv(self._ctx, reps, C.byref(ms), C.byref(by)))
        return ms.value, by.value
