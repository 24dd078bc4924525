"""ctypes binding of libsdx_b200.so (declarations in include/sdx_b200.h).

The CUDA library is the only implementation: there is no CPU fallback. Loading fails loudly when the
shared object is missing or was built for another device.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsdx_b200.so")

SDX_OK = 0
SDX_ASM_OBJ, SDX_ASM_RES, SDX_ASM_HESS, SDX_ASM_PSD = 1, 2, 4, 8
SDX_GUESS_UNKNOWN, SDX_GUESS_ZERO = 0, 1
SDX_F32, SDX_F64 = 0, 1
SDX_PREC_NONE, SDX_PREC_JACOBI, SDX_PREC_BLOCK_JACOBI = 0, 1, 2
SDX_WARM_ZERO, SDX_WARM_PREVIOUS, SDX_WARM_LEARNED, SDX_WARM_TEMPORAL = 0, 1, 2, 3
SDX_LINEAR_CONVERGED, SDX_LINEAR_STOPPED, SDX_LINEAR_DIVERGED = 1, 2, 3
SDX_BSR_ROW_STRIPS, SDX_BSR_BLOCKS = 0, 1
SDX_ERR_INVALID_ARGUMENT, SDX_ERR_DEVICE_TIMEOUT = -1, -4
SDX_MAT_NEO_HOOKEAN, SDX_MAT_ST_VENANT_KIRCHHOFF, SDX_MAT_LINEAR_ELASTIC, SDX_MAT_ARAP = 0, 1, 2, 5

# every entry point include/sdx_b200.h declares
EXPORTED = [
    "sdx_last_error", "sdx_version", "sdx_default_step_params", "sdx_default_linear_params",
    "sdx_pcg_solve", "sdx_pcg_solve_ctx", "sdx_create", "sdx_destroy", "sdx_upload_bodies",
    "sdx_set_colliders", "sdx_set_materials", "sdx_set_params", "sdx_set_state", "sdx_get_state", "sdx_get_sizes",
    "sdx_get_pattern", "sdx_get_faces", "sdx_assemble", "sdx_get_contact_pairs", "sdx_step",
    "sdx_get_stats", "sdx_bench_spmv", "sdx_kernel_launches", "sdx_get_stream",
    "sdx_set_profiling", "sdx_get_profile", "sdx_pcg_solve_device_noalloc", "sdx_mlp_init",
    "sdx_mlp_set_params", "sdx_mlp_get_params", "sdx_mlp_forward", "sdx_mlp_gradients", "sdx_mlp_train",
    "sdx_collect_training", "sdx_get_training_data", "sdx_write_state_masked", "sdx_capture_state",
    "sdx_restore_state", "sdx_release_state", "sdx_release_all_states", "sdx_is_equal_state",
    "sdx_capture_state_to_bytes", "sdx_restore_state_from_bytes", "sdx_get_pcg_cta_profile",
    "sdx_pcg_cluster_shape", "sdx_set_linear_solver",
]
SDX_MLP_PARAMS = 37264
SDX_NOALLOC_MAX_BLOCK_ROWS = 65536


class LinearParams(C.Structure):
    """KrylovSolverParams mirror (mochi_core/include/mochi_core/solvers/krylov_solver.h:43-82)."""

    _fields_ = [("rel_tol", C.c_double), ("abs_tol", C.c_double), ("rel_div_tol", C.c_double),
                ("max_iter", C.c_int), ("preconditioner", C.c_int), ("abort_if_not_spd", C.c_int),
                ("polak_ribiere", C.c_int), ("replace_every", C.c_int), ("value_layout", C.c_int),
                ("refine_inner_rel_tol", C.c_double), ("refine_max_passes", C.c_int)]


class LinearStatus(C.Structure):
    """LinearSolverStatus mirror (krylov_solver.h:85-116)."""

    _fields_ = [("num_iter", C.c_int), ("residual_norm", C.c_double),
                ("relative_residual_norm", C.c_double), ("convergence", C.c_int)]


class StepParams(C.Structure):
    _fields_ = [("dt", C.c_double), ("gravity", C.c_double * 3), ("psd_strategy", C.c_int),
                ("k_contact", C.c_double), ("t_half", C.c_double), ("thr", C.c_double),
                ("max_align", C.c_double), ("newton_max_iter", C.c_int),
                ("newton_rel_tol", C.c_double), ("newton_abs_tol", C.c_double),
                ("newton_rel_step_tol", C.c_double), ("ls_max_iter", C.c_int),
                ("ls_alpha", C.c_double), ("ew_forcing", C.c_int), ("rel_div_tol", C.c_double),
                ("abs_div_tol", C.c_double), ("warm_start", C.c_int), ("linear", LinearParams),
                ("mass_damping", C.c_double), ("stiffness_damping", C.c_double),
                ("stiffness_damping_geometric", C.c_int), ("friction_coulomb", C.c_double),
                ("friction_falloff_vel", C.c_double), ("friction_viscous", C.c_double),
                ("contact_normal_damping", C.c_double), ("friction_model", C.c_int),
                ("friction_fitted_hessian", C.c_int), ("friction_fade", C.c_int),
                ("friction_collider_normal", C.c_int), ("contact_explicit_normals", C.c_int),
                ("contact_implicit_normal_force", C.c_int), ("newton_graph", C.c_int)]


class DeviceSystem(C.Structure):
    """sdx_device_system: one Newton system handed to an external linear solver (user node order)."""

    _fields_ = [("n_envs", C.c_int), ("node_offsets", C.POINTER(C.c_int64)), ("env_mask", C.POINTER(C.c_uint8)),
                ("n_nodes", C.c_int64), ("nnzb", C.c_int64), ("row_ptr", C.c_void_p), ("col", C.c_void_p),
                ("values", C.c_void_p), ("b", C.c_void_p), ("x", C.c_void_p), ("zero_guess", C.c_int),
                ("stream", C.c_void_p)]


LINEAR_SOLVE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(DeviceSystem), C.POINTER(LinearParams),
                              C.POINTER(C.c_int))


class EnvStats(C.Structure):
    _fields_ = [("newton_iters", C.c_int), ("cg_iters", C.c_int), ("ls_iters", C.c_int),
                ("convergence", C.c_int), ("res_norm0", C.c_double), ("res_norm", C.c_double),
                ("n_contacts", C.c_int64)]


class Profile(C.Structure):
    _fields_ = [("pcg_ms", C.c_double), ("pcg_launches", C.c_int64), ("pcg_iters", C.c_int64),
                ("asm_hess_ms", C.c_double), ("asm_hess_launches", C.c_int64),
                ("asm_res_ms", C.c_double), ("asm_res_launches", C.c_int64),
                ("contact_ms", C.c_double), ("contact_launches", C.c_int64),
                ("seed_ms", C.c_double), ("seed_launches", C.c_int64), ("pcg_bytes", C.c_double),
                ("pcg_relaunches", C.c_int64), ("pcg_threads", C.c_int64), ("warm_ms", C.c_double),
                ("warm_launches", C.c_int64), ("pcg_cluster_solves", C.c_int64), ("pcg_cluster_size", C.c_int64),
                ("tune_grid_us", C.c_double), ("tune_cluster_us", C.c_double),
                ("elem_threads", C.c_int64), ("elem_res_threads", C.c_int64), ("elem_aggregated", C.c_int64),
                ("contact_threads", C.c_int64), ("tune_elem_us", C.c_double), ("tune_elem_default_us", C.c_double),
                ("pcg_cluster_ms", C.c_double), ("pcg_cluster_bytes", C.c_double)]


_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int32)
_lp = C.POINTER(C.c_int64)
_up = C.POINTER(C.c_uint8)
_vp = C.c_void_p

_lib = None


class SdxError(RuntimeError):
    pass


def lib():
    """Load libsdx_b200.so (raises when it is missing: there is no fallback path)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: run `python -m project_superdex_b200.build` "
                          "(the soft-body step has no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    L.sdx_last_error.restype = C.c_char_p
    L.sdx_default_step_params.argtypes = [C.POINTER(StepParams)]
    L.sdx_default_linear_params.argtypes = [C.POINTER(LinearParams)]
    L.sdx_pcg_solve.argtypes = [C.c_int, C.c_int64, _lp, _ip, _vp, C.c_int, _dp, _dp, C.c_int,
                                C.POINTER(LinearParams), C.POINTER(LinearStatus)]
    L.sdx_pcg_solve_ctx.argtypes = [_vp, C.c_int, C.c_int64, _lp, _ip, _vp, C.c_int, _dp, _dp,
                                    C.c_int, C.POINTER(LinearParams), C.POINTER(LinearStatus)]
    L.sdx_create.argtypes = [C.c_int]
    L.sdx_create.restype = _vp
    L.sdx_destroy.argtypes = [_vp]
    L.sdx_upload_bodies.argtypes = [_vp, C.c_int, _lp, _lp, _dp, _ip, _dp, _dp, _dp, _up]
    L.sdx_set_colliders.argtypes = [_vp, C.c_int, _ip, _dp]
    L.sdx_set_materials.argtypes = [_vp, C.c_int, _ip]
    L.sdx_set_params.argtypes = [_vp, C.POINTER(StepParams)]
    L.sdx_set_state.argtypes = [_vp, _dp, _dp, C.c_double]
    L.sdx_get_state.argtypes = [_vp, _dp, _dp, _dp]
    L.sdx_write_state_masked.argtypes = [_vp, _dp, _dp, _up, _up]
    L.sdx_get_pcg_cta_profile.argtypes = [_vp, C.c_int, _dp]
    L.sdx_capture_state.argtypes = [_vp, C.POINTER(C.c_uint64)]
    L.sdx_restore_state.argtypes = [_vp, C.c_uint64, C.c_int, _up]
    L.sdx_release_state.argtypes = [_vp, C.c_uint64]
    L.sdx_release_all_states.argtypes = [_vp]
    L.sdx_is_equal_state.argtypes = [_vp, C.c_uint64, C.c_uint64, C.POINTER(C.c_int)]
    L.sdx_capture_state_to_bytes.argtypes = [_vp, C.c_void_p, C.c_int64, _lp]
    L.sdx_restore_state_from_bytes.argtypes = [_vp, C.c_void_p, C.c_int64]
    L.sdx_get_sizes.argtypes = [_vp, _lp, _lp, _lp, _lp]
    L.sdx_get_pattern.argtypes = [_vp, _lp, _ip]
    L.sdx_get_faces.argtypes = [_vp, _ip, _ip, _dp]
    L.sdx_assemble.argtypes = [_vp, _dp, C.c_double, C.c_int, _dp, _dp, _fp, _lp]
    L.sdx_get_contact_pairs.argtypes = [_vp, _lp, C.c_int64, _lp]
    L.sdx_step.argtypes = [_vp, C.c_int]
    L.sdx_get_stats.argtypes = [_vp, C.POINTER(EnvStats)]
    L.sdx_bench_spmv.argtypes = [_vp, C.c_int, _dp, _dp]
    L.sdx_kernel_launches.argtypes = [_vp]
    L.sdx_kernel_launches.restype = C.c_int64
    L.sdx_get_stream.argtypes = [_vp, C.POINTER(C.c_void_p)]
    L.sdx_set_profiling.argtypes = [_vp, C.c_int]
    L.sdx_get_profile.argtypes = [_vp, C.POINTER(Profile)]
    L.sdx_pcg_cluster_shape.argtypes = [C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.sdx_set_linear_solver.argtypes = [_vp, _vp, _vp]
    _fp_ = C.POINTER(C.c_float)
    L.sdx_mlp_init.argtypes = [_vp, C.c_uint64]
    L.sdx_mlp_set_params.argtypes = [_vp, _fp_, C.c_int]
    L.sdx_mlp_get_params.argtypes = [_vp, _fp_, C.c_int]
    L.sdx_mlp_forward.argtypes = [_vp, _fp_, C.c_int, _fp_]
    L.sdx_mlp_gradients.argtypes = [_vp, _fp_, _fp_, C.c_int, _fp_, _dp]
    L.sdx_mlp_train.argtypes = [_vp, _fp_, _fp_, C.c_int64, C.c_int, C.c_int, C.c_float, C.c_uint64, _dp]
    L.sdx_collect_training.argtypes = [_vp, C.c_int, C.c_int64, C.c_uint64]
    L.sdx_get_training_data.argtypes = [_vp, _fp_, _fp_, C.c_int64, _lp]
    L.sdx_pcg_solve_device_noalloc.argtypes = [C.c_int, C.c_int64, _vp, _vp, _vp, _vp, _vp, C.c_int,
                                               C.POINTER(LinearParams), C.POINTER(LinearStatus), _vp]
    _lib = L
    return L


def check(rc: int):
    if rc != SDX_OK:
        raise SdxError(f"sdx error {rc}: {lib().sdx_last_error().decode()}")


def ptr(a, t=_dp):
    return None if a is None else a.ctypes.data_as(t)


def default_step_params() -> StepParams:
    p = StepParams()
    lib().sdx_default_step_params(C.byref(p))
    return p


def default_linear_params() -> LinearParams:
    p = LinearParams()
    lib().sdx_default_linear_params(C.byref(p))
    return p


def pcg_cluster_shape_sized(n_envs: int, cluster_size: int):
    """(clusters, CTAs per cluster) of the cluster PCG on the current device with cluster_size forced (the
    shape the autotuner would time), (0, 0) when that size does not fit on the device."""
    import os
    old = os.environ.get("SDX_PCG_CLUSTER_SIZE")
    os.environ["SDX_PCG_CLUSTER_SIZE"] = str(int(cluster_size))
    try:
        return pcg_cluster_shape(n_envs)
    except SdxError:
        return 0, 0
    finally:
        if old is None:
            del os.environ["SDX_PCG_CLUSTER_SIZE"]
        else:
            os.environ["SDX_PCG_CLUSTER_SIZE"] = old


def pcg_cluster_shape(n_envs: int):
    """(clusters, CTAs per cluster) the cluster PCG uses for a queue of n_envs envs on the current device;
    raises SdxError when no cluster shape fits."""
    n, size = C.c_int(), C.c_int()
    check(lib().sdx_pcg_cluster_shape(int(n_envs), C.byref(n), C.byref(size)))
    return n.value, size.value
