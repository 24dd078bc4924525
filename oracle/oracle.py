"""ctypes wrapper of the CPU oracle (oracle/liboracle.so) and of the reference shim
(oracle/_ref/libsdx_ref.so). Test infrastructure only: imported by tests/, by
__graft_entry__.smoke() and by bench.py's cpu_baseline leg, never by the product package.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libsdx_ref.so")
REF32_PATH = os.path.join(HERE, "_ref", "libsdx_ref_f32.so")

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
_lp = C.POINTER(C.c_int64)
_up = C.POINTER(C.c_uint8)


def build():
    """Compile the C restatement (and, where the reference tree is present, oracle/_ref)."""
    subprocess.check_call(["make", "-s", "-C", HERE, "all"])
    subprocess.check_call(["make", "-s", "-C", HERE, "ref"], stdout=subprocess.DEVNULL)


class OrCollider(C.Structure):
    _fields_ = [("type", C.c_int), ("p", C.c_double * 6), ("radius", C.c_double),
                ("vel", C.c_double * 3)]


class OrScene(C.Structure):
    _fields_ = [
        ("n_nodes", C.c_int), ("n_tets", C.c_int), ("n_faces", C.c_int),
        ("X", _dp), ("tets", _ip), ("mu", _dp), ("lam", _dp), ("rho", _dp), ("pin", _up),
        ("face_nodes", _ip), ("face_tet", _ip), ("face_area", _dp),
        ("dN", _dp), ("vol", _dp), ("row_ptr", _lp), ("col", _ip), ("nnzb", C.c_int64),
        ("mass", _dp),
        ("gravity", C.c_double * 3), ("dt", C.c_double), ("psd_strategy", C.c_int),
        ("min_eig", C.c_double),
        ("n_colliders", C.c_int), ("colliders", C.POINTER(OrCollider)),
        ("k_contact", C.c_double), ("t_half", C.c_double), ("thr", C.c_double),
        ("max_align", C.c_double), ("material", C.c_int), ("mass_damping", C.c_double),
        ("u_stage", _dp), ("stiffness_damping", C.c_double), ("stiffness_damping_geometric", C.c_int),
        ("coulomb", C.c_double), ("falloff_vel", C.c_double), ("viscous", C.c_double),
        ("normal_damping", C.c_double), ("collider_normal", C.c_int), ("explicit_normals", C.c_int),
        ("fade", C.c_int), ("implicit_normal_force", C.c_int), ("fitted", C.c_int), ("friction_model", C.c_int),
    ]


class OrContactParams(C.Structure):
    _fields_ = [("k", C.c_double), ("t_half", C.c_double), ("thr", C.c_double), ("max_align", C.c_double),
                ("coulomb", C.c_double), ("falloff_vel", C.c_double), ("viscous", C.c_double),
                ("normal_damping", C.c_double), ("collider_normal", C.c_int), ("explicit_normals", C.c_int),
                ("fade", C.c_int), ("implicit_normal_force", C.c_int), ("fitted", C.c_int), ("model", C.c_int)]


CONTACT_DEFAULTS = dict(k=1e4, t_half=5e-3, thr=1e-3, max_align=0.0, coulomb=0.5, falloff_vel=0.01, viscous=0.0,
                        normal_damping=0.0, collider_normal=1, explicit_normals=0, fade=1, implicit_normal_force=0,
                        fitted=1, model=0)


def contact_params(**kw):
    """OrContactParams from the reference's defaults (ContactParams, ContactEvalConfig) overridden by kw."""
    v = dict(CONTACT_DEFAULTS)
    for k_, x in kw.items():
        if k_ not in v:
            raise KeyError(k_)
        v[k_] = x
    return OrContactParams(**v)


class OrPcgParams(C.Structure):
    _fields_ = [("rel_tol", C.c_double), ("abs_tol", C.c_double), ("rel_div_tol", C.c_double),
                ("max_iter", C.c_int), ("precond", C.c_int), ("polak_ribiere", C.c_int),
                ("zero_guess", C.c_int)]


class OrPcgStatus(C.Structure):
    _fields_ = [("num_iter", C.c_int), ("res_norm", C.c_double), ("rel_res_norm", C.c_double),
                ("convergence", C.c_int)]


class OrNewtonParams(C.Structure):
    _fields_ = [("max_iter", C.c_int), ("rel_tol", C.c_double), ("abs_tol", C.c_double),
                ("rel_step_tol", C.c_double), ("ls_max_iter", C.c_int), ("ls_alpha", C.c_double),
                ("ew_forcing", C.c_int), ("rel_div_tol", C.c_double), ("abs_div_tol", C.c_double),
                ("lin", OrPcgParams)]


class OrNewtonStatus(C.Structure):
    _fields_ = [("newton_iters", C.c_int), ("cg_iters", C.c_int), ("ls_iters", C.c_int),
                ("res_norm0", C.c_double), ("res_norm", C.c_double), ("convergence", C.c_int),
                ("n_contacts", C.c_int64)]


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.or_smith_nh.argtypes = [C.c_double, C.c_double, _dp, C.c_int, C.c_int, C.c_double, _dp, _dp, _dp]
        L.or_material.argtypes = [C.c_int, C.c_double, C.c_double, _dp, C.c_int, C.c_int, C.c_double, _dp, _dp,
                                  _dp]
        L.or_stress_damping.argtypes = [_dp, C.c_double, _dp, _dp, C.c_double, C.c_double, C.c_double, C.c_int,
                                        C.c_int, _dp, _dp, _dp]
        L.or_polyrelu.argtypes = [C.c_double] * 3 + [_dp] * 3
        L.or_penalty.argtypes = [C.c_double, _dp, C.c_double, C.c_double, C.c_double, _dp, _dp, _dp]
        L.or_collision_response.argtypes = [C.POINTER(OrContactParams), C.c_double, _dp, C.c_double, _dp, _dp, _dp,
                                            _dp, C.c_double, C.c_int, _dp, _dp, _dp]
        L.or_pattern_nnzb.argtypes = [C.c_int, C.c_int, _ip]
        L.or_pattern_nnzb.restype = C.c_int64
        L.or_pattern_fill.argtypes = [C.c_int, C.c_int, _ip, _lp, _ip]
        L.or_rest_data.argtypes = [C.c_int, _ip, _dp, _dp, _dp]
        L.or_boundary_faces.argtypes = [C.c_int, C.c_int, _ip, _dp, _ip, _ip, _dp]
        L.or_boundary_faces.restype = C.c_int
        L.or_mass_blocks.argtypes = [C.POINTER(OrScene), _dp]
        L.or_assemble.argtypes = [C.POINTER(OrScene), _dp, _dp, C.c_double, C.c_int, _dp, _dp, _dp, _lp]
        L.or_assemble.restype = C.c_int64
        L.or_pcg.argtypes = [C.c_int, _lp, _ip, _dp, _dp, _dp, C.POINTER(OrPcgParams)]
        L.or_pcg.restype = OrPcgStatus
        L.or_bsr_apply.argtypes = [C.c_int, _lp, _ip, _dp, _dp, _dp]
        L.or_stop_status.argtypes = [C.c_double] * 5
        L.or_stop_status.restype = C.c_int
        L.or_step.argtypes = [C.POINTER(OrScene), _dp, _dp, C.c_double, C.POINTER(OrNewtonParams), _dp]
        L.or_step.restype = OrNewtonStatus
        L.or_default_newton_params.argtypes = [C.POINTER(OrNewtonParams)]
        L.or_num_threads.restype = C.c_int
        L.or_set_num_threads.argtypes = [C.c_int]
        _lib = L
    return _lib


def ref():
    """The reference's own code (FP64), or None when oracle/_ref was not built."""
    global _ref
    if _ref is None and os.path.exists(REF_PATH):
        R = C.CDLL(REF_PATH)
        R.ref_smith_nh.argtypes = [C.c_double, C.c_double, _dp, C.c_int, C.c_int, C.c_int, _dp, _dp, _dp]
        R.ref_material.argtypes = [C.c_int, C.c_double, C.c_double, _dp, C.c_int, C.c_int, _dp, _dp, _dp]
        R.ref_stress_damping.argtypes = [_dp, _dp, _dp, C.c_double, C.c_double, C.c_double, C.c_int, C.c_int, _dp,
                                         _dp, _dp]
        R.ref_reference_stiffness.argtypes = [C.c_int, C.c_double, C.c_double, _dp]
        R.ref_polyrelu.argtypes = [C.c_double] * 3 + [_dp] * 3
        R.ref_penalty.argtypes = [C.c_double, _dp, C.c_double, C.c_double, C.c_double, _dp, _dp, _dp]
        R.ref_collision_response.argtypes = ([C.c_double, _dp, C.c_double, _dp, _dp, _dp, _dp] + [C.c_double] * 8 +
                                             [C.c_int] * 7 + [C.c_double, C.c_int, _dp, _dp, _dp])
        R.ref_stress_work.argtypes = [_dp, _dp, C.c_double, C.c_double, C.c_int, C.c_int, _dp, _dp, _dp]
        R.ref_pcg_csr.argtypes = [C.c_int, _lp, _ip, _dp, _dp, _dp, C.c_double, C.c_double, C.c_double,
                                  C.c_int, C.c_int, C.c_int, C.c_int, _dp, _dp, C.POINTER(C.c_int)]
        R.ref_pcg_csr.restype = C.c_int
        R.ref_pcg_csr_real.argtypes = R.ref_pcg_csr.argtypes
        R.ref_pcg_csr_real.restype = C.c_int
        R.ref_stress_work.restype = None
        R.ref_bsr3_values.argtypes = [C.c_int, _ip, _ip, _dp, _dp]
        R.ref_bsr3_pcg.argtypes = [C.c_int, _ip, _ip, _dp, _dp, _dp, C.c_double, C.c_double, C.c_double, C.c_int,
                                   C.c_int, C.c_int, C.c_int, _dp, _dp, C.POINTER(C.c_int)]
        R.ref_bsr3_pcg.restype = C.c_int
        _ref = R
    return _ref


def ptr(a, t=_dp):
    return a.ctypes.data_as(t)


# --------------------------------------------------------------------------------------------
# constitutive / contact


def smith_nh(mu, lam, F, project=False, psd=1, min_eig=np.finfo(np.float64).eps):
    F = np.ascontiguousarray(F, np.float64).reshape(9)
    e = np.zeros(1)
    P = np.zeros(9)
    Cm = np.zeros(81)
    lib().or_smith_nh(mu, lam, ptr(F), int(project), psd, min_eig, ptr(e), ptr(P), ptr(Cm))
    return e[0], P.reshape(3, 3), Cm.reshape(9, 9)


def material(kind, mu, lam, F, project=False, psd=1, min_eig=np.finfo(np.float64).eps):
    """or_material: kind 0 Smith Neo-Hookean, 1 St. Venant-Kirchhoff, 2 linear elastic, 5 ARAP (stiffness mu)."""
    F = np.ascontiguousarray(F, np.float64).reshape(9)
    e = np.zeros(1)
    P = np.zeros(9)
    Cm = np.zeros(81)
    lib().or_material(int(kind), mu, lam, ptr(F), int(project), psd, min_eig, ptr(e), ptr(P), ptr(Cm))
    return e[0], P.reshape(3, 3), Cm.reshape(9, 9)


_ref32 = None


def ref32():
    """The reference's own code in its FP32 mode (MOCHI_USE_DOUBLE_PRECISION=0), or None when not built."""
    global _ref32
    if _ref32 is None and os.path.exists(REF32_PATH):
        R = C.CDLL(REF32_PATH)
        R.ref_stress_work.argtypes = [_dp, _dp, C.c_double, C.c_double, C.c_int, C.c_int, _dp, _dp, _dp]
        R.ref_pcg_csr_real.argtypes = [C.c_int, _lp, _ip, _dp, _dp, _dp, C.c_double, C.c_double, C.c_double,
                                       C.c_int, C.c_int, C.c_int, C.c_int, _dp, _dp, C.POINTER(C.c_int)]
        R.ref_pcg_csr_real.restype = C.c_int
        R.ref_real_size.restype = C.c_int
        assert R.ref_real_size() == 4, "libsdx_ref_f32.so is not an FP32-mode build"
        _ref32 = R
    return _ref32


def ref_stress_work(X12, u12, mu, lam, project=True, psd=1, fp32=False):
    """fem::StressWork of one Smith Neo-Hookean tet by the reference's compiled code, in its FP64 mode or
    (fp32=True) its FP32 mode. Returns (energy, residual 12, K 12x12)."""
    R = ref32() if fp32 else ref()
    X = np.ascontiguousarray(X12, np.float64).reshape(-1)
    u = np.ascontiguousarray(u12, np.float64).reshape(-1)
    e, r, K = np.zeros(1), np.zeros(12), np.zeros(144)
    R.ref_stress_work(ptr(X), ptr(u), float(mu), float(lam), int(project), int(psd), ptr(e), ptr(r), ptr(K))
    return float(e[0]), r, K.reshape(12, 12)


def ref_pcg_real(row_ptr, col, val, b, rel_tol=1e-6, jacobi=True, fp32=True, max_iter=10000):
    """krylov::PCG on a scalar CSR matrix in the reference build's own precision (FP32 mode: values, vectors,
    dots and the stop test in float). Returns (x, iters, convergence)."""
    R = ref32() if fp32 else ref()
    rp = np.ascontiguousarray(row_ptr, np.int64)
    cl = np.ascontiguousarray(col, np.int32)
    v = np.ascontiguousarray(val, np.float64)
    b = np.ascontiguousarray(b, np.float64)
    x = np.zeros_like(b)
    rn, rr, cv = C.c_double(), C.c_double(), C.c_int()
    it = R.ref_pcg_csr_real(b.size, ptr(rp, _lp), ptr(cl, _ip), ptr(v), ptr(b), ptr(x), rel_tol, 0.0, 1e10,
                            max_iter, int(jacobi), 1, 1, C.byref(rn), C.byref(rr), C.byref(cv))
    return x, int(it), int(cv.value)


def block_to_scalar_csr(row_ptr, col, blocks):
    """3x3 block CSR -> scalar CSR (row_ptr, col, values) with every stored block entry kept."""
    row_ptr = np.asarray(row_ptr, np.int64)
    col = np.asarray(col, np.int64)
    blocks = np.asarray(blocks).reshape(-1, 3, 3)
    n = row_ptr.size - 1
    nb = np.diff(row_ptr)
    srp = np.zeros(3 * n + 1, np.int64)
    srp[1:] = np.repeat(3 * nb, 3).cumsum()
    scol = np.empty(9 * col.size, np.int32)
    sval = np.empty(9 * col.size)
    for i in range(n):
        b0, b1 = row_ptr[i], row_ptr[i + 1]
        for lr in range(3):
            o = srp[3 * i + lr]
            cc = (3 * col[b0:b1, None] + np.arange(3)[None, :]).reshape(-1)
            scol[o:o + cc.size] = cc
            sval[o:o + cc.size] = blocks[b0:b1, lr, :].reshape(-1)
    return srp, scol, sval


def ref_bsr3_values(row_ptr, col, blocks):
    """Values() of the reference's BlockSparseMatrix<double,3> filled entry by entry through its own
    SetValue: the values in the reference's storage layout (row strips)."""
    rp = np.ascontiguousarray(row_ptr, np.int32)
    cl = np.ascontiguousarray(col, np.int32)
    bl = np.ascontiguousarray(np.asarray(blocks, np.float64).reshape(-1, 9))
    out = np.zeros(bl.size)
    ref().ref_bsr3_values(rp.size - 1, rp.ctypes.data_as(_ip), cl.ctypes.data_as(_ip), bl.ctypes.data_as(_dp),
                          out.ctypes.data_as(_dp))
    return out


def ref_bsr3_pcg(row_ptr, col, values, b, x0=None, rel_tol=1e-6, abs_tol=1e-30, rel_div_tol=1e10, max_iter=10000,
                 precond=1, polak_ribiere=True):
    """The reference's krylov::PCG on its BlockSparseMatrix<double,3> holding `values` (row-strip layout),
    with its BlockJacobiPrec (precond 1 Jacobi, 2 block Jacobi, 0 none). Returns (x, iters, |r|, |r|/|b|,
    convergence)."""
    rp = np.ascontiguousarray(row_ptr, np.int32)
    cl = np.ascontiguousarray(col, np.int32)
    v = np.ascontiguousarray(values, np.float64)
    b = np.ascontiguousarray(b, np.float64)
    x = np.zeros_like(b) if x0 is None else np.array(x0, np.float64)
    res, rel, conv = C.c_double(), C.c_double(), C.c_int()
    it = ref().ref_bsr3_pcg(rp.size - 1, rp.ctypes.data_as(_ip), cl.ctypes.data_as(_ip), v.ctypes.data_as(_dp),
                            b.ctypes.data_as(_dp), x.ctypes.data_as(_dp), rel_tol, abs_tol, rel_div_tol, max_iter,
                            precond, int(polak_ribiere), int(x0 is None), C.byref(res), C.byref(rel), C.byref(conv))
    return x, it, res.value, rel.value, conv.value


def ref_material(kind, mu, lam, F, project=False, psd=1):
    """The reference's own StVK (kind 1) / linear-elastic (kind 2) / ARAP (kind 5) response."""
    F = np.ascontiguousarray(F, np.float64).reshape(9)
    e = np.zeros(1)
    P = np.zeros(9)
    Cm = np.zeros(81)
    ref().ref_material(int(kind), mu, lam, ptr(F), int(project), psd, ptr(e), ptr(P), ptr(Cm))
    return e[0], P.reshape(3, 3), Cm.reshape(9, 9)


def ref_smith_nh(mu, lam, F, project=False, psd=1, oracle_kind=1):
    F = np.ascontiguousarray(F, np.float64).reshape(9)
    e = np.zeros(1)
    P = np.zeros(9)
    Cm = np.zeros(81)
    ref().ref_smith_nh(mu, lam, ptr(F), int(project), psd, oracle_kind, ptr(e), ptr(P), ptr(Cm))
    return e[0], P.reshape(3, 3), Cm.reshape(9, 9)


def penalty(d, grad, k, t_half, thr):
    g = np.ascontiguousarray(grad, np.float64)
    e = np.zeros(1)
    f = np.zeros(3)
    df = np.zeros(9)
    lib().or_penalty(d, ptr(g), k, t_half, thr, ptr(e), ptr(f), ptr(df))
    return e[0], f, df.reshape(3, 3)


def collision_response(prm, d, grad, d_ss, grad_ss, n_col, pos, pos_ss, dt, unit_grad=True, use_ref=False):
    """Energy, force (3) and dforce (3x3) of one contact sample (or_collision_response; with use_ref the
    reference's own ComputeBatchCollisionForceDForce). n_col None: colliding normals not valid."""
    a = [np.ascontiguousarray(v, np.float64) for v in (grad, grad_ss, n_col if n_col is not None else np.zeros(3),
                                                       pos, pos_ss)]
    e = np.zeros(1)
    f = np.zeros(3)
    df = np.zeros(9)
    if use_ref:
        ref().ref_collision_response(d, ptr(a[0]), d_ss, ptr(a[1]), ptr(a[2]), ptr(a[3]), ptr(a[4]), prm.k,
                                     prm.t_half, prm.thr, prm.max_align, prm.coulomb, prm.falloff_vel, prm.viscous,
                                     prm.normal_damping, prm.collider_normal, int(n_col is not None),
                                     prm.explicit_normals, prm.fade, prm.implicit_normal_force, prm.fitted,
                                     prm.model, dt, int(unit_grad), ptr(e), ptr(f), ptr(df))
    else:
        lib().or_collision_response(C.byref(prm), d, ptr(a[0]), d_ss, ptr(a[1]),
                                    ptr(a[2]) if n_col is not None else None, ptr(a[3]), ptr(a[4]), dt,
                                    int(unit_grad), ptr(e), ptr(f), ptr(df))
    return e[0], f, df.reshape(3, 3)


def polyrelu(x, t, shift, use_ref=False):
    f, df, ddf = C.c_double(), C.c_double(), C.c_double()
    fn = ref().ref_polyrelu if use_ref else lib().or_polyrelu
    fn(x, t, shift, C.byref(f), C.byref(df), C.byref(ddf))
    return f.value, df.value, ddf.value


# --------------------------------------------------------------------------------------------
# scenes


class Scene:
    """Oracle-side scene for ONE body: owns every array the C struct points to."""

    def __init__(self, body, cfg, psd_strategy=1, min_eig=None):
        L = lib()
        self.body = body
        self.cfg = cfg
        N, T = body.n_nodes, body.n_tets
        self.X = np.ascontiguousarray(body.X, np.float64).reshape(-1)
        self.tets = np.ascontiguousarray(body.tets, np.int32).reshape(-1)
        lam, mu = body.lame()
        self.lam = np.ascontiguousarray(lam, np.float64)
        self.mu = np.ascontiguousarray(mu, np.float64)
        self.rho = np.ascontiguousarray(body.rho, np.float64)
        self.pin = np.ascontiguousarray(body.pin, np.uint8)
        nf = L.or_boundary_faces(N, T, ptr(self.tets, _ip), ptr(self.X), None, None, None)
        self.face_nodes = np.zeros(3 * nf, np.int32)
        self.face_tet = np.zeros(nf, np.int32)
        self.face_area = np.zeros(nf)
        L.or_boundary_faces(N, T, ptr(self.tets, _ip), ptr(self.X), ptr(self.face_nodes, _ip),
                            ptr(self.face_tet, _ip), ptr(self.face_area))
        self.dN = np.zeros(12 * T)
        self.vol = np.zeros(T)
        L.or_rest_data(T, ptr(self.tets, _ip), ptr(self.X), ptr(self.dN), ptr(self.vol))
        nnzb = L.or_pattern_nnzb(N, T, ptr(self.tets, _ip))
        self.row_ptr = np.zeros(N + 1, np.int64)
        self.col = np.zeros(nnzb, np.int32)
        L.or_pattern_fill(N, T, ptr(self.tets, _ip), ptr(self.row_ptr, _lp), ptr(self.col, _ip))
        self.mass = np.zeros(nnzb)
        self.colliders = (OrCollider * max(1, len(body.colliders)))()
        for i, c in enumerate(body.colliders):
            self.colliders[i].type = c.type
            for k in range(6):
                self.colliders[i].p[k] = float(c.p[k])
            self.colliders[i].radius = float(c.radius)
            for k in range(3):
                self.colliders[i].vel[k] = float(c.vel[k])
        s = OrScene()
        s.n_nodes, s.n_tets, s.n_faces = N, T, nf
        s.X, s.tets, s.mu, s.lam, s.rho, s.pin = (ptr(self.X), ptr(self.tets, _ip), ptr(self.mu),
                                                  ptr(self.lam), ptr(self.rho), ptr(self.pin, _up))
        s.face_nodes, s.face_tet, s.face_area = (ptr(self.face_nodes, _ip), ptr(self.face_tet, _ip),
                                                 ptr(self.face_area))
        s.dN, s.vol = ptr(self.dN), ptr(self.vol)
        s.row_ptr, s.col, s.nnzb = ptr(self.row_ptr, _lp), ptr(self.col, _ip), nnzb
        s.mass = ptr(self.mass)
        s.material = int(getattr(body, "material", 0))
        s.mass_damping = float(getattr(cfg, "mass_damping", 0.0))
        s.stiffness_damping = float(getattr(cfg, "stiffness_damping", 0.0))
        s.stiffness_damping_geometric = int(bool(getattr(cfg, "stiffness_damping_geometric", False)))
        for k in range(3):
            s.gravity[k] = cfg.gravity[k]
        s.dt = cfg.dt
        s.psd_strategy = psd_strategy
        s.min_eig = np.finfo(np.float64).eps if min_eig is None else min_eig
        s.n_colliders = len(body.colliders)
        s.colliders = C.cast(self.colliders, C.POINTER(OrCollider))
        s.k_contact, s.t_half, s.thr, s.max_align = cfg.k_contact, cfg.t_half, cfg.thr, cfg.max_align
        s.coulomb = float(getattr(cfg, "friction_coulomb", 0.0))
        s.falloff_vel = float(getattr(cfg, "friction_falloff_vel", 0.01))
        s.viscous = float(getattr(cfg, "friction_viscous", 0.0))
        s.normal_damping = float(getattr(cfg, "contact_normal_damping", 0.0))
        s.collider_normal = int(bool(getattr(cfg, "friction_collider_normal", True)))
        s.explicit_normals = int(bool(getattr(cfg, "contact_explicit_normals", False)))
        s.fade = int(bool(getattr(cfg, "friction_fade", True)))
        s.implicit_normal_force = int(bool(getattr(cfg, "contact_implicit_normal_force", False)))
        s.fitted = int(bool(getattr(cfg, "friction_fitted_hessian", True)))
        s.friction_model = int(getattr(cfg, "friction_model", 0))
        self.s = s
        L.or_mass_blocks(C.byref(s), ptr(self.mass))
        self.nnzb = nnzb
        self.n_faces = nf

    def assemble(self, u, ut, t=0.0, obj=True, res=True, hess=True, psd=True, pairs=False, u_stage=None):
        N = self.body.n_nodes
        u = np.ascontiguousarray(u, np.float64).reshape(-1)
        ut = np.ascontiguousarray(ut, np.float64).reshape(-1)
        us = None if u_stage is None else np.ascontiguousarray(u_stage, np.float64).reshape(-1)
        self.s.u_stage = ptr(us) if us is not None else None
        flags = (1 if obj else 0) | (2 if res else 0) | (4 if hess else 0) | (8 if psd else 0)
        o = np.zeros(1)
        g = np.zeros(3 * N)
        H = np.zeros(9 * self.nnzb)
        cap = 3 * self.n_faces * max(1, len(self.body.colliders))
        pr = np.zeros(max(1, cap), np.int64) if pairs else None
        n = lib().or_assemble(C.byref(self.s), ptr(u), ptr(ut), t, flags, ptr(o), ptr(g), ptr(H),
                              ptr(pr, _lp) if pairs else None)
        out = {"obj": o[0], "g": g, "H": H.reshape(-1, 3, 3), "n_pairs": n}
        if pairs:
            out["pairs"] = pr[:n].copy()
        return out

    def step(self, u, v, t, params=None, warm=None):
        if params is None:
            params = default_newton_params()
        u = np.ascontiguousarray(u, np.float64).reshape(-1)
        v = np.ascontiguousarray(v, np.float64).reshape(-1)
        w = None if warm is None else np.ascontiguousarray(warm, np.float64).reshape(-1)
        st = lib().or_step(C.byref(self.s), ptr(u), ptr(v), t, C.byref(params),
                           ptr(w) if w is not None else None)
        return u, v, st


def default_newton_params():
    p = OrNewtonParams()
    lib().or_default_newton_params(C.byref(p))
    return p


def pcg(row_ptr, col, H, b, x=None, rel_tol=1e-6, abs_tol=1e-9, rel_div_tol=1e10, max_iter=10000,
        precond=1, polak_ribiere=1):
    n = row_ptr.size - 1
    b = np.ascontiguousarray(b, np.float64).reshape(-1)
    zero = x is None
    x = np.zeros(3 * n) if zero else np.ascontiguousarray(x, np.float64).reshape(-1).copy()
    p = OrPcgParams(rel_tol, abs_tol, rel_div_tol, max_iter, precond, polak_ribiere, int(zero))
    Hc = np.ascontiguousarray(H, np.float64).reshape(-1)
    st = lib().or_pcg(n, ptr(np.ascontiguousarray(row_ptr, np.int64), _lp),
                      ptr(np.ascontiguousarray(col, np.int32), _ip), ptr(Hc), ptr(b), ptr(x),
                      C.byref(p))
    return x, st


def stop_status(rr, bb, rel_tol, abs_tol, rel_div_tol):
    """or_stop_status: 0 active, 1 converged (relative), 2 converged (absolute), 3 diverged."""
    return int(lib().or_stop_status(float(rr), float(bb), float(rel_tol), float(abs_tol), float(rel_div_tol)))


def bsr_to_dense(row_ptr, col, H):
    n = row_ptr.size - 1
    A = np.zeros((3 * n, 3 * n))
    Hb = np.asarray(H).reshape(-1, 3, 3)
    for i in range(n):
        for b in range(row_ptr[i], row_ptr[i + 1]):
            j = col[b]
            A[3 * i:3 * i + 3, 3 * j:3 * j + 3] = Hb[b]
    return A
