"""Generates the golden fixtures of this directory from the reference (run where the reference tree
exists; the fixtures are committed, nothing reads the reference at test time).

  * smith_nh_reference.json — the 5 Smith Neo-Hookean known-answer cases of the reference test suite
    (mochi_core/test/data/material_test_data.h, smith_neo_hookean_test_data, E = 1, nu = 0.4), read
    as text from the header.
  * stvk_reference.json — the 6 St. Venant-Kirchhoff known-answer cases of the same header
    (st_venant_kirchhoff_test_data, E = 1, nu = 0.4).
  * krylov_psd100.json — the reference's 100 x 100 SPD golden system (matrix, rhs, solution) from
    mochi_core/test/data/krylov_solver_test_data.h, read as text.
  * bsr3_reference.json — the reference's BlockSparseMatrix<double,3> storage layout and its krylov::PCG
    on it (oracle/_ref): Values() of matrices filled through the class's own SetValue on seeded block
    patterns, and the iteration counts / solutions of krylov::PCG with BlockJacobiPrec (none, Jacobi,
    block Jacobi) on the 100 x 100 golden system in 3x3 blocks and on an assembled tet-grid Hessian.
  * fp32_mode_reference.json — the reference's FP32 mode (MOCHI_USE_DOUBLE_PRECISION=0, oracle/_ref/
    libsdx_ref_f32.so) against its FP64 mode on the soft cube (cfg0, seed 0) one step from rest: the
    relative error of the assembled elastic Hessian (fem::StressWork per tet, Smith Neo-Hookean,
    projected), and krylov::PCG (Jacobi, rel 1e-6) on that step's first Newton system in float — the
    error budget the GPU path's FP32 matrix / FP64 reductions is held to.
  * reference_vectors.json — outputs of the reference's own compiled code (oracle/_ref, built by
    oracle/build_ref.sh from the reference sources) on seeded inputs: Smith NH with every PSD
    strategy (projected tangents), St. Venant-Kirchhoff and linear elasticity with every PSD strategy,
    fem::StressDampingWork (Rayleigh stiffness damping) on single tets, PolyReLU, the penalty contact response, fem::StressWork on single
    tets, and krylov::PCG iteration counts / solutions on the two golden systems.

  python tests/golden/make_golden.py [--reference-root /path/to/reference]
"""
from __future__ import annotations

import argparse
import dataclasses
import ctypes as C
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

NUM = r"[-+]?(?:\d+\.\d*|\.\d+|\d+)(?:[eE][-+]?\d+)?"


def parse_smith(path):
    text = open(path).read()
    start = text.index("namespace smith_neo_hookean_test_data")
    end = text.index("} // namespace smith_neo_hookean_test_data")
    block = text[start:end]
    cases = []
    for chunk in re.split(r"\bTestData\{", block)[1:]:
        nums = [float(x) for x in re.findall(NUM + r"(?=_r)", chunk)]
        assert len(nums) == 9 + 1 + 9 + 81, len(nums)
        cases.append({"F": nums[0:9], "energy": nums[9], "pk1": nums[10:19], "tangent": nums[19:100]})
    return {"youngs_modulus": 1.0, "poisson_ratio": 0.4, "source": "material_test_data.h smith block",
            "cases": cases}


def parse_stvk(path):
    """The St. Venant-Kirchhoff known-answer cases (st_venant_kirchhoff_test_data, E = 1, nu = 0.4)."""
    text = open(path).read()
    start = text.index("namespace st_venant_kirchhoff_test_data")
    end = text.index("} // namespace st_venant_kirchhoff_test_data")
    block = text[start:end]
    cases = []
    for chunk in re.split(r"\bTestData\{", block)[1:]:
        nums = [float(x) for x in re.findall(NUM + r"(?=_r)", chunk)]
        energy = float(re.search(r"\.strainEnergy\s*=\s*(" + NUM + ")", chunk).group(1))
        assert len(nums) == 9 + 9 + 81, len(nums)
        cases.append({"F": nums[0:9], "energy": energy, "pk1": nums[9:18], "tangent": nums[18:99]})
    return {"youngs_modulus": 1.0, "poisson_ratio": 0.4, "source": "material_test_data.h st_venant_kirchhoff block",
            "cases": cases}


def parse_array(text, name, kind=float):
    m = re.search(name + r"\[\]\s*=\s*\{(.*?)\};", text, re.S)
    vals = re.findall(NUM, m.group(1))
    return [kind(v) for v in vals]


def parse_krylov(path):
    text = open(path).read()
    rows = parse_array(text, "kPsdMatrixRows", int)
    cols = parse_array(text, "kPsdMatrixCols", int)
    vals = parse_array(text, "kPsdMatrixVals")
    rhs = parse_array(text, "kPsdMatrixRhs")
    out = parse_array(text, "kPsdMatrixOut")
    assert len(rows) == len(cols) == len(vals) == 3718 and len(rhs) == len(out) == 100
    return {"n": 100, "rows": rows, "cols": cols, "vals": vals, "rhs": rhs, "solution": out,
            "source": "krylov_solver_test_data.h kPsdMatrix*"}


def tridiag64():
    n = 64
    A = np.diag(np.full(n, 2.0)) - np.diag(np.ones(n - 1), 1) - np.diag(np.ones(n - 1), -1)
    return A, np.ones(n)


def reference_vectors():
    from oracle import oracle as O
    R = O.ref()
    assert R is not None, "oracle/_ref/libsdx_ref.so missing: run oracle/build_ref.sh"
    rng = np.random.default_rng(20261203)
    out = {"smith": [], "polyrelu": [], "penalty": [], "stress_work": [], "pcg": [], "materials": [],
           "stress_damping": [], "collision": [], "arap": [], "reference_stiffness": []}
    for i in range(48):
        F = np.eye(3) + rng.normal(0, 0.35, (3, 3))
        if i % 4 == 0:
            F[:, 0] *= -1.0  # inverted element
        mu, lam = float(rng.uniform(0.2, 3.0)), float(rng.uniform(0.5, 30.0))
        for psd in (0, 1, 2, 3):
            e, P, Cm = O.ref_smith_nh(mu, lam, F, project=psd != 0, psd=psd, oracle_kind=1)
            out["smith"].append({"mu": mu, "lambda": lam, "F": F.reshape(-1).tolist(), "psd": psd,
                                 "energy": e, "pk1": P.reshape(-1).tolist(), "tangent": Cm.reshape(-1).tolist()})
    for x in np.linspace(-0.02, 0.02, 41):
        f, df, ddf = O.polyrelu(float(x), 0.005, 0.004, use_ref=True)
        out["polyrelu"].append({"x": float(x), "t": 0.005, "shift": 0.004, "f": f, "df": df, "ddf": ddf})
    for i in range(40):
        d = float(rng.uniform(-0.012, 0.003))
        g = rng.normal(size=3)
        g /= np.linalg.norm(g)
        k = float(10 ** rng.uniform(3, 9))
        e = np.zeros(1)
        f = np.zeros(3)
        df = np.zeros(6)
        R.ref_penalty(d, O.ptr(g), k, 0.005, 0.001, O.ptr(e), O.ptr(f), O.ptr(df))
        out["penalty"].append({"d": d, "grad": g.tolist(), "k": k, "t_half": 0.005, "thr": 0.001,
                               "energy": float(e[0]), "force": f.tolist(), "dforce6": df.tolist()})
    for i in range(24):
        X = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], float) * 0.01 + rng.normal(0, 0.001, (4, 3))
        D = np.stack([X[k] - X[0] for k in (1, 2, 3)], axis=1)
        if np.linalg.det(D) < 0:
            X[[1, 2]] = X[[2, 1]]
        u = rng.normal(0, 0.003, (4, 3))
        mu, lam = float(rng.uniform(1e3, 1e5)), float(rng.uniform(1e3, 1e6))
        for proj in (0, 1):
            e = np.zeros(1)
            r = np.zeros(12)
            K = np.zeros(144)
            R.ref_stress_work(O.ptr(np.ascontiguousarray(X.reshape(-1))), O.ptr(np.ascontiguousarray(u.reshape(-1))),
                              mu, lam, proj, 1, O.ptr(e), O.ptr(r), O.ptr(K))
            out["stress_work"].append({"X": X.reshape(-1).tolist(), "u": u.reshape(-1).tolist(), "mu": mu,
                                       "lambda": lam, "project": proj, "energy": float(e[0]),
                                       "res": r.tolist(), "K": K.tolist()})
    # krylov::PCG on the golden systems (residual-L2 stop test, Jacobi, Polak-Ribiere)
    kr = parse_krylov(os.path.join(args_ns.mc, "test/data/krylov_solver_test_data.h"))
    A100 = np.zeros((100, 100))
    for r_, c_, v_ in zip(kr["rows"], kr["cols"], kr["vals"]):
        A100[r_, c_] = v_
    systems = {"psd100": (A100, np.array(kr["rhs"])), "tridiag64": tridiag64()}
    for name, (A, b) in systems.items():
        n = A.shape[0]
        rp = np.zeros(n + 1, np.int64)
        cols, vals = [], []
        for i in range(n):
            nz = np.nonzero(A[i])[0]
            cols += nz.tolist()
            vals += A[i, nz].tolist()
            rp[i + 1] = len(cols)
        cols = np.asarray(cols, np.int32)
        vals = np.asarray(vals)
        for rel in (1e-6, 1e-10):
            for jac in (0, 1):
                x = np.zeros(n)
                rn, rr = np.zeros(1), np.zeros(1)
                cv = C.c_int()
                it = R.ref_pcg_csr(n, O.ptr(rp, O._lp), O.ptr(cols, O._ip), O.ptr(vals), O.ptr(b), O.ptr(x),
                                   rel, 1e-30, 1e10, 10000, jac, 1, 1, O.ptr(rn), O.ptr(rr), C.byref(cv))
                out["pcg"].append({"system": name, "rel_tol": rel, "jacobi": jac, "iters": int(it),
                                   "convergence": int(cv.value), "res_norm": float(rn[0]),
                                   "rel_res_norm": float(rr[0]), "x": x.tolist()})
    # St. Venant-Kirchhoff (1) and linear elasticity (2), every PSD strategy, inverted cases included
    rng = np.random.default_rng(7)
    for kind in (1, 2):
        for t in range(12):
            F = np.eye(3) + rng.normal(0.0, 0.35, (3, 3))
            if t % 3 == 0:
                F[:, 0] *= -0.6
            mu, lam = float(rng.uniform(0.2, 2.0)), float(rng.uniform(0.5, 5.0))
            for psd in (0, 1, 2, 3):
                e, P, Cm = O.ref_material(kind, mu, lam, F, project=psd != 0, psd=psd)
                out["materials"].append({"kind": kind, "mu": mu, "lambda": lam, "F": F.reshape(-1).tolist(),
                                         "psd": psd, "energy": e, "pk1": P.reshape(-1).tolist(),
                                         "tangent": Cm.reshape(-1).tolist()})
    # fem::StressDampingWork (Rayleigh stiffness damping) on single tets, with / without the geometric
    # term and its projection
    R = O.ref()
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    rng = np.random.default_rng(11)
    for t in range(16):
        X = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], float) * 0.01 + rng.normal(0, 0.001, (4, 3))
        if np.linalg.det(np.stack([X[1] - X[0], X[2] - X[0], X[3] - X[0]], 1)) < 0:
            X[[1, 2]] = X[[2, 1]]
        u = rng.normal(0, 0.002, 12)
        uss = u + rng.normal(0, 0.001, 12)
        kappa, lam, mu = float(rng.uniform(0.05, 2.0)), float(rng.uniform(1e4, 1e5)), float(rng.uniform(3e3, 3e4))
        geo, proj = t % 2, (t // 2) % 2
        e = np.zeros(1)
        r = np.zeros(12)
        K = np.zeros(144)
        Xf = np.ascontiguousarray(X.reshape(-1))
        R.ref_stress_damping(dp(Xf), dp(u), dp(uss), kappa, lam, mu, geo, proj, dp(e), dp(r), dp(K))
        out["stress_damping"].append({"X": Xf.tolist(), "u": u.tolist(), "uss": uss.tolist(), "kappa": kappa,
                                      "lambda": lam, "mu": mu, "geometric": geo, "project": proj,
                                      "energy": float(e[0]), "res": r.tolist(), "K": K.tolist()})
    # ComputeBatchCollisionForceDForce<1, GradTarget::Current>: penalty + Coulomb / viscous friction + normal
    # damping over random option sets, distances across the threshold and displacements across the
    # Coulomb smoothing width (frictionFalloffVel * dt = 4.2e-5 m at the defaults)
    for i in range(128):
        kw = dict(coulomb=float(rng.choice([0.0, 0.5, 0.9])), viscous=float(rng.choice([0.0, 0.4])),
                  normal_damping=float(rng.choice([0.0, 0.3])), collider_normal=int(rng.integers(2)),
                  explicit_normals=int(rng.integers(2)), fade=int(rng.integers(2)), fitted=int(rng.integers(2)),
                  model=int(rng.integers(2)), max_align=float(rng.choice([0.0, -0.3, 0.5, -1.0])),
                  falloff_vel=float(rng.choice([0.01, 0.1, 0.0])), k=float(10 ** rng.uniform(3, 9)))
        kw["implicit_normal_force"] = 0 if kw["explicit_normals"] else int(rng.integers(2))
        if kw["falloff_vel"] == 0.0 and kw["model"] == 0 and i % 2:
            kw["falloff_vel"] = 0.01
        prm = O.contact_params(**kw)
        g = rng.normal(size=3)
        g /= np.linalg.norm(g)
        gs = g + 0.1 * rng.normal(size=3)
        gs /= np.linalg.norm(gs)
        nc = -g + 0.5 * rng.normal(size=3)
        nc /= np.linalg.norm(nc)
        d, dss = float(rng.uniform(-0.008, 0.002)), float(rng.uniform(-0.008, 0.002))
        pos = rng.normal(size=3) * 0.01
        step = rng.normal(size=3) * float(rng.choice([1e-6, 1e-5, 1e-4, 1e-3]))
        if i % 16 == 0:
            step = g * 1e-4  # along the normal: no tangential displacement
        pss = pos - step
        valid = i % 5 != 0
        dt = 1.0 / 240.0
        e, f, df = O.collision_response(prm, d, g, dss, gs, nc if valid else None, pos, pss, dt, use_ref=True)
        out["collision"].append({"params": kw, "d": d, "grad": g.tolist(), "d_ss": dss, "grad_ss": gs.tolist(),
                                 "n_col": nc.tolist() if valid else None, "pos": pos.tolist(),
                                 "pos_ss": pss.tolist(), "dt": dt, "energy": float(e), "force": f.tolist(),
                                 "dforce": df.reshape(-1).tolist()})
    # BatchedArapConstitutiveResponse (stiffness = mu) with None / Projection / AbsEigenProjection, inverted
    # elements included, and the rest stiffness ComputeReferenceMaterialStiffnessVoigt gives each material
    for i in range(32):
        F = np.eye(3) + rng.normal(0, 0.35, (3, 3))
        if i % 4 == 0:
            F[:, 0] *= -1.0
        mu = float(rng.uniform(0.2, 3.0))
        for psd in (0, 1, 2):
            e, P, Cm = O.ref_material(5, mu, 0.0, F, project=psd != 0, psd=psd)
            out["arap"].append({"mu": mu, "F": F.reshape(-1).tolist(), "psd": psd, "energy": e,
                                "pk1": P.reshape(-1).tolist(), "tangent": Cm.reshape(-1).tolist()})
    for kind in (0, 1, 2, 5):
        c0 = np.zeros(36)
        R.ref_reference_stiffness(kind, 1000.0, 3000.0, O.ptr(c0))
        out["reference_stiffness"].append({"kind": kind, "mu": 1000.0, "lambda": 3000.0, "c0": c0.tolist()})
    out["source"] = "oracle/_ref/libsdx_ref.so (reference sources, FP64 build)"
    return out


def bsr3_vectors():
    """The reference's BSR3 value layout and its PCG on BSR3 matrices (oracle/_ref)."""
    from oracle import oracle as O
    from project_superdex_b200 import scenes
    assert O.ref() is not None, "oracle/_ref/libsdx_ref.so missing: run oracle/build_ref.sh"
    rng = np.random.default_rng(20261204)
    out = {"layout": [], "pcg": []}
    for nbr in (5, 17, 40):
        ptr, idx = [0], []
        for br in range(nbr):
            cols = sorted(set([br] + rng.choice(nbr, size=int(rng.integers(0, 7)), replace=True).tolist()))
            idx += cols
            ptr.append(len(idx))
        blocks = rng.normal(size=(len(idx), 9))
        vals = O.ref_bsr3_values(ptr, idx, blocks)
        out["layout"].append({"row_ptr": ptr, "col": idx, "blocks": blocks.reshape(-1).tolist(),
                              "values": vals.tolist()})
    # the 100 x 100 golden system in 3x3 blocks (padding rows: identity)
    kr = parse_krylov(os.path.join(args_ns.mc, "test/data/krylov_solver_test_data.h"))
    A = np.eye(102)
    for r_, c_, v_ in zip(kr["rows"], kr["cols"], kr["vals"]):
        A[r_, c_] = v_
    b = np.zeros(102)
    b[:100] = kr["rhs"]
    systems = {"psd100": (A, b)}
    # a projected Hessian and gradient of a seeded 4 x 3 x 3 tet grid (the oracle's assembly), FP32-rounded
    body = scenes.grid_body(4, 3, 3, 0.01, rng=np.random.default_rng(5), nu=0.45)
    body.E = np.exp(np.random.default_rng(6).uniform(np.log(1e4), np.log(1e6), size=body.n_tets))
    sc = O.Scene(body, scenes.SceneConfig())
    u = np.random.default_rng(7).normal(0, 5e-4, 3 * body.n_nodes) * (body.pin == 0).repeat(3)
    a = sc.assemble(u, u - 1e-4, psd=True)
    H = a["H"].astype(np.float32).astype(np.float64).reshape(-1, 3, 3)
    Ad = np.zeros((3 * body.n_nodes, 3 * body.n_nodes))
    for i in range(body.n_nodes):
        for k in range(sc.row_ptr[i], sc.row_ptr[i + 1]):
            j = sc.col[k]
            Ad[3 * i:3 * i + 3, 3 * j:3 * j + 3] = H[k]
    systems["tetgrid"] = (Ad, a["g"])
    for name, (Ad, b) in systems.items():
        nb = Ad.shape[0] // 3
        ptr, idx, blocks = [0], [], []
        for i in range(nb):
            for j in range(nb):
                blk = Ad[3 * i:3 * i + 3, 3 * j:3 * j + 3]
                if np.any(blk != 0.0):
                    idx.append(j)
                    blocks.append(blk.reshape(-1))
            ptr.append(len(idx))
        vals = O.ref_bsr3_values(ptr, idx, np.asarray(blocks))
        entry = {"system": name, "row_ptr": ptr, "col": idx, "values": vals.tolist(), "b": b.tolist(), "runs": []}
        for prec in (0, 1, 2):
            x, it, rn, rr, cv = O.ref_bsr3_pcg(ptr, idx, vals, b, rel_tol=1e-6, precond=prec)
            entry["runs"].append({"precond": prec, "rel_tol": 1e-6, "iters": int(it), "convergence": int(cv),
                                  "res_norm": rn, "rel_res_norm": rr, "x": x.tolist()})
        out["pcg"].append(entry)
    out["source"] = "oracle/_ref/libsdx_ref.so (reference BlockSparseMatrix, BlockJacobiPrec, krylov::PCG; FP64)"
    return out


def cfg0_state_after_one_step():
    """The soft cube (cfg0, seed 0) after one backward-Euler step from rest, by the FP64 oracle."""
    from oracle import oracle as O
    from project_superdex_b200 import scenes
    bodies, cfg = scenes.config0()
    b = bodies[0]
    sc = O.Scene(b, cfg, min_eig=float(np.finfo(np.float32).eps))
    p = O.default_newton_params()
    p.abs_tol = 1e-9
    u, v, _ = sc.step(np.zeros(3 * b.n_nodes), np.zeros(3 * b.n_nodes), cfg.dt, p)
    return b, cfg, sc, u, v


def fp32_mode_vectors():
    """The reference's FP32 mode against its FP64 mode on cfg0 (oracle/_ref/libsdx_ref_f32.so)."""
    from oracle import oracle as O
    assert O.ref() is not None and O.ref32() is not None, "run oracle/build_ref.sh (both modes)"
    b, cfg, sc, u, v = cfg0_state_after_one_step()
    X = b.X.reshape(-1, 3)
    lam, mu = b.lame()
    uu = u.reshape(-1, 3)
    free = np.repeat(b.pin == 0, 3)
    # elastic Hessian assembled from the reference's per-tet StressWork, both modes, on the oracle's pattern
    rp, col = sc.row_ptr, sc.col
    slot = {}
    for i in range(b.n_nodes):
        for k in range(rp[i], rp[i + 1]):
            slot[(i, int(col[k]))] = k
    H = {32: np.zeros((col.size, 3, 3)), 64: np.zeros((col.size, 3, 3))}
    for t, tet in enumerate(b.tets):
        X12, u12 = X[tet].reshape(-1), uu[tet].reshape(-1)
        for bits in (32, 64):
            _, _, K = O.ref_stress_work(X12, u12, mu[t], lam[t], project=True, psd=1, fp32=bits == 32)
            for a in range(4):
                for c in range(4):
                    H[bits][slot[(int(tet[a]), int(tet[c]))]] += K[3 * a:3 * a + 3, 3 * c:3 * c + 3]

    def dense_free(Hb):
        A = np.zeros((3 * b.n_nodes, 3 * b.n_nodes))
        for i in range(b.n_nodes):
            for k in range(rp[i], rp[i + 1]):
                j = col[k]
                A[3 * i:3 * i + 3, 3 * j:3 * j + 3] = Hb[k]
        return A[np.ix_(free, free)]
    A32, A64 = dense_free(H[32]), dense_free(H[64])
    # the oracle's own elastic Hessian (dt so large that inertia vanishes) agrees with the FP64 reference
    cfg_big = dataclasses.replace(cfg, dt=1e3)
    sc_big = O.Scene(b, cfg_big, min_eig=float(np.finfo(np.float64).eps))
    Ao = dense_free(sc_big.assemble(u, u, hess=True, psd=True)["H"])
    hess = {"rel_fro_err_fp32_mode": float(np.linalg.norm(A32 - A64) / np.linalg.norm(A64)),
            "max_abs_err_fp32_mode_over_max": float(np.abs(A32 - A64).max() / np.abs(A64).max()),
            "oracle_vs_fp64_mode_rel_fro": float(np.linalg.norm(Ao - A64) / np.linalg.norm(A64)),
            "u_abs_sum": float(np.abs(u).sum())}
    # the first Newton system of the second step (inertia target u + dt v), solved by krylov::PCG
    a = sc.assemble(u, u + cfg.dt * v, t=2 * cfg.dt, hess=True, psd=True)
    srp, scol, sval = O.block_to_scalar_csr(rp, col, a["H"])
    g = a["g"]
    x_exact, it_exact, _ = O.ref_pcg_real(srp, scol, sval, g, rel_tol=1e-13, fp32=False, max_iter=100000)
    x64, it64, c64 = O.ref_pcg_real(srp, scol, sval, g, rel_tol=1e-6, fp32=False)
    x32, it32, c32 = O.ref_pcg_real(srp, scol, sval, g, rel_tol=1e-6, fp32=True)
    nx = np.linalg.norm(x_exact)
    pcg = {"rel_tol": 1e-6, "jacobi": True, "iters_fp64_mode": it64, "iters_fp32_mode": it32,
           "convergence_fp64_mode": c64, "convergence_fp32_mode": c32,
           "rel_err_fp64_mode": float(np.linalg.norm(x64 - x_exact) / nx),
           "rel_err_fp32_mode": float(np.linalg.norm(x32 - x_exact) / nx),
           "iters_exact": it_exact, "g_norm": float(np.linalg.norm(g))}
    return {"config": "cfg0 seed 0, state after one step from rest (FP64 oracle), Smith NH, projection",
            "hessian": hess, "pcg": pcg,
            "source": "oracle/_ref/libsdx_ref_f32.so and libsdx_ref.so (reference sources, both precision modes)"}


def main():
    global args_ns
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference-root", default="/root/reference")
    ap.add_argument("--only-bsr3", action="store_true")
    args_ns = ap.parse_args()
    args_ns.mc = os.path.join(args_ns.reference_root, "superdex_physics/libraries/mochi/mochi_core")
    with open(os.path.join(HERE, "smith_nh_reference.json"), "w") as f:
        json.dump(parse_smith(os.path.join(args_ns.mc, "test/data/material_test_data.h")), f)
    with open(os.path.join(HERE, "stvk_reference.json"), "w") as f:
        json.dump(parse_stvk(os.path.join(args_ns.mc, "test/data/material_test_data.h")), f)
    with open(os.path.join(HERE, "krylov_psd100.json"), "w") as f:
        json.dump(parse_krylov(os.path.join(args_ns.mc, "test/data/krylov_solver_test_data.h")), f)
    with open(os.path.join(HERE, "bsr3_reference.json"), "w") as f:
        json.dump(bsr3_vectors(), f)
    with open(os.path.join(HERE, "fp32_mode_reference.json"), "w") as f:
        json.dump(fp32_mode_vectors(), f, indent=1)
    if "--only-bsr3" in sys.argv:
        return
    with open(os.path.join(HERE, "reference_vectors.json"), "w") as f:
        json.dump(reference_vectors(), f)
    print("wrote fixtures to", HERE)


if __name__ == "__main__":
    main()
