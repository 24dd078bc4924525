"""Parity on the configurations the benchmark reports, against the FP64 CPU oracle (oracle/sdx_oracle.c,
the reference's path restated and pinned to the reference's compiled code): the soft cube over its full
100-step run, and the first envs of the 1,024-body batch as one batch. Tolerance: vertex position within
1e-5 of the body size; Newton iteration counts equal (up to a rounding tie at the tolerance); CG
iteration counts within max(6, 10 %) (FP32 CG vectors against FP64)."""
import numpy as np
import pytest

from project_superdex_b200 import scenes

pytestmark = pytest.mark.gpu


def _oracle_scene(oracle, b, cfg):
    return oracle.Scene(b, cfg, min_eig=float(np.finfo(np.float32).eps))


def test_config0_full_run_matches_fp64_oracle(oracle):
    """cfg0 (10^3 cells, bottom pinned, gravity): all 100 backward-Euler steps, each compared."""
    from project_superdex_b200.soft_body import SoftBodyWorld
    bodies, cfg = scenes.config0()
    b = bodies[0]
    size = float(np.ptp(b.X, axis=0).max())
    w = SoftBodyWorld(bodies, cfg, newton_abs_tol=1e-9)
    s = _oracle_scene(oracle, b, cfg)
    p = oracle.default_newton_params()
    p.abs_tol = 1e-9
    u = np.zeros(3 * b.n_nodes)
    v = np.zeros_like(u)
    errs, newton_mismatch, cg_bad = [], [], []
    for k in range(100):
        w.step(1)
        u, v, st = s.step(u, v, (k + 1) * cfg.dt, p)
        ug, vg, _ = w.get_state()
        errs.append(float(np.abs(ug - u).max()))
        g = w.stats()[0]
        assert g["convergence"] == st.convergence == 1, (k, g, st.convergence)
        if g["newton_iters"] != st.newton_iters:
            newton_mismatch.append((k, g["newton_iters"], st.newton_iters))
        if abs(g["cg_iters"] - st.cg_iters) > max(6, int(0.1 * st.cg_iters)):
            cg_bad.append((k, g["cg_iters"], st.cg_iters))
    assert max(errs) <= 1e-5 * size, (max(errs), int(np.argmax(errs)))
    assert np.abs(u).max() > 1e3 * max(errs)  # the body moved: the comparison is not trivially small
    assert len(newton_mismatch) <= 5 and all(abs(a - o) <= 1 for _, a, o in newton_mismatch), newton_mismatch
    assert not cg_bad, cg_bad


def test_config2_first_envs_as_a_batch_match_fp64_oracle(oracle):
    """The first 8 envs of the batched workload (seed 0: 2,200-27,750 nodes, 515,466 tets, 5 capsules and a
    ground plane each) stepped together as one batch for 2 steps, against each env stepped alone by the
    oracle with the same Newton cap (12)."""
    from project_superdex_b200.soft_body import SoftBodyWorld
    all_bodies, cfg = scenes.config2(0, n_envs=8)
    bodies = all_bodies[:8]
    w = SoftBodyWorld(bodies, cfg, newton_abs_tol=1e-9, newton_max_iter=12)
    p = oracle.default_newton_params()
    p.abs_tol = 1e-9
    p.max_iter = 12
    sc = [_oracle_scene(oracle, b, cfg) for b in bodies]
    st_u = [np.zeros(3 * b.n_nodes) for b in bodies]
    st_v = [np.zeros(3 * b.n_nodes) for b in bodies]
    off = np.concatenate([[0], np.cumsum([3 * b.n_nodes for b in bodies])])
    for k in range(2):
        w.step(1)
        ug, _, _ = w.get_state()
        gs = w.stats()
        for e, b in enumerate(bodies):
            st_u[e], st_v[e], st = sc[e].step(st_u[e], st_v[e], (k + 1) * cfg.dt, p)
            size = float(np.ptp(b.X, axis=0).max())
            err = float(np.abs(ug[off[e]:off[e + 1]] - st_u[e]).max())
            assert gs[e]["convergence"] == st.convergence, (k, e, gs[e], st.convergence)
            assert err <= 1e-5 * size, (k, e, err / size)
            assert abs(gs[e]["newton_iters"] - st.newton_iters) <= 1, (k, e, gs[e]["newton_iters"], st.newton_iters)
        assert sum(g["n_contacts"] for g in gs) > 0


def _dense_free(row_ptr, col, blocks, free):
    n = row_ptr.size - 1
    A = np.zeros((3 * n, 3 * n))
    for i in range(n):
        for k in range(row_ptr[i], row_ptr[i + 1]):
            j = col[k]
            A[3 * i:3 * i + 3, 3 * j:3 * j + 3] = blocks[k]
    return A[np.ix_(free, free)]


def test_config0_precision_within_the_reference_fp32_mode(oracle, golden):
    """cfg0 against the reference's own FP32 build (MOCHI_USE_DOUBLE_PRECISION=0; fixture
    tests/golden/fp32_mode_reference.json, made from oracle/_ref/libsdx_ref_f32.so): one step from rest,
    the GPU's projected elastic Hessian (FP32 tangent) is at least as close to the FP64 result as the
    reference's FP32 mode is, and its linear solve of the next Newton system (FP32 matrix, FP64 x, r and
    dots) is within twice the FP32 mode's solution error, with the FP64 mode's iteration count."""
    import ctypes as C
    import dataclasses

    from project_superdex_b200 import capi
    from project_superdex_b200.soft_body import SoftBodyWorld
    fx = golden("fp32_mode_reference.json")
    bodies, cfg = scenes.config0()
    b = bodies[0]
    sc = _oracle_scene(oracle, b, cfg)
    p = oracle.default_newton_params()
    p.abs_tol = 1e-9
    u, v, _ = sc.step(np.zeros(3 * b.n_nodes), np.zeros(3 * b.n_nodes), cfg.dt, p)
    assert np.abs(u).sum() == pytest.approx(fx["hessian"]["u_abs_sum"], rel=1e-9)  # the fixture's state
    free = np.repeat(b.pin == 0, 3)
    # elastic Hessian (a dt so large that the inertia term vanishes), GPU vs FP64 oracle
    cfg_big = dataclasses.replace(cfg, dt=1e3)
    w = SoftBodyWorld(bodies, cfg_big)
    rp, col = w.pattern()
    assert np.array_equal(rp, sc.row_ptr) and np.array_equal(col, sc.col)
    Hg = w.assemble(u, hess=True, psd=True)["H"].astype(np.float64)
    Ho = _oracle_scene(oracle, b, cfg_big).assemble(u, u, hess=True, psd=True)["H"]
    Ag, Ao = _dense_free(rp, col, Hg, free), _dense_free(rp, col, Ho, free)
    err_gpu = float(np.linalg.norm(Ag - Ao) / np.linalg.norm(Ao))
    err_fp32_mode = fx["hessian"]["rel_fro_err_fp32_mode"]
    print(f"elastic Hessian rel. error vs FP64: GPU {err_gpu:.2e}, reference FP32 mode {err_fp32_mode:.2e}")
    assert err_gpu <= err_fp32_mode
    # the next Newton system, solved through sdx_pcg_solve (Jacobi, rel 1e-6)
    a = sc.assemble(u, u + cfg.dt * v, t=2 * cfg.dt, hess=True, psd=True)
    g = a["g"]
    x_exact, _ = oracle.pcg(sc.row_ptr, sc.col, a["H"], g, rel_tol=1e-13, abs_tol=0.0, max_iter=100000)
    lp = capi.default_linear_params()
    lp.rel_tol, lp.abs_tol, lp.value_layout = 1e-6, 0.0, capi.SDX_BSR_BLOCKS
    st = capi.LinearStatus()
    x = np.zeros_like(g)
    Hc = np.ascontiguousarray(a["H"].reshape(-1))
    capi.check(capi.lib().sdx_pcg_solve(b.n_nodes, col.size, capi.ptr(rp, capi._lp), capi.ptr(col, capi._ip),
                                        Hc.ctypes.data_as(C.c_void_p), capi.SDX_F64, capi.ptr(g), capi.ptr(x),
                                        capi.SDX_GUESS_ZERO, C.byref(lp), C.byref(st)))
    pc = fx["pcg"]
    err_x = float(np.linalg.norm(x - x_exact) / np.linalg.norm(x_exact))
    print(f"solution rel. error: GPU {err_x:.2e} ({st.num_iter} it), reference FP32 mode "
          f"{pc['rel_err_fp32_mode']:.2e} ({pc['iters_fp32_mode']} it), FP64 mode {pc['rel_err_fp64_mode']:.2e} "
          f"({pc['iters_fp64_mode']} it)")
    assert st.convergence == 1
    assert err_x <= 2.0 * pc["rel_err_fp32_mode"]
    assert abs(st.num_iter - pc["iters_fp64_mode"]) <= max(6, int(0.15 * pc["iters_fp64_mode"]))
