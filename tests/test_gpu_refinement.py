"""Mixed-precision iterative refinement around the PCG (sdx_linear_params.refine_inner_rel_tol): passes of
the FP32-matrix / FP64-reduction PCG to a loose inner tolerance, each later pass correcting x by a solve
against the FP64 residual b - A x, until ||b - A x|| meets the outer tolerance. Checked through the C-ABI
on the reference's golden systems and on an assembled tet system, and through Newton steps against the
FP64 oracle."""
import ctypes as C

import numpy as np
import pytest

from project_superdex_b200 import scenes

pytestmark = pytest.mark.gpu


def _fem_system(oracle, seed):
    rng = np.random.default_rng(seed)
    b = scenes.grid_body(8, 7, 6, 0.01, rng=rng, nu=0.45)
    b.E = np.exp(rng.uniform(np.log(1e4), np.log(1e7), size=b.n_tets))
    s = oracle.Scene(b, scenes.SceneConfig())
    u = rng.normal(0, 5e-4, 3 * b.n_nodes) * (b.pin == 0).repeat(3)
    a = s.assemble(u, u - 1e-4, psd=True)
    return s.row_ptr, s.col, a["H"].astype(np.float32), a["g"]


def _solve(rp, col, H, b, inner=0.0, passes=8, prec=1, rel_tol=1e-6):
    from project_superdex_b200 import capi
    lp = capi.default_linear_params()
    lp.rel_tol, lp.abs_tol, lp.preconditioner, lp.value_layout = rel_tol, 1e-30, prec, capi.SDX_BSR_BLOCKS
    lp.refine_inner_rel_tol, lp.refine_max_passes = inner, passes
    st = capi.LinearStatus()
    x = np.zeros_like(b)
    Hc = np.ascontiguousarray(H, np.float32)
    rp64 = np.ascontiguousarray(rp, np.int64)
    cl = np.ascontiguousarray(col, np.int32)
    rc = capi.lib().sdx_pcg_solve(rp64.size - 1, cl.size, capi.ptr(rp64, capi._lp), capi.ptr(cl, capi._ip),
                                  Hc.ctypes.data_as(C.c_void_p), capi.SDX_F32, capi.ptr(np.ascontiguousarray(b)),
                                  capi.ptr(x), capi.SDX_GUESS_ZERO, C.byref(lp), C.byref(st))
    capi.check(rc)
    return x, st


def _rel_residual(rp, col, H, x, b):
    y = np.zeros_like(b)
    for i in range(rp.size - 1):
        for k in range(rp[i], rp[i + 1]):
            y[3 * i:3 * i + 3] += H[k].astype(np.float64) @ x[3 * col[k]:3 * col[k] + 3]
    return np.linalg.norm(b - y) / np.linalg.norm(b)


def _golden_systems(golden):
    from project_superdex_b200.linear_solver import strips_to_blocks
    out = []
    for sysd in golden("bsr3_reference.json")["pcg"]:
        rp = np.array(sysd["row_ptr"])
        out.append((sysd["system"], rp, np.array(sysd["col"], np.int32),
                    strips_to_blocks(rp, np.array(sysd["values"])).astype(np.float32), np.array(sysd["b"])))
    return out


@pytest.mark.parametrize("inner", [1e-1, 1e-2, 1e-3])
def test_refined_solve_meets_the_outer_tolerance(oracle, golden, inner):
    systems = [(n, rp, col, H, b) for n, rp, col, H, b in _golden_systems(golden)]
    systems.append(("fem",) + _fem_system(oracle, 11))
    for name, rp, col, H, b in systems:
        x0, st0 = _solve(rp, col, H, b)
        x, st = _solve(rp, col, H, b, inner=inner)
        assert st.convergence == 1, name
        rel = _rel_residual(rp, col, H, x, b)
        assert rel <= 1.01e-6, (name, rel)
        assert st.relative_residual_norm == pytest.approx(rel, rel=1e-3, abs=1e-12)
        # both solutions lie within the tolerance's reach of A^-1 b
        np.testing.assert_allclose(x, x0, rtol=0, atol=2e-4 * np.abs(x0).max())
        # restarting the Krylov space costs iterations, within a small factor of the single solve
        assert st0.num_iter <= st.num_iter * 1.5 + 10 and st.num_iter <= 3 * st0.num_iter + 10, (name, st.num_iter,
                                                                                              st0.num_iter)


def test_refinement_pass_cap_stops_short(oracle):
    rp, col, H, b = _fem_system(oracle, 12)
    x, st = _solve(rp, col, H, b, inner=0.5, passes=0)
    assert st.convergence == 2  # stopped: pass 0 reached only the inner tolerance
    rel = _rel_residual(rp, col, H, x, b)
    assert 1e-6 < rel <= 0.5 and st.relative_residual_norm == pytest.approx(rel, rel=1e-3)


def test_refinement_rejects_bad_parameters(oracle):
    from project_superdex_b200 import capi
    rp, col, H, b = _fem_system(oracle, 13)
    with pytest.raises(capi.SdxError):
        _solve(rp, col, H, b, inner=1.5)
    with pytest.raises(capi.SdxError):
        _solve(rp, col, H, b, inner=1e-2, passes=-1)


@pytest.mark.parametrize("warm", [0, 1])
def test_refined_newton_steps_match_oracle(oracle, warm):
    """Zero and previous-solve starts (SDX_WARM_ZERO, SDX_WARM_PREVIOUS), a single body and a batch of three
    uneven bodies with contact."""
    import test_gpu_step as ts

    def check(bodies, ug, states, hist):
        off = 0
        for e, b in enumerate(bodies):
            size = np.ptp(b.X, axis=0).max()
            assert np.abs(ug[off:off + 3 * b.n_nodes] - states[e][0]).max() <= 1e-5 * size
            off += 3 * b.n_nodes
        for st_gpu, st_or in hist:
            for g, o in zip(st_gpu, st_or):
                assert g["convergence"] == o.convergence
                # the restarted passes cost iterations over one unrestarted solve (the oracle's)
                assert 0.5 * o.cg_iters - 6 <= g["cg_iters"] <= 1.6 * o.cg_iters + 6, (g["cg_iters"], o.cg_iters)

    bodies, cfg = scenes.config0()
    w, ug, vg, states, hist = ts._run(oracle, bodies, cfg, 3, warm_start=warm, linear_refine_inner_rel_tol=1e-2)
    check(bodies, ug, states, hist)
    batch = []
    for i, n in enumerate((3, 5, 4)):
        rng = np.random.default_rng(20 + i)
        b = scenes.grid_body(n, n, n, 0.01, rng=rng, E=float(rng.uniform(3e4, 3e5)), nu=0.4)
        b.colliders = [scenes.capsule((0.01, 0.01, n * 0.01 + 0.0035), (0.02, 0.02, n * 0.01 + 0.0035), 0.004,
                                      (0, 0, -0.1))]
        batch.append(b)
    cfg = scenes.SceneConfig(k_contact=1e6)
    w, ug, vg, states, hist = ts._run(oracle, batch, cfg, 3, warm_start=warm, linear_refine_inner_rel_tol=1e-2)
    check(batch, ug, states, hist)
