"""Pins the CPU oracle (oracle/sdx_oracle.c) to the reference: its golden vectors (read as text from the
reference test data) and outputs of the reference's own compiled code (tests/golden/reference_vectors.json)."""
import numpy as np
import pytest

from conftest import dense_from_coo, scalar_to_block


def test_smith_nh_known_answers(oracle, golden):
    """material_test_data.h smith_neo_hookean_test_data (E = 1, nu = 0.4), as batched_materials_test.cpp:413."""
    g = golden("smith_nh_reference.json")
    lam, mu = 1.0 * 0.4 / ((1 + 0.4) * (1 - 0.8)), 1.0 / (2 * 1.4)
    assert len(g["cases"]) == 5
    for c in g["cases"]:
        e, P, C = oracle.smith_nh(mu, lam, np.array(c["F"]), project=False, psd=0)
        # golden data carries 7 significant digits
        assert e == pytest.approx(c["energy"], rel=2e-5, abs=1e-6)
        np.testing.assert_allclose(P.reshape(-1), c["pk1"], rtol=2e-5, atol=2e-6)
        np.testing.assert_allclose(C.reshape(-1), c["tangent"], rtol=2e-5, atol=2e-6)


def test_stvk_known_answers(oracle, golden):
    """material_test_data.h st_venant_kirchhoff_test_data (E = 1, nu = 0.4), as batched_materials_test.cpp:240."""
    g = golden("stvk_reference.json")
    lam, mu = 1.0 * 0.4 / ((1 + 0.4) * (1 - 0.8)), 1.0 / (2 * 1.4)
    assert len(g["cases"]) == 6
    for c in g["cases"]:
        e, P, C = oracle.material(1, mu, lam, np.array(c["F"]), project=False, psd=0)
        assert e == pytest.approx(c["energy"], rel=2e-5, abs=1e-6)
        np.testing.assert_allclose(P.reshape(-1), c["pk1"], rtol=2e-5, atol=2e-6)
        np.testing.assert_allclose(C.reshape(-1), c["tangent"], rtol=2e-5, atol=2e-6)


def test_stvk_and_linear_elastic_match_reference_code(oracle, golden):
    """St. Venant-Kirchhoff and linear elasticity with every PSD strategy against the reference's own
    compiled translation units (batched_st_venant_kirchhoff.cpp, batched_linear_elastic.cpp)."""
    v = golden("reference_vectors.json")
    assert len(v["materials"]) == 96
    for c in v["materials"]:
        e, P, C = oracle.material(c["kind"], c["mu"], c["lambda"], np.array(c["F"]), project=c["psd"] != 0,
                                  psd=c["psd"])
        scale = max(1.0, np.abs(c["tangent"]).max())
        assert e == pytest.approx(c["energy"], rel=1e-11, abs=1e-11)
        np.testing.assert_allclose(P.reshape(-1), c["pk1"], rtol=1e-11, atol=1e-11)
        np.testing.assert_allclose(C.reshape(-1), c["tangent"], rtol=1e-9, atol=1e-10 * scale)


def test_smith_nh_all_psd_strategies_match_reference_code(oracle, golden):
    v = golden("reference_vectors.json")
    assert len(v["smith"]) == 192
    for c in v["smith"]:
        e, P, C = oracle.smith_nh(c["mu"], c["lambda"], np.array(c["F"]), project=c["psd"] != 0, psd=c["psd"])
        scale = max(1.0, np.abs(c["tangent"]).max())
        assert e == pytest.approx(c["energy"], rel=1e-11, abs=1e-11)
        np.testing.assert_allclose(P.reshape(-1), c["pk1"], rtol=1e-11, atol=1e-11)
        np.testing.assert_allclose(C.reshape(-1), c["tangent"], rtol=1e-9, atol=1e-10 * scale)


def test_projected_tangent_is_psd(oracle, golden):
    v = golden("reference_vectors.json")
    for c in v["smith"]:
        if c["psd"] in (1, 2):
            _, _, C = oracle.smith_nh(c["mu"], c["lambda"], np.array(c["F"]), project=True, psd=c["psd"])
            assert np.linalg.eigvalsh(0.5 * (C + C.T)).min() > -1e-9 * np.abs(C).max()


def test_polyrelu_matches_reference(oracle, golden):
    for c in golden("reference_vectors.json")["polyrelu"]:
        f, df, ddf = oracle.polyrelu(c["x"], c["t"], c["shift"])
        assert (f, df, ddf) == pytest.approx((c["f"], c["df"], c["ddf"]), rel=1e-14, abs=1e-16)


def test_penalty_matches_reference(oracle, golden):
    for c in golden("reference_vectors.json")["penalty"]:
        e, f, df = oracle.penalty(c["d"], np.array(c["grad"]), c["k"], c["t_half"], c["thr"])
        assert e == pytest.approx(c["energy"], rel=1e-12, abs=1e-300)
        np.testing.assert_allclose(f, c["force"], rtol=1e-12, atol=1e-300)
        d6 = [df[0, 0], df[1, 1], df[2, 2], df[0, 1], df[0, 2], df[1, 2]]
        np.testing.assert_allclose(d6, c["dforce6"], rtol=1e-12, atol=1e-300)


def test_stress_work_matches_reference(oracle, golden):
    """Single-tet StressWork (fem_stress.h:107) through the oracle's assembly (no inertia/gravity)."""
    from project_superdex_b200 import scenes
    for c in golden("reference_vectors.json")["stress_work"]:
        X = np.array(c["X"]).reshape(4, 3)
        b = scenes.Body(X=X, tets=np.array([[0, 1, 2, 3]], np.int32), E=np.array([1.0]), nu=np.array([0.3]),
                        rho=np.array([0.0]), pin=np.zeros(4, np.uint8), colliders=[])
        s = oracle.Scene(b, scenes.SceneConfig(gravity=(0, 0, 0)))
        s.mu[:] = c["mu"]
        s.lam[:] = c["lambda"]
        u = np.array(c["u"])
        out = s.assemble(u, u, psd=bool(c["project"]))
        K = oracle.bsr_to_dense(s.row_ptr, s.col, out["H"])
        assert out["obj"] == pytest.approx(c["energy"], rel=1e-11)
        np.testing.assert_allclose(out["g"], c["res"], rtol=1e-10, atol=1e-12 * np.abs(c["res"]).max())
        np.testing.assert_allclose(K.reshape(-1), c["K"], rtol=1e-9, atol=1e-11 * np.abs(c["K"]).max())


@pytest.mark.parametrize("system", ["psd100", "tridiag64"])
def test_pcg_iteration_counts_match_reference(oracle, golden, system):
    """krylov::PCG (pcg.h:70) on the reference's golden systems: identical iteration counts."""
    kr = golden("krylov_psd100.json")
    if system == "psd100":
        A = dense_from_coo(100, kr["rows"], kr["cols"], kr["vals"])
        b = np.array(kr["rhs"])
        x_true = np.array(kr["solution"])
    else:
        A = np.diag(np.full(64, 2.0)) - np.diag(np.ones(63), 1) - np.diag(np.ones(63), -1)
        b = np.ones(64)
        x_true = np.array([(i + 1) * (64 - i) / 2.0 for i in range(64)])
    n = A.shape[0]
    rp, col, vals, bp = scalar_to_block(A, b)
    for ref in [p for p in golden("reference_vectors.json")["pcg"] if p["system"] == system]:
        # the oracle's Jacobi on the block embedding equals the reference's scalar Jacobi
        x, st = oracle.pcg(rp, col, vals, bp, rel_tol=ref["rel_tol"], abs_tol=1e-30,
                           precond=1 if ref["jacobi"] else 0)
        assert st.num_iter == ref["iters"]
        assert st.convergence == ref["convergence"]
        np.testing.assert_allclose(x[:n], ref["x"], rtol=1e-9, atol=1e-9 * np.abs(ref["x"]).max())
        if ref["rel_tol"] == 1e-10:
            # golden solution of the test data (krylov_solver_test_data.h kPsdMatrixOut) within the
            # reference test's own bound eps_f32 * n * cond (krylov_solver_test_helpers.h:34-38)
            cond = 2.4104e05 if system == "psd100" else 1712.0
            err = np.linalg.norm(x[:n] - x_true) / np.linalg.norm(x_true)
            assert err < np.finfo(np.float32).eps * n * cond


def test_pcg_stop_and_divergence_statuses(oracle):
    A = np.diag(np.arange(1.0, 10.0))
    rp, col, vals, bp = scalar_to_block(A, np.ones(9))
    x, st = oracle.pcg(rp, col, vals, bp, rel_tol=1e-12, max_iter=2, precond=0)
    assert st.convergence == 2 and st.num_iter == 2  # Stopped at maxIter
    x, st = oracle.pcg(rp, col, vals, bp, rel_tol=1e-12, precond=1)
    assert st.convergence == 1 and st.num_iter == 1  # Jacobi solves a diagonal system at once
    Z = np.zeros((9, 9))
    rp, col, vals, bp = scalar_to_block(Z + np.eye(9), np.zeros(9))
    x, st = oracle.pcg(rp, col, vals, bp)
    assert st.convergence == 1 and st.num_iter == 0  # b = 0: converged at iteration 0


def test_stop_test_classification_known_answers(oracle):
    """The reference's StopTest known answers (mochi_core/test/stopping_criterion_test.cpp:24-39, 41-46):
    relTol 1e-3, absTol 1e-6, relDivTol 10, scaling 1, by squared residual norm. 0 active, 1 converged
    (relative), 2 converged (absolute), 3 diverged."""
    eps = np.finfo(np.float64).eps

    def cls(rr):
        return oracle.stop_status(rr, 1.0, 1e-3, 1e-6, 10.0)

    assert cls(-1.0) == 3                    # negative beyond round-off: DivergedRes
    assert cls(-eps) == 2                    # round-off below zero counts as 0: ConvergedAtol
    assert cls(1e-14) == 2                   # ConvergedAtol
    assert cls(1e-8) == 1                    # ConvergedRtol
    assert cls(1e-3) == 0                    # Active
    assert cls(101.0) == 3                   # DivergedRes
    assert cls(float("nan")) == 3 and cls(float("inf")) == 3


def test_stiffness_damping_matches_reference_code(oracle, golden):
    """The oracle's viscous-stress damping against fem::StressDampingWork compiled from the reference."""
    import ctypes as C
    L = oracle.lib()
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    v = golden("reference_vectors.json")
    assert len(v["stress_damping"]) == 16
    for c in v["stress_damping"]:
        X = np.array(c["X"])
        tets = np.arange(4, dtype=np.int32)
        dN = np.zeros(12)
        vol = np.zeros(1)
        L.or_rest_data(1, tets.ctypes.data_as(C.POINTER(C.c_int32)), dp(X), dp(dN), dp(vol))
        e, r, K = np.zeros(1), np.zeros(12), np.zeros(144)
        L.or_stress_damping(dp(dN), vol[0], dp(np.array(c["u"])), dp(np.array(c["uss"])), c["kappa"], c["lambda"],
                            c["mu"], c["geometric"], c["project"], dp(e), dp(r), dp(K))
        assert e[0] == pytest.approx(c["energy"], rel=1e-11, abs=1e-18)
        np.testing.assert_allclose(r, c["res"], rtol=1e-10, atol=1e-12 * np.abs(c["res"]).max())
        np.testing.assert_allclose(K, c["K"], rtol=1e-10, atol=1e-12 * np.abs(c["K"]).max())


def test_collision_response_matches_reference_code(oracle, golden):
    """or_collision_response (penalty + Coulomb / viscous friction + normal viscous damping) against the
    reference's ComputeBatchCollisionForceDForce<1, GradTarget::Current> compiled from its sources, over
    random option sets (friction model, fitted Hessian, explicit normals, implicit normal force, fading,
    friction normal, invalid colliding normals)."""
    v = golden("reference_vectors.json")["collision"]
    assert len(v) == 128
    n_diss = 0
    for c in v:
        prm = oracle.contact_params(**c["params"])
        e, f, df = oracle.collision_response(prm, c["d"], c["grad"], c["d_ss"], c["grad_ss"], c["n_col"], c["pos"],
                                             c["pos_ss"], c["dt"])
        fs = max(np.abs(c["force"]).max(), 1e-300)
        ds = max(np.abs(c["dforce"]).max(), 1e-300)
        assert e == pytest.approx(c["energy"], rel=1e-12, abs=1e-300)
        np.testing.assert_allclose(f, c["force"], rtol=1e-12, atol=1e-13 * fs)
        np.testing.assert_allclose(df.reshape(-1), c["dforce"], rtol=1e-12, atol=1e-13 * ds)
        p = c["params"]
        n_diss += (p["coulomb"] > 0 or p["viscous"] > 0 or p["normal_damping"] > 0) and c["energy"] > 0
    assert n_diss >= 40  # the set exercises the dissipative terms, not only the penalty


def test_arap_matches_reference_code(oracle, golden):
    """The oracle's ARAP (own rotation-variant SVD, exact Hessian, spectral clamp) against the reference's
    BatchedArapConstitutiveResponse compiled from batched_arap.cpp, inverted elements and every PSD strategy
    it supports."""
    v = golden("reference_vectors.json")["arap"]
    assert len(v) == 96
    for c in v:
        e, P, C = oracle.material(5, c["mu"], 0.0, np.array(c["F"]), project=c["psd"] != 0, psd=c["psd"])
        scale = max(1.0, np.abs(c["tangent"]).max())
        assert e == pytest.approx(c["energy"], rel=1e-11, abs=1e-12)
        np.testing.assert_allclose(P.reshape(-1), c["pk1"], rtol=1e-10, atol=1e-11)
        np.testing.assert_allclose(C.reshape(-1), c["tangent"], rtol=1e-9, atol=1e-10 * scale)


def test_reference_stiffness_of_each_material(golden):
    """The rest stiffness the Rayleigh stiffness damping uses (ComputeReferenceMaterialStiffnessVoigt) is the
    isotropic (lambda, mu) for Neo-Hookean, StVK and linear elasticity and (0, mu / 2) for ARAP."""
    for c in golden("reference_vectors.json")["reference_stiffness"]:
        lam0, mu0 = (0.0, 0.5 * c["mu"]) if c["kind"] == 5 else (c["lambda"], c["mu"])
        want = np.zeros((6, 6))
        want[:3, :3] = lam0
        want[np.arange(3), np.arange(3)] += 2 * mu0
        want[np.arange(3, 6), np.arange(3, 6)] = mu0
        np.testing.assert_allclose(np.array(c["c0"]).reshape(6, 6), want, rtol=1e-9, atol=1e-9 * c["lambda"])


def test_fp32_mode_fixture_matches_this_oracle(oracle, golden):
    """The FP32-mode fixture (the reference's MOCHI_USE_DOUBLE_PRECISION=0 build against its FP64 build on
    cfg0) was made at the state this oracle reaches one step from rest, and its FP64 side agrees with the
    oracle's own elastic Hessian."""
    from project_superdex_b200 import scenes
    fx = golden("fp32_mode_reference.json")
    bodies, cfg = scenes.config0()
    b = bodies[0]
    sc = oracle.Scene(b, cfg, min_eig=float(np.finfo(np.float32).eps))
    p = oracle.default_newton_params()
    p.abs_tol = 1e-9
    u, v, _ = sc.step(np.zeros(3 * b.n_nodes), np.zeros(3 * b.n_nodes), cfg.dt, p)
    assert np.abs(u).sum() == pytest.approx(fx["hessian"]["u_abs_sum"], rel=1e-9)
    assert fx["hessian"]["oracle_vs_fp64_mode_rel_fro"] < 1e-6
    assert fx["pcg"]["convergence_fp32_mode"] == fx["pcg"]["convergence_fp64_mode"] == 1


def test_gravity_work_analytic_properties(oracle):
    """The reference's gravity known answers (mochi_core/test/fem_gravity_test.cpp:96-170, the analytic
    check) on the oracle's assembled system: with a non-axis-aligned gravity g, the gravity part of the
    residual (assembly with g minus assembly with g = 0 at the same state) is -rho vol/4 g at each of a tet's
    nodes, summed over the tets (zero on pinned DoFs), independent of the displacement; and its energy obeys
    E(u) - E(0) = <r, u>."""
    from project_superdex_b200 import scenes
    rng = np.random.default_rng(3)
    b = scenes.grid_body(4, 3, 3, 0.01, rng=rng, rho=1234.5)
    g = (0.31, -9.81, 1.73)
    cfg_g, cfg_0 = scenes.SceneConfig(gravity=g), scenes.SceneConfig(gravity=(0.0, 0.0, 0.0))
    free = (b.pin == 0).repeat(3)
    X, T = b.X, b.tets
    vol = np.abs(np.einsum("ij,ij->i", np.cross(X[T[:, 1]] - X[T[:, 0]], X[T[:, 2]] - X[T[:, 0]]),
                           X[T[:, 3]] - X[T[:, 0]])) / 6.0
    want = np.zeros((b.n_nodes, 3))
    for k in range(4):
        np.add.at(want, T[:, k], -(b.rho * vol / 4.0)[:, None] * np.asarray(g)[None, :])
    want = want.reshape(-1) * free
    parts = []
    for u in (np.zeros(3 * b.n_nodes), rng.normal(0, 1e-3, 3 * b.n_nodes) * free):
        ag = oracle.Scene(b, cfg_g).assemble(u, u, hess=False)
        a0 = oracle.Scene(b, cfg_0).assemble(u, u, hess=False)
        parts.append((ag["obj"] - a0["obj"], ag["g"] - a0["g"], u))
    for _, r, _ in parts:
        np.testing.assert_allclose(r, want, rtol=1e-12, atol=1e-12 * np.abs(want).max())
    (e0, _, _), (e1, r1, u1) = parts
    assert e1 - e0 == pytest.approx(float(r1 @ u1), rel=1e-9)


def test_inertia_work_matches_the_consistent_mass_matrix(oracle):
    """The reference's inertia identities (mochi_core/test/fem_inertia_test.cpp:30-37) on the oracle's
    assembly: with a = u - ut and M the P1 consistent mass matrix (rho vol / 20 (1 + delta_fg) per node
    pair, assembled here independently of the oracle), the inertia part of the residual is M a / dt^2 and of
    the energy a^T M a / (2 dt^2); the elastic part cancels between two assemblies at the same u."""
    from project_superdex_b200 import scenes
    rng = np.random.default_rng(5)
    b = scenes.grid_body(3, 3, 2, 0.01, rng=rng, rho=870.0, pin_bottom=False)
    cfg = scenes.SceneConfig(gravity=(0.0, 0.0, 0.0))
    X, T = b.X, b.tets
    vol = np.abs(np.einsum("ij,ij->i", np.cross(X[T[:, 1]] - X[T[:, 0]], X[T[:, 2]] - X[T[:, 0]]),
                           X[T[:, 3]] - X[T[:, 0]])) / 6.0
    M = np.zeros((b.n_nodes, b.n_nodes))
    for t in range(b.n_tets):
        m = b.rho[t] * vol[t] / 20.0
        for f in range(4):
            for g in range(4):
                M[T[t, f], T[t, g]] += m * (2.0 if f == g else 1.0)
    u = rng.normal(0, 1e-3, 3 * b.n_nodes)
    ut = u - rng.normal(0, 1e-3, 3 * b.n_nodes)
    s = oracle.Scene(b, cfg)
    a_in = s.assemble(u, ut, hess=False)
    a_el = s.assemble(u, u, hess=False)
    inv_dt2 = 1.0 / cfg.dt ** 2
    a = (u - ut).reshape(-1, 3)
    want_r = inv_dt2 * (M @ a).reshape(-1)
    np.testing.assert_allclose(a_in["g"] - a_el["g"], want_r, rtol=1e-10, atol=1e-10 * np.abs(want_r).max())
    want_e = 0.5 * inv_dt2 * float(np.sum(a * (M @ a)))
    assert a_in["obj"] - a_el["obj"] == pytest.approx(want_e, rel=1e-9)
    assert M.sum() == pytest.approx(float(np.sum(b.rho * vol)), rel=1e-12)  # total mass
