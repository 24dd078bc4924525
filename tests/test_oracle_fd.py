"""Finite-difference consistency of the oracle's incremental potential (energy -> gradient -> Hessian),
the reference's own test strategy for StressWork / contact (fem_stress_test.cpp:562-598,
contact_utils_test.cpp:359), plus invariants of the assembled system."""
import numpy as np
import pytest

from project_superdex_b200 import scenes


def _scene(oracle, with_contact=True, n=3):
    rng = np.random.default_rng(5)
    b = scenes.grid_body(n, n, n, 0.01, rng=rng, E=2e4, nu=0.4)
    if with_contact:
        top = n * 0.01
        b.colliders = [scenes.capsule((0.008, 0.015, top + 0.0035), (0.022, 0.015, top + 0.0035), 0.004, (0, 0, 0)),
                       scenes.plane((0, 0, 1), -0.0005)]
    cfg = scenes.SceneConfig(k_contact=1e6)
    return b, oracle.Scene(b, cfg, psd_strategy=0)


@pytest.mark.parametrize("with_contact", [False, True])
def test_gradient_and_hessian_match_finite_differences(oracle, with_contact):
    b, s = _scene(oracle, with_contact)
    rng = np.random.default_rng(1)
    free = (b.pin == 0).repeat(3)
    u = rng.normal(0, 4e-4, 3 * b.n_nodes) * free
    ut = u + rng.normal(0, 1e-4, u.size) * free
    out = s.assemble(u, ut, psd=False)
    g, H = out["g"], oracle.bsr_to_dense(s.row_ptr, s.col, out["H"])
    h = 1e-7
    idx = np.nonzero(free)[0][:: max(1, free.sum() // 12)]
    for i in idx:
        up, um = u.copy(), u.copy()
        up[i] += h
        um[i] -= h
        ep = s.assemble(up, ut, hess=False)["obj"]
        em = s.assemble(um, ut, hess=False)["obj"]
        assert (ep - em) / (2 * h) == pytest.approx(g[i], rel=1e-4, abs=1e-6 * np.abs(g).max())
        gp = s.assemble(up, ut, hess=False)["g"]
        gm = s.assemble(um, ut, hess=False)["g"]
        col = (gp - gm) / (2 * h)
        # contact Hessian omits the SDF curvature term (contact_utils.h:558-569): compare off-contact
        # columns tightly and contact columns loosely
        tol = 1e-4 if not with_contact else 5e-2
        np.testing.assert_allclose(col[free], H[free, i], rtol=tol, atol=tol * np.abs(H[:, i]).max())


def test_hessian_symmetric_psd_and_dirichlet(oracle):
    b, s = _scene(oracle, True)
    s.s.psd_strategy = 1
    rng = np.random.default_rng(2)
    u = rng.normal(0, 2e-3, 3 * b.n_nodes) * (b.pin == 0).repeat(3)
    out = s.assemble(u, u, psd=True)
    H = oracle.bsr_to_dense(s.row_ptr, s.col, out["H"])
    np.testing.assert_allclose(H, H.T, atol=1e-9 * np.abs(H).max())
    assert np.linalg.eigvalsh(H).min() > 0
    pinned = np.nonzero(b.pin.repeat(3))[0]
    assert np.all(out["g"][pinned] == 0)
    for i in pinned:
        row = H[i].copy()
        assert row[i] == 1.0
        row[i] = 0.0
        assert np.all(row == 0) and np.all(H[:, i][np.arange(H.shape[0]) != i] == 0)


def test_newton_step_reduces_residual_and_conserves_static_equilibrium(oracle):
    b, s = _scene(oracle, False, n=4)
    u = np.zeros(3 * b.n_nodes)
    v = np.zeros_like(u)
    p = oracle.default_newton_params()
    p.abs_tol = 1e-12
    u, v, st = s.step(u, v, s.cfg.dt, p)
    assert st.convergence == 1
    assert st.res_norm <= 1e-6 * st.res_norm0
    # the pinned bottom face does not move; gravity pulls the rest down
    assert np.all(u[np.nonzero(b.pin.repeat(3))[0]] == 0)
    assert u[2::3].min() < 0


def test_contact_pairs_sorted_unique(oracle):
    b, s = _scene(oracle, True)
    u = np.zeros(3 * b.n_nodes)
    u[2::3] = 0.002 * (b.X[:, 2] / b.X[:, 2].max())
    out = s.assemble(u, u, pairs=True)
    pr = out["pairs"]
    assert out["n_pairs"] > 0 and np.all(np.diff(pr) > 0)
    assert np.all(pr % len(b.colliders) < len(b.colliders))


@pytest.mark.parametrize("material", [0, 1, 2, 5])
def test_damped_materials_match_finite_differences(oracle, material):
    """Energy -> gradient -> Hessian consistency with Rayleigh mass and stiffness damping (about a
    stage-start displacement; the stiffness-damping Hessian with its geometric term is exact) for each
    soft material."""
    rng = np.random.default_rng(9 + material)
    b = scenes.grid_body(3, 3, 3, 0.01, rng=rng, E=2e4, nu=0.4)
    b.material = material
    cfg = scenes.SceneConfig(k_contact=1e6, mass_damping=3.0, stiffness_damping=0.02,
                             stiffness_damping_geometric=True)
    s = oracle.Scene(b, cfg, psd_strategy=0)
    free = (b.pin == 0).repeat(3)
    u = rng.normal(0, 4e-4, 3 * b.n_nodes) * free
    ut = u + rng.normal(0, 1e-4, u.size) * free
    us = u + rng.normal(0, 2e-4, u.size) * free
    out = s.assemble(u, ut, psd=False, u_stage=us)
    g, H = out["g"], oracle.bsr_to_dense(s.row_ptr, s.col, out["H"])
    h = 1e-7
    for i in np.nonzero(free)[0][:: max(1, free.sum() // 10)]:
        up, um = u.copy(), u.copy()
        up[i] += h
        um[i] -= h
        ep = s.assemble(up, ut, hess=False, u_stage=us)["obj"]
        em = s.assemble(um, ut, hess=False, u_stage=us)["obj"]
        assert (ep - em) / (2 * h) == pytest.approx(g[i], rel=1e-4, abs=1e-6 * np.abs(g).max())
        col = (s.assemble(up, ut, hess=False, u_stage=us)["g"] - s.assemble(um, ut, hess=False, u_stage=us)["g"]) / (2 * h)
        np.testing.assert_allclose(col[free], H[free, i], rtol=1e-4, atol=1e-4 * np.abs(H[:, i]).max())


@pytest.mark.parametrize("model", [0, 1])
def test_friction_response_is_the_derivative_of_its_energy(oracle, model):
    """With explicit normals the dissipation's normal force and friction plane are fixed by the stage
    start, so the dissipative force is minus the gradient of its energy in the sample position and, with
    the exact (unfitted) Coulomb Hessian, dforce is the force's derivative (contact_utils.h:700-960)."""
    rng = np.random.default_rng(11 + model)
    width = 0.01 / 240.0  # frictionFalloffVel * dt
    kw = dict(k=1e5, coulomb=0.6, viscous=0.2, normal_damping=0.3, explicit_normals=1, fitted=0, model=model)
    prm = oracle.contact_params(**kw)
    pen = oracle.contact_params(**{**kw, "coulomb": 0.0, "viscous": 0.0, "normal_damping": 0.0})
    dt = 1.0 / 240.0
    for trial in range(16):
        g = rng.normal(size=3)
        g /= np.linalg.norm(g)
        gs = g + 0.05 * rng.normal(size=3)
        gs /= np.linalg.norm(gs)
        nc = -gs + 0.2 * rng.normal(size=3)
        nc /= np.linalg.norm(nc)
        d, dss = -0.002, float(rng.uniform(-0.004, 0.0))
        pss = rng.normal(size=3) * 0.01
        step = rng.normal(size=3) * width * float(rng.choice([0.2, 0.6, 3.0, 30.0]))
        pos = pss + step
        e0, f0, d0 = oracle.collision_response(pen, d, g, dss, gs, nc, pos, pss, dt)
        e, f, D = oracle.collision_response(prm, d, g, dss, gs, nc, pos, pss, dt)
        fd, Dd = f - f0, D - d0
        h = 1e-4 * np.linalg.norm(step)
        for i in range(3):
            dp = np.zeros(3)
            dp[i] = h
            ep, fp, _ = oracle.collision_response(prm, d, g, dss, gs, nc, pos + dp, pss, dt)
            em, fm, _ = oracle.collision_response(prm, d, g, dss, gs, nc, pos - dp, pss, dt)
            assert -(ep - em) / (2 * h) == pytest.approx(fd[i], rel=1e-5, abs=1e-7 * np.abs(fd).max())
            np.testing.assert_allclose((fp - fm) / (2 * h), Dd[:, i], rtol=1e-4, atol=1e-5 * np.abs(Dd).max())


def test_friction_with_explicit_normals_is_a_gradient_system(oracle):
    """Assembled over a body with a plane pressing on its top and sliding along it: with explicit normals
    the contact residual is the exact gradient of the contact merit (ExperimentalEvalParams::
    explicitNormals, eval_params.h:73-85), and with the unfitted Coulomb Hessian and a flat collider the
    Hessian is its exact derivative."""
    rng = np.random.default_rng(7)
    n = 3
    b = scenes.grid_body(n, n, n, 0.01, rng=rng, E=2e4, nu=0.4)
    top = n * 0.01
    b.colliders = [scenes.plane((0, 0, -1), -(top - 0.0015), (0.05, 0.02, 0.0))]
    kw = dict(friction_coulomb=0.6, friction_viscous=0.1, contact_normal_damping=0.05, contact_explicit_normals=True,
              friction_fitted_hessian=False)
    cfg = scenes.SceneConfig(k_contact=1e9, **kw)  # the reference's default penalty stiffness
    s = oracle.Scene(b, cfg, psd_strategy=0)
    free = (b.pin == 0).repeat(3)
    us = rng.normal(0, 1e-4, 3 * b.n_nodes) * free
    u = us + rng.normal(0, 6e-5, 3 * b.n_nodes) * free
    ut = us.copy()
    t = 0.02
    out = s.assemble(u, ut, t=t, psd=False, u_stage=us)
    assert out["n_pairs"] > 0
    s0 = oracle.Scene(b, scenes.SceneConfig(k_contact=1e9, contact_explicit_normals=True), psd_strategy=0)
    g0 = s0.assemble(u, ut, t=t, psd=False, u_stage=us)["g"]
    assert np.abs(out["g"] - g0).max() > 0.2 * np.abs(out["g"]).max()  # the dissipative terms matter here
    g, H = out["g"], oracle.bsr_to_dense(s.row_ptr, s.col, out["H"])
    h = 1e-8
    top_nodes = np.nonzero(np.abs(b.X[:, 2] - top) < 1e-9)[0]
    idx = [3 * i + r for i in top_nodes[:: max(1, top_nodes.size // 6)] for r in range(3)]
    for i in idx:
        up, um = u.copy(), u.copy()
        up[i] += h
        um[i] -= h
        ap = s.assemble(up, ut, t=t, hess=False, u_stage=us)
        am = s.assemble(um, ut, t=t, hess=False, u_stage=us)
        assert (ap["obj"] - am["obj"]) / (2 * h) == pytest.approx(g[i], rel=1e-5, abs=1e-7 * np.abs(g).max())
        col = (ap["g"] - am["g"]) / (2 * h)
        np.testing.assert_allclose(col[free], H[free, i], rtol=1e-4, atol=1e-5 * np.abs(H[:, i]).max())
