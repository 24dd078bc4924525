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


@pytest.mark.parametrize("material", [0, 1, 2])
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
