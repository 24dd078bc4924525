"""GPU FEM-body assembly (sdx_assemble) against the CPU oracle: gradient (FP64 path), Hessian (FP32
path, every PSD strategy), objective, Dirichlet rows, block pattern, boundary faces, and bit-exact
contact-pair indexing."""
import numpy as np
import pytest

from project_superdex_b200 import scenes

pytestmark = pytest.mark.gpu


def _body(seed=0, n=5, contact=True):
    rng = np.random.default_rng(seed)
    b = scenes.grid_body(n, n + 1, n - 1, 0.01, rng=rng, E=1e5, nu=0.45)
    b.E = np.exp(rng.uniform(np.log(1e4), np.log(1e6), size=b.n_tets))
    if contact:
        top = (n - 1) * 0.01
        b.colliders = [scenes.capsule((0.012, 0.02, top + 0.0032), (0.032, 0.03, top + 0.0032), 0.004, (0, 0, -0.05)),
                       scenes.capsule((0.02, 0.045, top + 0.0045), (0.03, 0.05, top + 0.0045), 0.004, (0.01, 0, -0.05)),
                       scenes.plane((1, 0, 0), -0.0008, (0.01, 0, 0))]
    return b


def _pair(oracle, b, cfg, psd=1):
    from project_superdex_b200.soft_body import SoftBodyWorld
    w = SoftBodyWorld([b], cfg, psd_strategy=psd)
    s = oracle.Scene(b, cfg, psd_strategy=psd, min_eig=float(np.finfo(np.float32).eps))
    return w, s


@pytest.mark.parametrize("psd", [0, 1, 2, 3])
def test_assembly_matches_oracle(oracle, psd):
    b = _body(psd)
    cfg = scenes.SceneConfig(k_contact=1e6)
    w, s = _pair(oracle, b, cfg, psd)
    rng = np.random.default_rng(100 + psd)
    free = (b.pin == 0).repeat(3)
    # large enough deformation that some tets are indefinite (exercises the projection path)
    u = rng.normal(0, 1.5e-3, 3 * b.n_nodes) * free
    v = rng.normal(0, 2e-2, 3 * b.n_nodes) * free
    w.set_state(np.zeros_like(u), v, 0.0)
    t = 0.02
    a_gpu = w.assemble(u, t=t, psd=psd != 0)
    a_or = s.assemble(u, cfg.dt * v, t=t, psd=psd != 0, pairs=True)
    rp, col = w.pattern()
    assert np.array_equal(rp, s.row_ptr) and np.array_equal(col, s.col)
    g_scale = np.abs(a_or["g"]).max()
    np.testing.assert_allclose(a_gpu["g"], a_or["g"], rtol=0, atol=1e-6 * g_scale)
    H_scale = np.abs(a_or["H"]).max()
    np.testing.assert_allclose(a_gpu["H"], a_or["H"], rtol=0, atol=2e-5 * H_scale)
    assert a_gpu["obj"][0] == pytest.approx(a_or["obj"], rel=1e-6)
    assert a_gpu["n_pairs"][0] == a_or["n_pairs"] > 0
    assert np.array_equal(w.contact_pairs(), a_or["pairs"])  # bit-exact pair indexing


def test_faces_and_dirichlet(oracle):
    b = _body(7)
    cfg = scenes.SceneConfig(k_contact=1e6)
    w, s = _pair(oracle, b, cfg)
    fn, ft, fa = w.faces()
    assert np.array_equal(fn, s.face_nodes) and np.array_equal(ft, s.face_tet)
    np.testing.assert_allclose(fa, s.face_area, rtol=1e-15)
    a = w.assemble(np.zeros(3 * b.n_nodes), t=0.0)
    pinned = np.nonzero(b.pin)[0]
    assert np.all(a["g"].reshape(-1, 3)[pinned] == 0)
    rp, col = w.pattern()
    H = a["H"]
    for i in pinned[:20]:
        for k in range(rp[i], rp[i + 1]):
            blk = H[k]
            if col[k] == i:
                assert np.array_equal(blk, np.eye(3, dtype=np.float32))
            else:
                assert np.all(blk == 0)
            # column side: block (col, i) is zero too
            j = col[k]
            kk = rp[j] + np.searchsorted(col[rp[j]:rp[j + 1]], i)
            if j != i:
                assert np.all(H[kk] == 0)


def test_batched_uneven_envs_match_per_env_oracle(oracle):
    from project_superdex_b200.soft_body import SoftBodyWorld
    bodies = [_body(11, n=3), _body(12, n=6), _body(13, n=4)]
    bodies[1].pin[:] = 0
    cfg = scenes.SceneConfig(k_contact=1e6)
    w = SoftBodyWorld(bodies, cfg)
    rng = np.random.default_rng(4)
    us = [rng.normal(0, 5e-4, 3 * b.n_nodes) * (b.pin == 0).repeat(3) for b in bodies]
    w.set_state(np.zeros(sum(u.size for u in us)), np.zeros(sum(u.size for u in us)), 0.0)
    a = w.assemble(np.concatenate(us), t=0.01)
    off = 0
    for e, (b, u) in enumerate(zip(bodies, us)):
        s = oracle.Scene(b, cfg, min_eig=float(np.finfo(np.float32).eps))
        ao = s.assemble(u, np.zeros_like(u), t=0.01)
        g = a["g"][off:off + u.size]
        np.testing.assert_allclose(g, ao["g"], rtol=0, atol=1e-6 * np.abs(ao["g"]).max())
        assert a["obj"][e] == pytest.approx(ao["obj"], rel=1e-6)
        assert a["n_pairs"][e] == ao["n_pairs"]
        off += u.size


@pytest.mark.parametrize("material,psd", [(1, 0), (1, 1), (1, 2), (1, 3), (2, 1), (5, 0), (5, 1), (5, 2)])
def test_other_materials_assembly_matches_oracle(oracle, material, psd):
    """St. Venant-Kirchhoff (every PSD strategy, eigensystem projection on the GPU, 9x9 eigen-solve in the
    oracle), linear elasticity and ARAP (FP64 SVD for energy and stress, twist-mode clamp on the GPU),
    with contact."""
    b = _body(10 + material)
    b.material = material
    cfg = scenes.SceneConfig(k_contact=1e6)
    w, s = _pair(oracle, b, cfg, psd)
    rng = np.random.default_rng(200 + 10 * material + psd)
    free = (b.pin == 0).repeat(3)
    u = rng.normal(0, 1.5e-3, 3 * b.n_nodes) * free
    v = rng.normal(0, 2e-2, 3 * b.n_nodes) * free
    w.set_state(np.zeros_like(u), v, 0.0)
    a_gpu = w.assemble(u, t=0.02, psd=psd != 0)
    a_or = s.assemble(u, cfg.dt * v, t=0.02, psd=psd != 0, pairs=True)
    g_scale = np.abs(a_or["g"]).max()
    np.testing.assert_allclose(a_gpu["g"], a_or["g"], rtol=0, atol=1e-6 * g_scale)
    H_scale = np.abs(a_or["H"]).max()
    np.testing.assert_allclose(a_gpu["H"], a_or["H"], rtol=0, atol=2e-5 * H_scale)
    assert a_gpu["obj"][0] == pytest.approx(a_or["obj"], rel=1e-6)


def test_mass_damping_assembly_matches_oracle(oracle):
    """Rayleigh mass damping about the state's displacement (the stage start) with an StVK body."""
    b = _body(21)
    b.material = 1
    cfg = scenes.SceneConfig(k_contact=1e6, mass_damping=4.0)
    w, s = _pair(oracle, b, cfg, 1)
    rng = np.random.default_rng(321)
    free = (b.pin == 0).repeat(3)
    us = rng.normal(0, 5e-4, 3 * b.n_nodes) * free
    u = us + rng.normal(0, 1e-3, 3 * b.n_nodes) * free
    v = rng.normal(0, 2e-2, 3 * b.n_nodes) * free
    w.set_state(us, v, 0.0)
    a_gpu = w.assemble(u, t=0.01, psd=True)
    a_or = s.assemble(u, us + cfg.dt * v, t=0.01, psd=True, u_stage=us)
    g_scale = np.abs(a_or["g"]).max()
    np.testing.assert_allclose(a_gpu["g"], a_or["g"], rtol=0, atol=1e-6 * g_scale)
    H_scale = np.abs(a_or["H"]).max()
    np.testing.assert_allclose(a_gpu["H"], a_or["H"], rtol=0, atol=2e-5 * H_scale)
    assert a_gpu["obj"][0] == pytest.approx(a_or["obj"], rel=1e-6)


@pytest.mark.parametrize("geometric,psd", [(False, 1), (True, 0), (True, 1)])
def test_stiffness_damping_assembly_matches_oracle(oracle, geometric, psd):
    """Rayleigh stiffness damping (viscous stress about the stage start), with and without its geometric
    Hessian term and its projection."""
    b = _body(31)
    cfg = scenes.SceneConfig(k_contact=1e6, mass_damping=2.0, stiffness_damping=0.01,
                             stiffness_damping_geometric=geometric)
    w, s = _pair(oracle, b, cfg, psd)
    rng = np.random.default_rng(431 + psd)
    free = (b.pin == 0).repeat(3)
    us = rng.normal(0, 5e-4, 3 * b.n_nodes) * free
    u = us + rng.normal(0, 1e-3, 3 * b.n_nodes) * free
    v = rng.normal(0, 2e-2, 3 * b.n_nodes) * free
    w.set_state(us, v, 0.0)
    a_gpu = w.assemble(u, t=0.01, psd=psd != 0)
    a_or = s.assemble(u, us + cfg.dt * v, t=0.01, psd=psd != 0, u_stage=us)
    g_scale = np.abs(a_or["g"]).max()
    np.testing.assert_allclose(a_gpu["g"], a_or["g"], rtol=0, atol=1e-6 * g_scale)
    H_scale = np.abs(a_or["H"]).max()
    np.testing.assert_allclose(a_gpu["H"], a_or["H"], rtol=0, atol=2e-5 * H_scale)
    assert a_gpu["obj"][0] == pytest.approx(a_or["obj"], rel=1e-6)


_FRICTION_CASES = [
    dict(friction_coulomb=0.5),  # the reference's friction defaults: C1, fitted Hessian, fading, collider normal
    dict(friction_coulomb=0.8, friction_model=1, friction_fitted_hessian=False, friction_viscous=0.3,
         contact_normal_damping=0.2),
    dict(friction_coulomb=0.5, contact_explicit_normals=True, friction_fitted_hessian=False,
         contact_normal_damping=0.1),
    dict(friction_coulomb=0.4, friction_viscous=0.2, contact_implicit_normal_force=True,
         friction_collider_normal=False, friction_fade=False),
]


@pytest.mark.parametrize("case", range(len(_FRICTION_CASES)))
def test_friction_assembly_matches_oracle(oracle, case):
    """Contact with Coulomb / viscous friction and normal damping (ComputeBatchCollisionForceDForce):
    capsules pressing and sliding on the top and a plane on the side, the stage start at the state."""
    b = _body(41 + case)
    top = b.X[:, 2].max()
    b.colliders[0] = scenes.capsule((0.012, 0.02, top + 0.0025), (0.032, 0.03, top + 0.0025), 0.004,
                                    (0.08, 0.03, -0.05))
    cfg = scenes.SceneConfig(k_contact=1e9, **_FRICTION_CASES[case])
    w, s = _pair(oracle, b, cfg, 1)
    rng = np.random.default_rng(500 + case)
    free = (b.pin == 0).repeat(3)
    us = rng.normal(0, 3e-4, 3 * b.n_nodes) * free
    u = us + rng.normal(0, 1e-4, 3 * b.n_nodes) * free
    v = rng.normal(0, 2e-2, 3 * b.n_nodes) * free
    w.set_state(us, v, 0.0)
    t = 0.01
    a_gpu = w.assemble(u, t=t, psd=True)
    a_or = s.assemble(u, us + cfg.dt * v, t=t, psd=True, u_stage=us, pairs=True)
    s0 = oracle.Scene(b, scenes.SceneConfig(k_contact=1e9, contact_explicit_normals=cfg.contact_explicit_normals),
                      psd_strategy=1, min_eig=float(np.finfo(np.float32).eps))
    g0 = s0.assemble(u, us + cfg.dt * v, t=t, psd=True, u_stage=us)["g"]
    g_scale = np.abs(a_or["g"]).max()
    assert np.abs(a_or["g"] - g0).max() > 0.005 * g_scale  # the dissipative terms: 5000x the tolerance below
    np.testing.assert_allclose(a_gpu["g"], a_or["g"], rtol=0, atol=1e-6 * g_scale)
    H_scale = np.abs(a_or["H"]).max()
    np.testing.assert_allclose(a_gpu["H"], a_or["H"], rtol=0, atol=2e-5 * H_scale)
    assert a_gpu["obj"][0] == pytest.approx(a_or["obj"], rel=1e-6)
    assert a_gpu["n_pairs"][0] == a_or["n_pairs"] > 0
    assert np.array_equal(w.contact_pairs(), a_or["pairs"])


def test_arap_with_stiffness_damping_and_mixed_envs_matches_oracle(oracle):
    """A batch mixing ARAP and Neo-Hookean envs (the ARAP-capable element kernel), with Rayleigh stiffness
    damping, whose reference stiffness for ARAP is (0, mu / 2)."""
    from project_superdex_b200.soft_body import SoftBodyWorld
    bodies = [_body(60), _body(61, n=4)]
    bodies[0].material = 5
    cfg = scenes.SceneConfig(k_contact=1e6, stiffness_damping=0.01, stiffness_damping_geometric=True)
    w = SoftBodyWorld(bodies, cfg, psd_strategy=1)
    rng = np.random.default_rng(700)
    us_all, u_all, v_all, g_or, obj_or = [], [], [], [], []
    for b in bodies:
        free = (b.pin == 0).repeat(3)
        us = rng.normal(0, 5e-4, 3 * b.n_nodes) * free
        u = us + rng.normal(0, 1e-3, 3 * b.n_nodes) * free
        v = rng.normal(0, 2e-2, 3 * b.n_nodes) * free
        s = oracle.Scene(b, cfg, psd_strategy=1, min_eig=float(np.finfo(np.float32).eps))
        a = s.assemble(u, us + cfg.dt * v, t=0.01, psd=True, u_stage=us)
        us_all.append(us), u_all.append(u), v_all.append(v), g_or.append(a["g"]), obj_or.append(a["obj"])
    w.set_state(np.concatenate(us_all), np.concatenate(v_all), 0.0)
    a_gpu = w.assemble(np.concatenate(u_all), t=0.01, psd=True)
    g = np.concatenate(g_or)
    np.testing.assert_allclose(a_gpu["g"], g, rtol=0, atol=1e-6 * np.abs(g).max())
    np.testing.assert_allclose(a_gpu["obj"], obj_or, rtol=1e-6)
    with pytest.raises(Exception, match="Fast"):
        w.set_params(psd_strategy=3)
