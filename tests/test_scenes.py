"""Synthetic scene generator: sizes of the measured configurations, orientation, pins, determinism."""
import numpy as np

from project_superdex_b200 import scenes


def _volumes(b):
    D = np.stack([b.X[b.tets[:, k]] - b.X[b.tets[:, 0]] for k in (1, 2, 3)], axis=2)
    return np.linalg.det(D) / 6.0


def test_config0_sizes_and_orientation():
    (bodies, cfg) = scenes.config0()
    b = bodies[0]
    assert (b.n_nodes, b.n_tets) == (1331, 6000)
    v = _volumes(b)
    assert v.min() > 0 and abs(v.sum() - 0.1 ** 3) < 1e-12
    assert (b.pin == 7).sum() == 121  # bottom face (11 x 11 nodes)
    assert cfg.dt == 1.0 / 240.0 and cfg.steps == 100


def test_config1_sizes():
    (bodies, cfg) = scenes.config1()
    b = bodies[0]
    assert (b.n_nodes, b.n_tets) == (274625, 1572864)
    assert len(b.colliders) == 5 and all(c.type == scenes.COLLIDER_CAPSULE for c in b.colliders)
    assert 1e4 <= b.E.min() and b.E.max() <= 1e6
    assert cfg.k_contact == 1e4 and cfg.thr == 0.001 and cfg.steps == 200
    for c in b.colliders:
        assert abs(np.linalg.norm(c.vel) - 0.05) < 1e-12 and c.radius == 0.004
        assert abs(np.linalg.norm(c.p[3:] - c.p[:3]) - 0.02) < 1e-12


def test_jitter_keeps_boundary_and_is_seeded():
    a = scenes.grid_body(5, 4, 3, 0.01, rng=np.random.default_rng(3))
    b = scenes.grid_body(5, 4, 3, 0.01, rng=np.random.default_rng(3))
    assert np.array_equal(a.X, b.X) and np.array_equal(a.tets, b.tets)
    on_bnd = (np.isclose(a.X[:, 0], 0) | np.isclose(a.X[:, 0], 0.05) | np.isclose(a.X[:, 2], 0))
    assert on_bnd.sum() > 0
    assert _volumes(a).min() > 0


def test_config2_distribution_small():
    bodies, cfg = scenes.config2(seed=1, n_envs=6)
    assert len(bodies) == 6
    for b in bodies:
        nx, ny, nz = b.cells
        assert 8 <= nx <= 40 and 8 <= ny <= 40 and 8 <= nz <= 40
        assert b.n_tets == 6 * nx * ny * nz
        assert len(b.colliders) == 6 and b.colliders[0].type == scenes.COLLIDER_PLANE
        assert 0.3 <= b.nu[0] <= 0.48 and 1e4 <= b.E[0] <= 1e6
    node_off, tet_off, X, tets = scenes.concat_bodies(bodies)
    for e in range(6):
        t = tets[tet_off[e]:tet_off[e + 1]]
        assert t.min() >= node_off[e] and t.max() < node_off[e + 1]
