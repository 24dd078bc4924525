"""The assembled Hessian is symmetric (CG needs an SPD operator): elasticity with each PSD strategy, Rayleigh
damping, penalty contact and every friction and normal-damping variant. The two triangles accumulate the
same terms in different orders, so on the GPU they agree to FP32 rounding."""
import numpy as np
import pytest

from project_superdex_b200 import scenes

pytestmark = pytest.mark.gpu


def _body(seed):
    rng = np.random.default_rng(seed)
    b = scenes.grid_body(5, 6, 4, 0.01, rng=rng, E=1e5, nu=0.45)
    b.E = np.exp(rng.uniform(np.log(1e4), np.log(1e6), size=b.n_tets))
    top = 0.03
    b.colliders = [scenes.capsule((0.012, 0.02, top + 0.0025), (0.032, 0.03, top + 0.0025), 0.004, (0.08, 0.03, -0.05)),
                   scenes.plane((1, 0, 0), -0.0008, (0.01, 0, 0))]
    return b


_CASES = [
    dict(psd=0, cfg=dict(k_contact=1e9)),
    dict(psd=1, cfg=dict(k_contact=1e9)),
    dict(psd=2, cfg=dict(k_contact=1e9)),
    dict(psd=3, cfg=dict(k_contact=1e9)),
    dict(psd=1, cfg=dict(k_contact=1e9, mass_damping=2.0, stiffness_damping=0.01)),
    dict(psd=1, cfg=dict(k_contact=1e9, stiffness_damping=0.01, stiffness_damping_geometric=True)),
    dict(psd=1, cfg=dict(k_contact=1e9, friction_coulomb=0.5)),
    dict(psd=1, cfg=dict(k_contact=1e9, friction_coulomb=0.8, friction_model=1, friction_fitted_hessian=False,
                         friction_viscous=0.3, contact_normal_damping=0.2)),
    dict(psd=1, cfg=dict(k_contact=1e9, friction_coulomb=0.5, contact_explicit_normals=True,
                         friction_fitted_hessian=False, contact_normal_damping=0.1)),
    dict(psd=1, cfg=dict(k_contact=1e9, friction_coulomb=0.4, friction_viscous=0.2,
                         contact_implicit_normal_force=True, friction_collider_normal=False, friction_fade=False)),
]


def asymmetry(rp, col, H):
    """max over blocks of |H_ij - H_ji^T| relative to max |H| (user pattern order)."""
    n = rp.size - 1
    rows = np.repeat(np.arange(n), np.diff(rp))
    key = rows.astype(np.int64) * n + col
    tkey = col.astype(np.int64) * n + rows
    order = np.argsort(key)
    pos = order[np.searchsorted(key[order], tkey)]
    assert np.array_equal(key[pos], tkey)  # the pattern is structurally symmetric
    d = np.abs(H - np.transpose(H[pos], (0, 2, 1))).max()
    return d / np.abs(H).max()


@pytest.mark.parametrize("case", range(len(_CASES)))
def test_assembled_hessian_is_symmetric(case):
    from project_superdex_b200.soft_body import SoftBodyWorld
    c = _CASES[case]
    b = _body(70 + case)
    cfg = scenes.SceneConfig(**c["cfg"])
    w = SoftBodyWorld([b], cfg, psd_strategy=c["psd"])
    rng = np.random.default_rng(900 + case)
    free = (b.pin == 0).repeat(3)
    us = rng.normal(0, 3e-4, 3 * b.n_nodes) * free
    u = us + rng.normal(0, 1e-3, 3 * b.n_nodes) * free  # large enough for indefinite tets
    v = rng.normal(0, 2e-2, 3 * b.n_nodes) * free
    w.set_state(us, v, 0.0)
    a = w.assemble(u, t=0.01, psd=True)
    assert a["n_pairs"][0] > 0
    rp, col = w.pattern()
    assert asymmetry(rp, col, a["H"]) <= 1e-5

