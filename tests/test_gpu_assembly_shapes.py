"""Assembly launch shapes: every element-kernel CTA size (64, 128, 256) with the plain and the warp-aggregated
block scatter, and every contact-kernel CTA size, assemble what the oracle assembles; the assembly tuner
(SDX_AUTOTUNE=1) picks one of them on the first Newton pass and the steps still match the oracle."""
import numpy as np
import pytest

from project_superdex_b200 import scenes

pytestmark = pytest.mark.gpu

_SHAPE_VARS = ("SDX_ELEM_THREADS", "SDX_ELEM_RES_THREADS", "SDX_CONTACT_THREADS", "SDX_ELEM_AGG")


def _bodies():
    """Three uneven bodies with contact: warps of the element kernel straddle env boundaries."""
    out = []
    for i, (nx, ny, nz) in enumerate(((5, 6, 4), (3, 4, 5), (6, 5, 5))):
        rng = np.random.default_rng(40 + i)
        b = scenes.grid_body(nx, ny, nz, 0.01, rng=rng, nu=0.45)
        b.E = np.exp(rng.uniform(np.log(1e4), np.log(1e6), size=b.n_tets))
        top = nz * 0.01
        b.colliders = [scenes.capsule((0.012, 0.015, top + 0.0032), (0.03, 0.025, top + 0.0032), 0.004, (0, 0, -0.05)),
                       scenes.plane((1, 0, 0), -0.0008, (0.01, 0, 0))]
        out.append(b)
    return out


@pytest.mark.parametrize("threads", [64, 128, 256])
@pytest.mark.parametrize("agg", [0, 1])
def test_assembly_shapes_match_oracle(oracle, monkeypatch, threads, agg):
    from project_superdex_b200.soft_body import SoftBodyWorld
    for k, v in zip(_SHAPE_VARS, (threads, threads, threads, agg)):
        monkeypatch.setenv(k, str(v))
    bodies = _bodies()
    cfg = scenes.SceneConfig(k_contact=1e6)
    w = SoftBodyWorld(bodies, cfg, psd_strategy=1)
    rng = np.random.default_rng(7)
    us = [rng.normal(0, 1.5e-3, 3 * b.n_nodes) * (b.pin == 0).repeat(3) for b in bodies]
    t = 0.02
    w.set_state(None, None, 0.0)
    a = w.assemble(np.concatenate(us), t=t)
    rp, col = w.pattern()
    off_n, off_b = 0, 0
    for e, b in enumerate(bodies):
        s = oracle.Scene(b, cfg, psd_strategy=1, min_eig=float(np.finfo(np.float32).eps))
        o = s.assemble(us[e], np.zeros_like(us[e]), t=t, psd=True, pairs=True)
        nb = s.row_ptr[-1]
        g = a["g"][3 * off_n:3 * (off_n + b.n_nodes)]
        H = a["H"][off_b:off_b + nb]
        assert np.array_equal(rp[off_n:off_n + b.n_nodes + 1] - rp[off_n], s.row_ptr)
        assert np.array_equal(col[off_b:off_b + nb] - off_n, s.col)
        np.testing.assert_allclose(g, o["g"], rtol=0, atol=1e-6 * np.abs(o["g"]).max())
        np.testing.assert_allclose(H, o["H"], rtol=0, atol=2e-5 * np.abs(o["H"]).max())
        assert a["obj"][e] == pytest.approx(o["obj"], rel=1e-6)
        assert a["n_pairs"][e] == o["n_pairs"]
        off_n += b.n_nodes
        off_b += nb


def test_aggregated_scatter_equals_plain_scatter_to_rounding(monkeypatch):
    """The warp-aggregated scatter only regroups the FP32 additions into each block: same matrix to FP32
    rounding of the sums, identical residual (its scatter is not aggregated)."""
    from project_superdex_b200.soft_body import SoftBodyWorld
    bodies = _bodies()
    cfg = scenes.SceneConfig(k_contact=1e6)
    w = SoftBodyWorld(bodies, cfg, psd_strategy=1)
    rng = np.random.default_rng(8)
    u = np.concatenate([rng.normal(0, 1e-3, 3 * b.n_nodes) * (b.pin == 0).repeat(3) for b in bodies])
    out = []
    for agg in (0, 1):
        monkeypatch.setenv("SDX_ELEM_AGG", str(agg))
        out.append(w.assemble(u, t=0.01))
    h0, h1 = out[0]["H"], out[1]["H"]
    assert np.abs(h1 - h0).max() <= 1e-6 * np.abs(h0).max()
    np.testing.assert_allclose(out[1]["g"], out[0]["g"], rtol=0, atol=1e-12 * np.abs(out[0]["g"]).max())


def test_assembly_tuner_picks_a_shape_and_steps_match_oracle(oracle, monkeypatch):
    import test_gpu_step as ts
    for k in _SHAPE_VARS:
        monkeypatch.delenv(k, raising=False)
    monkeypatch.setenv("SDX_AUTOTUNE", "1")
    bodies = _bodies()
    cfg = scenes.SceneConfig(k_contact=1e6)
    w, ug, vg, states, hist = ts._run(oracle, bodies, cfg, 2)
    w.set_profiling(True)
    p = w.profile()
    assert p["elem_threads"] in (64, 128, 256) and p["elem_res_threads"] in (64, 128, 256)
    assert p["contact_threads"] in (64, 128, 256) and p["elem_aggregated"] in (0, 1)
    assert 0.0 < p["tune_elem_us"] <= p["tune_elem_default_us"]
    ts._check(bodies, ug, states, hist, newton_exact=False)
