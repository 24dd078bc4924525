"""The plain FP64 comparison solver (bench_arms/libsdx_plain_fp64.so: the reference's CUDA PCG path, FP64
BSR with cuSPARSE, cuBLAS vector operations, bursts of 8 iterations), plugged into sdx_step through the
external linear-solver hook, reaches the CPU oracle's Newton states like the library's own solver does;
its CG counts are the oracle's rounded up to the burst length."""
import numpy as np
import pytest

from project_superdex_b200 import scenes
from test_gpu_step import _run

pytestmark = pytest.mark.gpu


def _check_plain(bodies, ug, states, hist):
    off = 0
    for e, b in enumerate(bodies):
        size = np.ptp(b.X, axis=0).max()
        err = np.abs(ug[off:off + 3 * b.n_nodes] - states[e][0]).max()
        assert err <= 1e-5 * size, (e, err)
        off += 3 * b.n_nodes
    for st_gpu, st_or in hist:
        for g, o in zip(st_gpu, st_or):
            assert g["convergence"] == o.convergence
            assert abs(g["cg_iters"] - o.cg_iters) <= 8 * g["newton_iters"] + int(0.1 * o.cg_iters), \
                (g["cg_iters"], o.cg_iters)


def _plain(world):
    from bench_arms.plain import PlainFp64
    return PlainFp64(world)


def test_plain_fp64_steps_match_oracle(oracle):
    bodies, cfg = scenes.config0()
    w, ug, vg, states, hist = _run(oracle, bodies, cfg, 3, setup=_plain)
    _check_plain(bodies, ug, states, hist)


def test_plain_fp64_batched_envs_match_oracle(oracle):
    bodies = []
    for i, n in enumerate((3, 5, 4)):
        rng = np.random.default_rng(20 + i)
        b = scenes.grid_body(n, n, n, 0.01, rng=rng, E=float(rng.uniform(3e4, 3e5)), nu=0.4)
        b.colliders = [scenes.capsule((0.01, 0.01, n * 0.01 + 0.0035), (0.02, 0.02, n * 0.01 + 0.0035), 0.004,
                                      (0, 0, -0.1))]
        bodies.append(b)
    cfg = scenes.SceneConfig(k_contact=1e6)
    w, ug, vg, states, hist = _run(oracle, bodies, cfg, 3, setup=_plain)
    _check_plain(bodies, ug, states, hist)
