"""Host-side logic of bench.py that needs no GPU: the workloads it builds, the config dict both arms print,
the CPU baseline's bounded sample and how one arm's runs over several evaluation episodes are combined
(the learned warm start's protocol on the batched distribution times each arm on 20 held-out episodes)."""
import argparse

import bench


def _run(env_steps, steps, ms, iters, launches, sm_mhz, reasons, conv):
    return {"ms": ms, "e2e_ms": 1.1 * ms, "env_steps": env_steps, "steps": steps, "launches": launches,
            "step_ms": [ms / steps] * steps, "converged_env_steps": conv,
            "prof": {"pcg_ms": 0.9 * ms, "pcg_iters": iters, "pcg_launches": 4 * steps,
                     "pcg_bytes": 1e9 * iters, "pcg_threads": 512},
            "clocks": {"sm_mhz": sm_mhz, "sm_max_mhz": 1965.0, "reasons": reasons, "samples": 10},
            "newton_per_env_step": 4.0, "cg_per_env_step": iters / env_steps}


def test_merge_aggregates_episodes():
    a = _run(160, 10, 1000.0, 3000, 500, 1965.0, [], 150)
    b = _run(160, 10, 3000.0, 5000, 700, 1900.0, ["sw_power_cap"], 160)
    m = bench.merge(a, b)
    assert m["env_steps"] == 320 and m["steps"] == 20 and m["ms"] == 4000.0 and m["launches"] == 1200
    assert m["e2e_ms"] == 1.1 * 4000.0 and m["converged_env_steps"] == 310 and len(m["step_ms"]) == 20
    assert m["prof"]["pcg_iters"] == 8000 and m["prof"]["pcg_bytes"] == 8e12
    assert m["prof"]["pcg_threads"] == 512  # a launch shape, not a sum
    assert m["cg_per_env_step"] == 8000 / 320 and m["newton_per_env_step"] == 4.0
    assert m["clocks"]["reasons"] == ["sw_power_cap"] and m["clocks"]["samples"] == 20


def test_batched_workloads_and_newton_caps(monkeypatch):
    monkeypatch.setenv("SDX_CFG3_ENVS", "3")
    (bodies, cfg), desc = bench.build_workload("cfg3", seed=5)
    assert len(bodies) == 3 and "3 uneven bodies" in desc
    (bodies2, _), _ = bench.build_workload("cfg3", seed=5)
    assert [b.n_nodes for b in bodies] == [b.n_nodes for b in bodies2]  # seeded
    (held_out, _), _ = bench.build_workload("cfg3", seed=bench.TRAIN_SEED0 + 5)
    assert [b.n_nodes for b in held_out] != [b.n_nodes for b in bodies]

    class A:
        newton_max_iter = 0
        workload = "cfg3"
    assert bench.newton_max_iter(A) == 12
    A.workload = "cfg1"
    assert bench.newton_max_iter(A) == 50


def test_both_arms_print_the_same_config(monkeypatch):
    """--impl reference and ours build `config` from the workload alone."""
    monkeypatch.setenv("SDX_CFG2_ENVS", "4")
    args = argparse.Namespace(workload="cfg2", newton_max_iter=0, steps=20, warmup=5)
    (bodies, _), desc = bench.build_workload("cfg2", seed=0)
    c1 = bench.workload_config(args, 0, bodies, desc, 1)
    (bodies2, _), desc2 = bench.build_workload("cfg2", seed=0)
    c2 = bench.workload_config(args, 0, bodies2, desc2, 1)
    assert c1 == c2 and c1["n_envs"] == 4 and c1["n_tets"] == sum(b.n_tets for b in bodies)


def test_cpu_sample_is_bounded(monkeypatch):
    monkeypatch.setenv("SDX_CFG2_ENVS", "64")
    (bodies, _), _ = bench.build_workload("cfg2", seed=0)
    idx = bench.sample_envs(bodies, 400000)
    assert idx == list(range(len(idx))) and len(idx) >= 1
    assert sum(bodies[i].n_tets for i in idx) <= 400000 or len(idx) == 1
    assert bench.sample_envs(bodies, 1) == [0]


def test_pcg_time_split_by_kernel_and_shape_keys():
    """The bench line's PCG split: the cluster kernel's share of the time and bytes, the grid kernel the rest;
    launch-shape entries of the profile are kept, not summed, across merged runs."""
    prof = {"pcg_ms": 1000.0, "pcg_bytes": 4.0e12, "pcg_cluster_ms": 800.0, "pcg_cluster_bytes": 3.6e12}
    sp = bench.pcg_split(prof)
    assert sp["cluster"]["ms"] == 800.0 and abs(sp["cluster"]["gbs"] - 4500.0) < 1e-9
    assert sp["grid"]["ms"] == 200.0 and abs(sp["grid"]["gbs"] - 2000.0) < 1e-9
    assert bench.pcg_split({"pcg_ms": 0.0, "pcg_bytes": 0.0})["grid"]["gbs"] is None
    a = _run(160, 10, 1000.0, 3000, 500, 1965.0, [], 150)
    b = _run(160, 10, 3000.0, 5000, 700, 1900.0, [], 160)
    for r in (a, b):
        r["prof"].update(elem_threads=64, tune_elem_us=19.5, pcg_cluster_ms=100.0)
    m = bench.merge(a, b)
    assert m["prof"]["elem_threads"] == 64 and m["prof"]["tune_elem_us"] == 19.5
    assert m["prof"]["pcg_cluster_ms"] == 200.0


def test_refined_arm_names_set_the_start_and_the_refinement():
    """`<arm>_refined` selects the same warm start with mixed-precision iterative refinement (inner relative
    tolerance bench.REFINE_INNER_REL_TOL); the plain names turn refinement off."""
    from project_superdex_b200 import capi

    class FakeWorld:
        def __init__(self):
            self.calls = []

        def set_params(self, **kw):
            self.calls.append(kw)

    w = FakeWorld()
    for arm in ("fused_zero_refined", "temporal_refined", "temporal", "fused_zero"):
        bench.set_arm(w, arm, None)
    want = [(capi.SDX_WARM_ZERO, bench.REFINE_INNER_REL_TOL), (capi.SDX_WARM_TEMPORAL, bench.REFINE_INNER_REL_TOL),
            (capi.SDX_WARM_TEMPORAL, 0.0), (capi.SDX_WARM_ZERO, 0.0)]
    assert [(c["warm_start"], c["linear_refine_inner_rel_tol"]) for c in w.calls] == want
