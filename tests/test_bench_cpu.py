"""Host-side logic of bench.py that needs no GPU: the workloads it builds and how one arm's runs over
several evaluation episodes are combined (the learned warm start's protocol on the batched
distribution times each arm on 20 held-out episodes and reports the aggregate)."""
import bench


def _run(env_steps, steps, ms, iters, launches, sm_mhz, reasons):
    return {"value": env_steps / (ms / 1000.0), "ms": ms, "env_steps": env_steps, "steps": steps,
            "launches": launches, "prof": {"pcg_ms": 0.9 * ms, "pcg_iters": iters, "pcg_launches": 4 * steps,
                                           "pcg_bytes": 1e9 * iters, "pcg_threads": 512},
            "clocks": {"sm_mhz": sm_mhz, "sm_max_mhz": 1965.0, "reasons": reasons, "samples": 10},
            "cg_iters_per_step": iters / steps, "newton_iters_per_step": 4.0,
            "last_step_cg_iters_mean_env": [iters / steps / 16]}


def test_merge_runs_aggregates_episodes():
    a = _run(160, 10, 1000.0, 3000, 500, 1965.0, [])
    b = _run(160, 10, 3000.0, 5000, 700, 1900.0, ["sw_power_cap"])
    m = bench.merge_runs(a, b)
    assert m["env_steps"] == 320 and m["steps"] == 20 and m["ms"] == 4000.0 and m["launches"] == 1200
    assert m["value"] == 320 / 4.0  # env-steps over the summed timed seconds, not a mean of rates
    assert m["prof"]["pcg_iters"] == 8000 and m["prof"]["pcg_bytes"] == 8e12
    assert m["prof"]["pcg_threads"] == 512  # a launch shape, not a sum
    assert m["cg_iters_per_step"] == 400.0 and m["newton_iters_per_step"] == 4.0
    assert m["clocks"]["reasons"] == ["sw_power_cap"] and m["clocks"]["samples"] == 20
    assert m["last_step_cg_iters_mean_env"] == a["last_step_cg_iters_mean_env"] + b["last_step_cg_iters_mean_env"]


def test_batched_workloads_and_newton_caps(monkeypatch):
    monkeypatch.setenv("SDX_CFG3_ENVS", "3")
    (bodies, cfg), desc = bench.build_workload("cfg3", seed=5)
    assert len(bodies) == 3 and "3 uneven bodies" in desc
    (bodies2, _), _ = bench.build_workload("cfg3", seed=5)
    assert [b.n_nodes for b in bodies] == [b.n_nodes for b in bodies2]  # seeded
    (held_out, _), _ = bench.build_workload("cfg3", seed=1005)
    assert [b.n_nodes for b in held_out] != [b.n_nodes for b in bodies]

    class A:
        newton_max_iter = 0
        workload = "cfg3"
    assert bench.newton_max_iter(A) == 12
    A.workload = "cfg1"
    assert bench.newton_max_iter(A) == 50
