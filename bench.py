#!/usr/bin/env python
"""Benchmark of the B200 implicit soft-body step (one JSON line on rank 0).

Workload (default): the single large body with contact — a 64^3-cell tet grid (274,625 nodes,
1,572,864 tets) of heterogeneous stable Neo-Hookean (E log-uniform [1e4, 1e6] Pa, nu = 0.45) pressed
by 5 moving capsules (penalty stiffness 1e4, activation distance 1 mm), backward Euler dt = 1/240,
Newton to rel 1e-6 with Jacobi-PCG at rel. residual 1e-6. A step is one backward-Euler step of every
env of the batch. Inputs (matrix ~160 MB, tet data ~300 MB) exceed the 126 MB L2.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload cfg1|cfg0|cfg2|cfg3|cfg4] [--arms plain_fp64,fused_zero,temporal,learned]

`--workload cfg3` is the learned warm start's own protocol on the batched distribution: the MLP is trained
on plain-solver episodes of 50 seeds (episodes of 16 uneven bodies, cells/axis U{8..40}, 5 capsules and a
ground plane each; Adam, lr 1e-3), then each arm is timed on 20 held-out seeded episodes and the line
aggregates them (env-steps over the summed timed seconds, CG iterations per step).

Four solver arms on the same GPU and the same seeded workload, each a full Newton step:
  plain_fp64  the reference's CUDA PCG path restated (FP64 3x3 BSR with cuSPARSE bsrmv, cuBLAS vector
              operations, CUDA-graph bursts of 8 iterations with a host convergence check, one env after
              the other), zero initial guess;
  fused_zero  this library's persistent batched PCG (FP32 matrix / SpMV, FP64 x, r and reductions),
              zero initial guess (the reference's Newton behaviour);
  temporal    the same, started from the previous step's Newton update at the same Newton iteration
              (energy-optimal scaling; zero when it would raise the residual);
  learned     the same, started by a Galerkin step on span{temporal guess, MLP correction} (per-vertex
              MLP trained first, on the GPU, from plain-solver episodes of held-out seeds).
The headline `value` is the last arm (learned); `arms` gives each and the ratios.

N > 1 runs one independent replica per GPU (the path shards by environment and has no exchange),
launched by torchrun; timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "env-steps/sec at rel-res 1e-6: learned warm-start vs plain PCG; SpMV HBM GB/s"
UNIT = "env-steps/s"


def measured_peaks():
    p = os.path.join(HERE, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(kernel: str):
    """Per-launch DRAM bytes of `kernel` from the committed ncu summary (profiles/traffic.txt)."""
    p = os.path.join(HERE, "profiles", "traffic.txt")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        for line in f:
            parts = line.split()
            if len(parts) >= 2 and parts[0] == kernel:
                try:
                    return float(parts[1])
                except ValueError:
                    return None
    return None


def build_workload(name: str, seed: int = 0):
    from project_superdex_b200 import scenes
    if name == "cfg0":
        return scenes.config0(seed), "single soft cube 10^3 cells (1,331 nodes, 6,000 tets), no contact"
    if name == "cfg1":
        return scenes.config1(seed), ("single body 64^3 cells (274,625 nodes, 1,572,864 tets), E log-uniform "
                                      "[1e4,1e6], nu 0.45, 5 capsules r=4mm L=20mm at 0.05 m/s, k=1e4")
    if name == "cfg4":
        return scenes.config4(seed), ("stiff heterogeneous body 96^3 cells (912,673 nodes, 5,308,416 tets), nu 0.49, "
                                      "E log-uniform [1e4,1e7] with 10 inclusions x100, 2 closing planes + 5 capsules")
    if name == "cfg3":
        n = int(os.environ.get("SDX_CFG3_ENVS", "16"))
        return scenes.config2(seed, n_envs=n), (f"learned warm start on the batched distribution: an episode is {n} "
                                                "uneven bodies, cells/axis U{8..40}, 5 capsules + plane each")
    if name == "cfg2":
        n = int(os.environ.get("SDX_CFG2_ENVS", "1024"))
        return scenes.config2(seed, n_envs=n), f"{n} uneven bodies, cells/axis U{{8..40}}, 5 capsules + plane each"
    raise ValueError(name)


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}
        if not self.path or not os.path.exists(self.path):
            return out
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                cols = [c.strip() for c in line.split(",")]
                if len(cols) < 9:
                    continue
                try:
                    sm.append(float(cols[1]))
                    mx.append(float(cols[2]))
                except ValueError:
                    continue
                for nme, v in zip(names, cols[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(nme)
        os.unlink(self.path)
        if sm:
            out["sm_mhz"] = statistics.median(sm)
            out["sm_max_mhz"] = max(mx)
        out["reasons"] = sorted(reasons)
        out["samples"] = len(sm)
        return out


def cpu_oracle_sample(workload: str, seed: int = 0, steps: int = 1, warmup: int = 0):
    """The CPU restatement of the reference path (oracle/) on a bounded sample: env 0 of the workload from
    rest, `warmup` untimed backward-Euler steps, then `steps` timed steps continuing the trajectory, all
    host threads."""
    from oracle import oracle as O
    (bodies, cfg), _ = build_workload(workload, seed)
    b = bodies[0]
    s = O.Scene(b, cfg)
    u = np.zeros(3 * b.n_nodes)
    v = np.zeros_like(u)
    prm = O.default_newton_params()
    prm.abs_tol = 1e-9  # same Newton stopping test as the GPU arm: rel 1e-6
    if workload in ("cfg2", "cfg3"):
        prm.max_iter = 12  # same Newton cap as the GPU arm
    t = 0.0
    for _ in range(warmup):
        t += cfg.dt
        u, v, st = s.step(u, v, t, prm)
    newton = cg = 0
    t0 = time.perf_counter()
    for _ in range(steps):
        t += cfg.dt
        u, v, st = s.step(u, v, t, prm)
        newton += st.newton_iters
        cg += st.cg_iters
    dt = time.perf_counter() - t0
    return {"value": steps / dt, "unit": UNIT, "cores": int(O.lib().or_num_threads()), "kind": "port",
            "sample": (f"env 0 of {workload}: {warmup} untimed + {steps} timed backward-Euler steps from rest "
                       f"({newton} Newton, {cg} CG iterations timed) in {dt:.2f} s")}


def vector_bytes_per_node():
    # algorithmic bytes per node per CG iteration of the fused PCG besides the matrix:
    # phase 1: z own 12 + z gather 12 + p r/w 24 + q r/w 24; phase 2: x r/w 48 (FP64),
    # r r/w 48 (FP64), p 12, q 12, dinv 12, z r/w 24
    return 12 + 12 + 24 + 24 + 48 + 48 + 12 + 12 + 12 + 24


def newton_max_iter(args):
    """Newton iteration cap: 50 by default; 12 for the batched workload, where 1-2 % of the envs stall
    between relative residual 1e-5 and 1e-3 on the penalty contact's non-smooth activation (the FP64 CPU
    oracle stalls at the same residuals), and would otherwise run every step to the cap."""
    if args.newton_max_iter:
        return args.newton_max_iter
    return 12 if args.workload in ("cfg2", "cfg3") else 50


def train_warm_start(args, local_rank):
    """Train the warm-start MLP on the GPU from plain-solver episodes of held-out seeds of the same
    workload (never the evaluated seed). Returns (params, info)."""
    from project_superdex_b200.learned import Mlp, collect
    from project_superdex_b200.soft_body import SoftBodyWorld
    t0 = time.perf_counter()
    Xs, Ts = [], []
    # the training set is capped at train_samples vertices, spread evenly over the episodes (cfg3's 50
    # episodes take a few thousand vertices from each Newton solve; cfg1's two take the first 1 M each)
    cap = max(4096, args.train_samples // args.train_episodes)
    per_solve = 65536 if args.workload != "cfg3" else max(1024, min(65536, cap // (4 * args.train_steps)))
    for k in range(args.train_episodes):
        (bodies, cfg), _ = build_workload(args.workload, seed=args.seed + 1000 + k)
        tw = SoftBodyWorld(bodies, cfg, device=local_rank, newton_abs_tol=1e-9,
                           newton_max_iter=newton_max_iter(args))
        X, T = collect(tw, args.train_steps, samples_per_solve=per_solve, capacity=cap, seed=k)
        Xs.append(X)
        Ts.append(T)
        if k < args.train_episodes - 1:
            tw.close()
    X, T = np.concatenate(Xs), np.concatenate(Ts)
    m = Mlp(tw._ctx)
    m.init(args.seed)
    losses = m.train(X, T, batch=4096, epochs=args.train_epochs, lr=1e-3, seed=args.seed)
    params = m.get_params()
    tw.close()
    return params, {"episodes": args.train_episodes, "steps_per_episode": args.train_steps,
                    "samples": int(X.shape[0]), "epochs": args.train_epochs, "loss_first": float(losses[0]),
                    "loss_last": float(losses[-1]), "seconds": time.perf_counter() - t0,
                    "seeds": f"{args.seed + 1000}..{args.seed + 999 + args.train_episodes} (held out)"}


def time_arm(w, args, stream, local_rank, dist, world):
    """W untimed steps, then exactly K steps between CUDA events on the library stream."""
    import torch
    w.step(args.warmup)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    launches0 = w.kernel_launches()
    w.set_profiling(True)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        torch.cuda.synchronize()
        ev0.record(stream)
        w.step(args.steps)
        ev1.record(stream)
        ev1.synchronize()
    ms = ev0.elapsed_time(ev1)
    prof = w.profile()
    w.set_profiling(False)
    launches = w.kernel_launches() - launches0
    stats = w.stats()
    if dist:
        t = torch.tensor([ms], device=f"cuda:{local_rank}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    n_envs = w.n_envs
    # over the K timed steps: one PCG launch per Newton iteration (all envs together), and per launch the
    # iterations of its slowest env
    return {"value": world * n_envs * args.steps / (ms / 1000.0), "ms": ms, "prof": prof, "launches": launches,
            "clocks": clk.summary(), "env_steps": world * n_envs * args.steps, "steps": args.steps,
            "cg_iters_per_step": prof["pcg_iters"] / args.steps,
            "newton_iters_per_step": prof["pcg_launches"] / args.steps,
            "last_step_cg_iters_mean_env": [sum(s["cg_iters"] for s in stats) / max(1, n_envs)]}


def merge_runs(a, b):
    """One arm timed on several episodes: sums of env-steps, time, launches and the solver profile."""
    out = dict(b)
    out["env_steps"] = a["env_steps"] + b["env_steps"]
    out["steps"] = a["steps"] + b["steps"]
    out["ms"] = a["ms"] + b["ms"]
    out["launches"] = a["launches"] + b["launches"]
    out["last_step_cg_iters_mean_env"] = a["last_step_cg_iters_mean_env"] + b["last_step_cg_iters_mean_env"]
    out["value"] = out["env_steps"] / (out["ms"] / 1000.0)
    out["prof"] = {k: (a["prof"].get(k, 0) + v if k != "pcg_threads" else v) for k, v in b["prof"].items()}
    out["cg_iters_per_step"] = out["prof"]["pcg_iters"] / out["steps"]
    out["newton_iters_per_step"] = out["prof"]["pcg_launches"] / out["steps"]
    ca, cb = a["clocks"], b["clocks"]
    sm = [x for x in (ca.get("sm_mhz"), cb.get("sm_mhz")) if x is not None]
    out["clocks"] = {"sm_mhz": statistics.median(sm) if sm else None,
                     "sm_max_mhz": max([x for x in (ca.get("sm_max_mhz"), cb.get("sm_max_mhz")) if x is not None],
                                       default=None),
                     "reasons": sorted(set(ca.get("reasons", [])) | set(cb.get("reasons", []))),
                     "samples": ca.get("samples", 0) + cb.get("samples", 0)}
    return out


def run_ours(args, rank, world, local_rank):
    # the PCG launch shape is picked by the library's autotuner on each world's first Newton solve
    os.environ.setdefault("SDX_PCG_AUTOTUNE", "1")
    import torch
    from project_superdex_b200 import capi
    from project_superdex_b200.learned import Mlp
    from project_superdex_b200.soft_body import SoftBodyWorld
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
    arms = [a for a in args.arms.split(",") if a]
    params, train_info = (None, None)
    if "learned" in arms:
        params, train_info = train_warm_start(args, local_rank)
    # cfg3: every arm on each held-out episode (seeds args.seed.., training used args.seed + 1000..)
    seeds = [args.seed + i for i in range(args.eval_episodes)] if args.workload == "cfg3" else [args.seed]
    results = {}
    w = None
    for seed in seeds:
        (bodies, cfg), desc = build_workload(args.workload, seed=seed)
        for arm in arms:
            if w is not None:
                w.close()
            # Newton to rel 1e-6 (the absolute floor is only a guard for an exactly zero residual)
            w = SoftBodyWorld(bodies, cfg, device=local_rank, newton_abs_tol=1e-9,
                              newton_max_iter=newton_max_iter(args))
            if arm == "learned":
                Mlp(w._ctx).set_params(params)
            w.set_params(warm_start={"learned": capi.SDX_WARM_LEARNED, "temporal": capi.SDX_WARM_TEMPORAL}.get(
                             arm, capi.SDX_WARM_ZERO))
            if arm == "plain_fp64":  # the comparison solver, plugged into the Newton solves (bench_arms/)
                from bench_arms.plain import PlainFp64
                w._plain = PlainFp64(w)
            stream = torch.cuda.ExternalStream(w.stream_handle(), device=local_rank)
            r = time_arm(w, args, stream, local_rank, dist, world)
            results[arm] = merge_runs(results[arm], r) if arm in results else r
    head = results[arms[-1]]  # the headline arm is the last one (learned by default); w is its world
    n_envs = w.n_envs
    ms, prof = head["ms"], head["prof"]

    # roofline of the dominant kernel (the persistent PCG)
    peak, peak_kind = measured_peaks()
    # algorithmic bytes: per env, its CG iterations x (40 B per block + 4 B per row pointer + 228 B per
    # row), summed by the library over the timed launches (envs of a batch converge at different counts)
    bytes_iter = w.nnzb * 40 + 4 * (w.n_nodes + 1) + vector_bytes_per_node() * w.n_nodes
    pcg_s = prof["pcg_ms"] / 1000.0
    achieved = prof["pcg_bytes"] / pcg_s / 1e9 if pcg_s > 0 else None
    traffic = ncu_traffic("k_pcg_per_iter") if args.workload == "cfg1" else None
    pcg_kernel = ("k_pcg (persistent Jacobi-PCG) and k_pcg_cluster (one cluster per env), every PCG solve"
                  if prof.get("pcg_cluster_solves", 0) else "k_pcg (persistent Jacobi-PCG)")
    roofline = {"bound": "hbm", "kernel": pcg_kernel, "achieved": achieved,
                "peak": peak, "unit": "GB/s", "frac": (achieved / peak) if achieved else None,
                "peak_source": peak_kind, "traffic": traffic, "bytes_per_iter": bytes_iter,
                "iters": prof["pcg_iters"], "share_of_step": prof["pcg_ms"] / ms}
    # standalone SpMV on the last assembled matrix
    spmv_ms, spmv_bytes = w.bench_spmv(reps=20)
    spmv = {"achieved_gbs": spmv_bytes / (spmv_ms / 1000.0) / 1e9, "ms": spmv_ms, "bytes": spmv_bytes}
    spmv["frac"] = spmv["achieved_gbs"] / peak

    # end to end through the public API with pinned host buffers, copies inside the timed region
    stream = torch.cuda.ExternalStream(w.stream_handle(), device=local_rank)
    hu = torch.empty(3 * w.n_nodes, dtype=torch.float64, pin_memory=True).numpy()
    hv = torch.empty(3 * w.n_nodes, dtype=torch.float64, pin_memory=True).numpy()
    _, _, t_state = w.get_state(hu, hv)
    e2e_steps = max(1, min(args.steps, 5))
    w.set_profiling(True)  # same per-kernel event overhead as the timed arms; gives the e2e solver counts
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e2e_steps):
        w.set_state(hu, hv, t_state)
        w.step(1)
        _, _, t_state = w.get_state(hu, hv)
    e1.record(stream)
    e1.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    eprof = w.profile()
    w.set_profiling(False)
    if dist:
        t = torch.tensor([e2e_ms], device=f"cuda:{local_rank}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e = {"value": world * n_envs * e2e_steps / (e2e_ms / 1000.0), "unit": UNIT,
           "h2d_bytes_per_step": 2 * 3 * 8 * w.n_nodes, "d2h_bytes_per_step": 2 * 3 * 8 * w.n_nodes,
           "steps": e2e_steps, "warm_start": arms[-1],
           "note": "the steps after the timed ones, continuing the trajectory",
           "cg_iters_per_step": eprof["pcg_iters"] / e2e_steps,
           "newton_iters_per_step": eprof["pcg_launches"] / e2e_steps}
    arm_summary = {a: {"value": r["value"], "ms_per_step": r["ms"] / r["steps"],
                       "cg_iters_per_step": r["cg_iters_per_step"],
                       "newton_iters_per_step": r["newton_iters_per_step"],
                       # each env's own CG iterations in the last timed step (a launch runs until its
                       # slowest env converges; cg_iters_per_step counts those launch-level iterations)
                       "cg_iters_per_env_last_step": float(np.mean(r["last_step_cg_iters_mean_env"]))}
                   for a, r in results.items()}
    for base in ("plain_fp64", "fused_zero", "temporal"):
        if base in results and "learned" in results:
            arm_summary[f"learned_over_{base}"] = results["learned"]["value"] / results[base]["value"]
            arm_summary[f"cg_iters_learned_over_{base}"] = (results["learned"]["cg_iters_per_step"]
                                                            / results[base]["cg_iters_per_step"])
    reasons = sorted(set().union(*[set(r["clocks"].get("reasons", [])) for r in results.values()]))
    clocks = dict(head["clocks"])
    clocks["reasons_all_arms"] = reasons
    line = {
        "metric": METRIC, "value": head["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / head["steps"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
        "data": "synthetic (seeded tet grids, random materials and collider trajectories)",
        "config": {"workload": f"{args.workload}: {desc}", "n_envs": n_envs, "n_nodes": w.n_nodes,
                   "n_tets": w.n_tets, "nnzb": w.nnzb,
                   "precision": "FP32 Hessian assembly + SpMV, FP64 residual / energy / CG dots / x,r",
                   "warm_start": arms[-1], "arms": arms,
                   "cg_rel_tol": 1e-6, "newton_rel_tol": 1e-6, "newton_abs_tol": 1e-9,
                   "newton_max_iter": newton_max_iter(args),
                   "l2": "inputs larger than L2 (matrix + tet data > 126 MB)",
                   "pcg_threads_autotuned": int(prof.get("pcg_threads", 0)),
                   "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
                   "episodes": len(seeds), "seeds": f"{seeds[0]}..{seeds[-1]}"},
        "arms": arm_summary, "training": train_info,
        "roofline": roofline, "spmv": spmv, "e2e": e2e, "gpu_launches": head["launches"],
        "clocks": clocks,
        "solver": {"cg_iters_per_step": head["cg_iters_per_step"],
                   "newton_iters_per_step": head["newton_iters_per_step"],
                   "pcg_cluster_solves": int(prof.get("pcg_cluster_solves", 0)),
                   "profile_ms": {k: v for k, v in prof.items() if k.endswith("_ms")}},
    }
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_oracle_sample(args.workload, args.seed)
    w.close()
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="cfg1", choices=["cfg0", "cfg1", "cfg2", "cfg3", "cfg4"])
    ap.add_argument("--arms", default=None,
                    help="comma list of solver arms to time, headline last: plain_fp64 (the reference's CUDA "
                         "PCG path restated: FP64 BSR, cuSPARSE/cuBLAS, zero start), fused_zero (this "
                         "library's PCG, zero start), temporal (start from the previous step's update at the "
                         "same Newton iteration), learned (temporal guess + learned correction, Galerkin); "
                         "default plain_fp64,fused_zero,temporal,learned (cfg3: fused_zero,temporal,learned)")
    ap.add_argument("--train-episodes", type=int, default=None, dest="train_episodes",
                    help="plain-solver training episodes (default 2; cfg3: 50)")
    ap.add_argument("--train-steps", type=int, default=None, dest="train_steps",
                    help="steps per training episode (default 8; cfg3: 2)")
    ap.add_argument("--train-epochs", type=int, default=8, dest="train_epochs")
    ap.add_argument("--train-samples", type=int, default=1 << 21, dest="train_samples",
                    help="training vertices kept over all episodes")
    ap.add_argument("--eval-episodes", type=int, default=20, dest="eval_episodes",
                    help="cfg3: held-out episodes each arm is timed on")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--newton-max-iter", type=int, default=0, dest="newton_max_iter")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    cfg3 = args.workload == "cfg3"
    if args.arms is None:
        args.arms = "fused_zero,temporal,learned" if cfg3 else "plain_fp64,fused_zero,temporal,learned"
    if args.train_episodes is None:
        args.train_episodes = 50 if cfg3 else 2
    if args.train_steps is None:
        args.train_steps = 2 if cfg3 else 8
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        # The reference's own implementation of this path is CPU code; its timed stand-in is the CPU
        # restatement in oracle/ (the reference's full step needs its cmake build). Rank 0 only.
        if rank != 0:
            return 0
        cb = cpu_oracle_sample(args.workload, args.seed, steps=args.steps, warmup=args.warmup)
        _, desc = build_workload(args.workload, seed=args.seed)
        line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 / cb["value"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded tet grids, random materials and collider trajectories)",
                "config": {"workload": f"{args.workload}: {desc}", "sample": "env 0",
                           "newton_max_iter": newton_max_iter(args)},
                "cpu_baseline": cb,
                "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return 0

    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    line = run_ours(args, rank, world, local_rank)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
