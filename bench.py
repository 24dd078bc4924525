#!/usr/bin/env python
"""Benchmark of the B200 implicit soft-body step (one JSON line on rank 0).

Workload (default, cfg2): 1,024 independent soft bodies of uneven size in one batch — tet boxes with
cells per axis U{8..40} (seed 0: 16,189,547 nodes, 86,022,012 tets), stable Neo-Hookean with E in
[1e4, 1e6] Pa and nu in [0.3, 0.48] per body, each pressed by 5 capsule fingertips onto a ground plane
(penalty contact); backward Euler dt = 1/240, Newton to rel 1e-6 (capped at 12 iterations) with
Jacobi-PCG at rel. residual 1e-6. A step is one backward-Euler step of every env of the batch. The working
set (~10 GB) is far larger than the 126 MB L2.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload cfg2|cfg1|cfg0|cfg3|cfg4] [--arms fused_zero,temporal,learned]

Solver arms, on the same GPU, the same workload and the same steps (each restored from one snapshot taken
after the W warm-up steps):
  plain_fp64  the reference's CUDA PCG path restated (bench_arms/libsdx_plain_fp64.so: FP64 3x3 BSR with
              cuSPARSE bsrmv, cuBLAS vector operations, graph bursts of 8 iterations with a host convergence
              check, one env after the other), zero initial guess; single-body workloads only (minutes per
              step on the batch);
  fused_zero  this library's persistent batched PCG (FP32 matrix / SpMV, FP64 x, r and reductions), zero
              initial guess: the plain PCG start of the reference's Newton loop;
  temporal    the same, started from the previous step's Newton update at the same Newton iteration;
  learned     the headline: the same, started by a Galerkin step on span{temporal guess, MLP correction}.
              The per-vertex MLP is trained first, on the GPU, on the learned part's own protocol: (state,
              RHS, solution) triples of the plain solver on 50 held-out seeded episodes of 16 bodies of the
              same distribution (seeds 1000..1049, run as one batch of 800 bodies, 2 steps), Adam lr 1e-3.
  <arm>_refined  any of the above with mixed-precision iterative refinement: PCG passes to relative 1e-2 of
              each pass's right-hand side, corrected against the FP64 residual until rel 1e-6 (the default
              arms of the stiff cfg4 case: plain_fp64, fused_zero, learned_refined).
The headline arm is timed on K steps through the public API (sdx_set_state / sdx_step / sdx_get_state with
pinned host buffers): `value` is the device time of the steps (CUDA events on the library stream around
each sdx_step), `e2e` the whole loop with the host<->device copies, on the same steps. The comparison arms
are timed on the first min(K, --compare-steps) of those steps, and the ratios use the headline arm's time on
the same steps.

`--workload cfg3` times each arm on 20 held-out seeded episodes of 16 bodies (the learned part's evaluation
protocol); cfg1 is the single 64^3 body with 5 capsules, cfg0 the 10^3 soft cube, cfg4 the 96^3 stiff body.

N > 1 runs one independent replica per GPU (the path shards by environment and has no exchange; each rank
its own seeded batch), launched by torchrun; timing is the max over ranks.
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

# profile entries that describe launch shapes (kept, not summed, when runs are merged)
SHAPE_KEYS = ("pcg_threads", "pcg_cluster_size", "tune_grid_us", "tune_cluster_us", "elem_threads",
              "elem_res_threads", "elem_aggregated", "contact_threads", "tune_elem_us", "tune_elem_default_us")
METRIC = "env-steps/sec at rel-res 1e-6: learned warm-start vs plain PCG; SpMV HBM GB/s"
UNIT = "env-steps/s"
TRAIN_SEED0 = 1000  # training episodes use seeds TRAIN_SEED0.. (never an evaluated seed)


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


def newton_max_iter(args):
    """Newton iteration cap: 50 by default; 12 for the batched workloads, where 1-2 % of the envs stall
    between relative residual 1e-5 and 1e-3 on the penalty contact's non-smooth activation (the FP64 CPU
    oracle stalls at the same residuals), and would otherwise run every step to the cap. The line reports
    the share of env-steps that reached rel 1e-6."""
    if args.newton_max_iter:
        return args.newton_max_iter
    return 12 if args.workload in ("cfg2", "cfg3") else 50


def workload_config(args, seed: int, bodies, desc: str, world: int):
    """The `config` dict both arms (ours and --impl reference) print: the workload itself."""
    n_nodes = int(sum(b.n_nodes for b in bodies))
    n_tets = int(sum(b.n_tets for b in bodies))
    return {"workload": f"{args.workload}: {desc}", "seed": seed, "n_envs": len(bodies), "n_nodes": n_nodes,
            "n_tets": n_tets, "precision": "FP32 Hessian assembly + SpMV, FP64 residual / energy / CG dots / x,r",
            "cg_rel_tol": 1e-6, "newton_rel_tol": 1e-6, "newton_max_iter": newton_max_iter(args),
            "steps_per_measurement": args.steps, "warmup_steps": args.warmup,
            "l2": "inputs larger than L2 (matrix + tet data > 126 MB)",
            "parallelism": f"replicas x{world} (one seeded batch per GPU)" if world > 1 else "1 GPU"}


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


# ------------------------------------------------------------------------------------------------
# the CPU baseline (the oracle: the reference's path restated in C, all host threads)

def sample_envs(bodies, tet_budget: int):
    """The first envs of the batch whose tets sum to at most tet_budget (at least one)."""
    idx, tot = [], 0
    for i, b in enumerate(bodies):
        if idx and tot + b.n_tets > tet_budget:
            break
        idx.append(i)
        tot += b.n_tets
    return idx


def cpu_oracle_run(args, seed: int, steps: int, warmup: int, tet_budget: int):
    """The CPU restatement of the reference path on a bounded sample: the first envs of the workload (up to
    tet_budget tets), each stepped from rest for `warmup` untimed and `steps` timed backward-Euler steps
    with all host threads, the envs one after the other (the reference steps independent islands as
    parallel tasks; here the threads go to each env's assembly and CG). Returns env-steps/s over the
    sample's timed steps."""
    from oracle import oracle as O
    (bodies, cfg), _ = build_workload(args.workload, seed)
    envs = sample_envs(bodies, tet_budget)
    prm = O.default_newton_params()
    prm.abs_tol = 1e-9  # same Newton stopping test as the GPU arm: rel 1e-6
    prm.max_iter = newton_max_iter(args)
    states = []
    for e in envs:
        s = O.Scene(bodies[e], cfg)
        u = np.zeros(3 * bodies[e].n_nodes)
        states.append([s, u, np.zeros_like(u), 0.0])
    for _ in range(warmup):
        for st in states:
            st[3] += cfg.dt
            st[1], st[2], _ = st[0].step(st[1], st[2], st[3], prm)
    newton = cg = 0
    t0 = time.perf_counter()
    for _ in range(steps):
        for st in states:
            st[3] += cfg.dt
            st[1], st[2], r = st[0].step(st[1], st[2], st[3], prm)
            newton += r.newton_iters
            cg += r.cg_iters
    dt = time.perf_counter() - t0
    tets = sum(bodies[e].n_tets for e in envs)
    return {"value": len(envs) * steps / dt, "unit": UNIT, "cores": int(O.lib().or_num_threads()), "kind": "port",
            "sample": (f"envs {envs[0]}..{envs[-1]} of {args.workload} seed {seed} ({len(envs)} of {len(bodies)} "
                       f"envs, {tets} tets): {warmup} untimed + {steps} timed backward-Euler steps from rest, "
                       f"{newton} Newton / {cg} CG iterations timed, {dt:.2f} s")}


def reference_pcg_sample(args, seed: int):
    """One Newton system solved three ways: env 0's first system of a step from rest (assembled by the CPU
    oracle) by the reference's own compiled krylov::PCG on its BlockSparseMatrix<double,3> with
    BlockJacobiPrec (oracle/_ref, built from the reference's sources; single-threaded, its serial
    scheduler), by the oracle's PCG (all host threads), and by this library's sdx_pcg_solve through the
    C-ABI (host arrays in and out, the matrix in the reference's row-strip layout). Jacobi, rel 1e-6.
    None when oracle/_ref was not built."""
    from oracle import oracle as O
    if O.ref() is None:
        return None
    import ctypes as C
    from project_superdex_b200 import capi
    from project_superdex_b200.linear_solver import blocks_to_strips
    (bodies, cfg), _ = build_workload(args.workload, seed)
    b0 = bodies[0]
    sc = O.Scene(b0, cfg)
    u = np.zeros(3 * b0.n_nodes)
    a = sc.assemble(u, u, t=cfg.dt, obj=False, psd=True)
    rp, col, H, g = sc.row_ptr, sc.col, a["H"], a["g"]
    strips = blocks_to_strips(rp, H)
    out = {"system": f"env 0 of {args.workload} seed {seed}: first Newton system of a step from rest "
                     f"({3 * b0.n_nodes} DoF, {int(rp[-1])} blocks), Jacobi, rel 1e-6"}
    t0 = time.perf_counter()
    _, it_ref, _, rel_ref, _ = O.ref_bsr3_pcg(rp, col, strips, g, rel_tol=1e-6, abs_tol=1e-9, precond=1)
    out["reference_krylov_pcg"] = {"ms": 1e3 * (time.perf_counter() - t0), "iters": int(it_ref),
                                   "rel_res": float(rel_ref), "threads": 1}
    t0 = time.perf_counter()
    _, st = O.pcg(rp, col, H, g, rel_tol=1e-6, abs_tol=1e-9)
    out["oracle_pcg"] = {"ms": 1e3 * (time.perf_counter() - t0), "iters": int(st.num_iter),
                         "threads": int(O.lib().or_num_threads())}
    lp = capi.default_linear_params()
    lp.rel_tol, lp.abs_tol = 1e-6, 1e-9
    x = np.zeros_like(g)
    sst = capi.LinearStatus()
    rp64 = np.ascontiguousarray(rp, np.int64)
    cl = np.ascontiguousarray(col, np.int32)
    vals = np.ascontiguousarray(strips, np.float64)
    args_c = (rp64.size - 1, cl.size, capi.ptr(rp64, capi._lp), capi.ptr(cl, capi._ip),
              vals.ctypes.data_as(C.c_void_p), capi.SDX_F64, capi.ptr(np.ascontiguousarray(g)), capi.ptr(x),
              capi.SDX_GUESS_ZERO, C.byref(lp), C.byref(sst))
    capi.check(capi.lib().sdx_pcg_solve(*args_c))  # first call: device set-up
    t0 = time.perf_counter()
    capi.check(capi.lib().sdx_pcg_solve(*args_c))
    out["sdx_pcg_solve"] = {"ms": 1e3 * (time.perf_counter() - t0), "iters": int(sst.num_iter),
                            "note": "one call through the C-ABI: upload, FP32 conversion, solve, download"}
    return out


# ------------------------------------------------------------------------------------------------
# training of the learned warm start (the learned part's own protocol)

def train_warm_start(args, local_rank):
    """Train the warm-start MLP on the GPU from plain-solver (zero start) episodes of held-out seeds of the
    batched distribution: `train_episodes` episodes of 16 bodies (seeds TRAIN_SEED0..), run together as one
    batch, `train_steps` steps, up to `train_samples` (features, solution) vertex samples; Adam lr 1e-3.
    Returns (params, info)."""
    from project_superdex_b200 import scenes
    from project_superdex_b200.learned import Mlp, collect
    from project_superdex_b200.soft_body import SoftBodyWorld
    t0 = time.perf_counter()
    if args.workload in ("cfg2", "cfg3"):
        bodies = []
        for k in range(args.train_episodes):
            bodies += scenes.config2(TRAIN_SEED0 + k, n_envs=16)[0]
        cfg = scenes.config2(TRAIN_SEED0, n_envs=1)[1]
        groups = [bodies]
        per_solve_div = 4 * args.train_steps
    else:  # single-body workloads: episodes of the same body with held-out seeds
        groups = []
        for k in range(args.train_episodes):
            (bb, cfg), _ = build_workload(args.workload, seed=TRAIN_SEED0 + k)
            groups.append(bb)
        per_solve_div = 4 * args.train_steps * args.train_episodes
    Xs, Ts = [], []
    cap = args.train_samples // len(groups)
    per_solve = max(1024, min(1 << 20, cap // per_solve_div))
    tw = None
    for k, bodies in enumerate(groups):
        if tw is not None:
            tw.close()
        tw = SoftBodyWorld(bodies, cfg, device=local_rank, newton_abs_tol=1e-9, newton_max_iter=newton_max_iter(args))
        X, T = collect(tw, args.train_steps, samples_per_solve=per_solve, capacity=cap, seed=k)
        Xs.append(X)
        Ts.append(T)
    t_data = time.perf_counter() - t0
    X, T = np.concatenate(Xs), np.concatenate(Ts)
    m = Mlp(tw._ctx)
    m.init(args.seed)
    losses = m.train(X, T, batch=4096, epochs=args.train_epochs, lr=1e-3, seed=args.seed)
    params = m.get_params()
    tw.close()
    return params, {"episodes": args.train_episodes, "steps_per_episode": args.train_steps,
                    "bodies_per_episode": 16 if args.workload in ("cfg2", "cfg3") else 1,
                    "samples": int(X.shape[0]), "epochs": args.train_epochs, "lr": 1e-3,
                    "loss_first": float(losses[0]), "loss_last": float(losses[-1]),
                    "data_seconds": t_data, "seconds": time.perf_counter() - t0,
                    "seeds": f"{TRAIN_SEED0}..{TRAIN_SEED0 + args.train_episodes - 1} (held out)"}


# ------------------------------------------------------------------------------------------------
# timing

def _events(n):
    import torch
    return [torch.cuda.Event(enable_timing=True) for _ in range(n)]


def time_headline(w, args, stream, local_rank):
    """K steps through the public API with pinned host buffers: per step sdx_set_state (host -> device),
    sdx_step, sdx_get_state (device -> host). Device time of each sdx_step from CUDA events on the library
    stream; the e2e time covers the whole loop, copies included. Per-step env convergence is read from the
    statistics after each step."""
    import torch
    K = args.steps
    hu = torch.empty(3 * w.n_nodes, dtype=torch.float64, pin_memory=True).numpy()
    hv = torch.empty(3 * w.n_nodes, dtype=torch.float64, pin_memory=True).numpy()
    _, _, t_state = w.get_state(hu, hv)
    ev_a, ev_b, ev_c = _events(K), _events(K), _events(K)
    ev_end = _events(1)[0]
    launches0 = w.kernel_launches()
    w.set_profiling(True)
    conv_steps = 0
    newton = cg_env = 0
    torch.cuda.synchronize()
    # the timed steps are the only region a profiler started with --profile-from-start off records
    torch.cuda.profiler.start()
    with ClockSampler(local_rank) as clk:
        for k in range(K):
            ev_a[k].record(stream)
            w.set_state(hu, hv, t_state)
            ev_b[k].record(stream)
            w.step(1)
            ev_c[k].record(stream)
            _, _, t_state = w.get_state(hu, hv)
            st = w.stats()
            conv_steps += sum(1 for s in st if s["convergence"] == 1)
            newton += sum(s["newton_iters"] for s in st)
            cg_env += sum(s["cg_iters"] for s in st)
        ev_end.record(stream)
        ev_end.synchronize()
    torch.cuda.profiler.stop()
    step_ms = [ev_b[k].elapsed_time(ev_c[k]) for k in range(K)]
    e2e_ms = ev_a[0].elapsed_time(ev_end)
    prof = w.profile()
    w.set_profiling(False)
    n = w.n_envs
    return {"step_ms": step_ms, "ms": sum(step_ms), "e2e_ms": e2e_ms, "prof": prof,
            "launches": w.kernel_launches() - launches0, "clocks": clk.summary(), "env_steps": n * K,
            "steps": K, "converged_env_steps": conv_steps, "newton_per_env_step": newton / (n * K),
            "cg_per_env_step": cg_env / (n * K), "h2d_bytes_per_step": 2 * 3 * 8 * w.n_nodes,
            "d2h_bytes_per_step": 2 * 3 * 8 * w.n_nodes}


def time_steps(w, n_steps, stream):
    """n_steps of sdx_step, each between CUDA events on the library stream (inputs resident)."""
    import torch
    ev0, ev1 = _events(n_steps), _events(n_steps)
    w.set_profiling(True)
    newton = cg_env = conv = 0
    torch.cuda.synchronize()
    for k in range(n_steps):
        ev0[k].record(stream)
        w.step(1)
        ev1[k].record(stream)
        st = w.stats()
        conv += sum(1 for s in st if s["convergence"] == 1)
        newton += sum(s["newton_iters"] for s in st)
        cg_env += sum(s["cg_iters"] for s in st)
    ev1[-1].synchronize()
    prof = w.profile()
    w.set_profiling(False)
    step_ms = [ev0[k].elapsed_time(ev1[k]) for k in range(n_steps)]
    n = w.n_envs
    return {"step_ms": step_ms, "ms": sum(step_ms), "prof": prof, "env_steps": n * n_steps, "steps": n_steps,
            "converged_env_steps": conv, "newton_per_env_step": newton / (n * n_steps),
            "cg_per_env_step": cg_env / (n * n_steps)}


def max_over_ranks(x, dist, local_rank):
    if not dist:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{local_rank}")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# inner relative tolerance of the arms with mixed-precision iterative refinement ("<start>_refined")
REFINE_INNER_REL_TOL = 1e-2


def pcg_split(prof):
    """Algorithmic GB/s of the PCG solves by kernel: the cluster kernel (long queues of envs) and the grid
    kernel (the rest)."""
    out = {}
    cm, cb = prof.get("pcg_cluster_ms", 0.0), prof.get("pcg_cluster_bytes", 0.0)
    gm, gb = prof.get("pcg_ms", 0.0) - cm, prof.get("pcg_bytes", 0.0) - cb
    for name, ms, by in (("cluster", cm, cb), ("grid", gm, gb)):
        out[name] = {"ms": ms, "gbs": by / (ms * 1e-3) / 1e9 if ms > 0 else None}
    return out


def set_arm(w, arm, params):
    from project_superdex_b200 import capi
    from project_superdex_b200.learned import Mlp
    refined = arm.endswith("_refined")
    arm = arm[:-len("_refined")] if refined else arm
    if arm == "learned":
        Mlp(w._ctx).set_params(params)
    w.set_params(warm_start={"learned": capi.SDX_WARM_LEARNED, "temporal": capi.SDX_WARM_TEMPORAL}.get(
        arm, capi.SDX_WARM_ZERO), linear_refine_inner_rel_tol=REFINE_INNER_REL_TOL if refined else 0.0)
    if getattr(w, "_plain", None) is not None:
        w._plain.close()
        w._plain = None
    if arm == "plain_fp64":  # the comparison solver, plugged into the Newton solves (bench_arms/)
        from bench_arms.plain import PlainFp64
        w._plain = PlainFp64(w)


def parity_env0(args, bodies, cfg, states_gpu, stats_gpu):
    """Env 0 of the headline workload: the GPU state after each of the first steps from rest against the
    FP64 CPU oracle (the reference's path restated) stepped the same way."""
    from oracle import oracle as O
    b = bodies[0]
    # the PSD projection's eigenvalue floor at the GPU's FP32 tangent precision
    s = O.Scene(b, cfg, min_eig=float(np.finfo(np.float32).eps))
    prm = O.default_newton_params()
    prm.abs_tol = 1e-9
    prm.max_iter = newton_max_iter(args)
    u = np.zeros(3 * b.n_nodes)
    v = np.zeros_like(u)
    size = float(np.ptp(b.X, axis=0).max())
    out = {"env": 0, "n_nodes": int(b.n_nodes), "n_tets": int(b.n_tets), "body_size_m": size, "steps": []}
    t0 = time.perf_counter()
    for k, (ug, sg) in enumerate(zip(states_gpu, stats_gpu)):
        u, v, st = s.step(u, v, (k + 1) * cfg.dt, prm)
        err = float(np.abs(ug - u).max())
        out["steps"].append({"max_abs_err_m": err, "err_over_body_size": err / size,
                             "newton_gpu": sg["newton_iters"], "newton_oracle": int(st.newton_iters),
                             "cg_gpu": sg["cg_iters"], "cg_oracle": int(st.cg_iters),
                             "converged_gpu": sg["convergence"] == 1, "converged_oracle": int(st.convergence) == 1})
    out["max_err_over_body_size"] = max(x["err_over_body_size"] for x in out["steps"])
    out["tolerance"] = 1e-5
    out["ok"] = out["max_err_over_body_size"] <= 1e-5
    out["oracle_seconds"] = time.perf_counter() - t0
    out["reference"] = "FP64 CPU oracle (oracle/sdx_oracle.c, pinned to the reference's compiled code)"
    return out


def merge(a, b):
    """One arm timed on several episodes: sums of env-steps, time, launches and the solver profile."""
    out = dict(b)
    for k in ("env_steps", "steps", "ms", "e2e_ms", "launches", "converged_env_steps"):
        if k in a:
            out[k] = a[k] + b[k]
    out["step_ms"] = a["step_ms"] + b["step_ms"]
    for k in ("newton_per_env_step", "cg_per_env_step"):
        out[k] = (a[k] * a["env_steps"] + b[k] * b["env_steps"]) / out["env_steps"]
    out["prof"] = {k: (a["prof"].get(k, 0) + v if k not in SHAPE_KEYS else v) for k, v in b["prof"].items()}
    if "clocks" in a:
        ca, cb = a["clocks"], b["clocks"]
        sm = [x for x in (ca.get("sm_mhz"), cb.get("sm_mhz")) if x is not None]
        out["clocks"] = {"sm_mhz": statistics.median(sm) if sm else None,
                         "sm_max_mhz": max([x for x in (ca.get("sm_max_mhz"), cb.get("sm_max_mhz")) if x is not None],
                                           default=None),
                         "reasons": sorted(set(ca.get("reasons", [])) | set(cb.get("reasons", []))),
                         "samples": ca.get("samples", 0) + cb.get("samples", 0)}
    return out


def run_ours(args, rank, world, local_rank):
    # the PCG and assembly launch shapes are picked by the library's autotuners on the world's first Newton
    # pass
    os.environ.setdefault("SDX_AUTOTUNE", "1")
    import torch
    from project_superdex_b200.replicas import replica_seed
    from project_superdex_b200.soft_body import SoftBodyWorld
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
    arms = [a for a in args.arms.split(",") if a]
    head_arm = arms[-1]
    params, train_info = (None, None)
    if any(a.startswith("learned") for a in arms):
        params, train_info = train_warm_start(args, local_rank)
    seed0 = replica_seed(args.seed, rank)
    seeds = [seed0 + i for i in range(args.eval_episodes)] if args.workload == "cfg3" else [seed0]
    n_cmp = min(args.steps, args.compare_steps)
    head = None
    comp = {a: None for a in arms[:-1]}
    head_first = 0.0  # the headline arm's device time on the comparison steps
    parity = None
    w = None
    for ei, seed in enumerate(seeds):
        (bodies, cfg), desc = build_workload(args.workload, seed=seed)
        if ei == 0:
            config = workload_config(args, seed, bodies, desc, world)
        if w is not None:
            w.close()
        # Newton to rel 1e-6 (the absolute floor is only a guard for an exactly zero residual)
        w = SoftBodyWorld(bodies, cfg, device=local_rank, newton_abs_tol=1e-9, newton_max_iter=newton_max_iter(args))
        stream = torch.cuda.ExternalStream(w.stream_handle(), device=local_rank)
        set_arm(w, head_arm, params)
        # warm-up from rest with the headline arm; env 0's first two states for the parity check
        par_u, par_st = [], []
        for k in range(args.warmup):
            w.step(1)
            if ei == 0 and k < 2 and rank == 0:
                u, _, _ = w.get_state()
                par_u.append(u[:3 * bodies[0].n_nodes].copy())
                par_st.append(w.stats()[0])
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        snap = w.capture_state()
        r = time_headline(w, args, stream, local_rank)
        head = r if head is None else merge(head, r)
        head_first += sum(r["step_ms"][:n_cmp])
        for a in arms[:-1]:
            w.restore_state(snap)
            set_arm(w, a, params)
            rc = time_steps(w, n_cmp, stream)
            comp[a] = rc if comp[a] is None else merge(comp[a], rc)
        set_arm(w, head_arm, params)
        w.release_all_states()
        if ei == 0 and par_u and not args.no_parity:
            parity = parity_env0(args, bodies, cfg, par_u, par_st)
    ms = max_over_ranks(head["ms"], dist, local_rank)
    e2e_ms = max_over_ranks(head["e2e_ms"], dist, local_rank)
    prof = head["prof"]
    value = world * head["env_steps"] / (ms / 1000.0)

    # roofline of the dominant kernel (the persistent PCG): algorithmic bytes per env per CG iteration
    # (40 B per block + 4 B per row pointer + 228 B per row, 156 with r and x carried in FP32) x that env's
    # iterations, summed by the library
    # over the timed launches, over the PCG launches' CUDA-event time
    peak, peak_kind = measured_peaks()
    pcg_s = prof["pcg_ms"] / 1000.0
    achieved = prof["pcg_bytes"] / pcg_s / 1e9 if pcg_s > 0 else None
    frac = (achieved / peak) if achieved else None
    frac_note = None
    if frac is not None and frac > 1.2:
        # above the copy bandwidth: the vectors were L2-resident (small envs) or the byte count is stale
        frac_note = f"frac {frac:.2f} > 1.2 rejected: the PCG ran from L2, HBM is not its bound here"
        frac = None
    traffic = ncu_traffic(f"k_pcg_per_iter_{args.workload}")
    if traffic is None and args.workload == "cfg1":
        traffic = ncu_traffic("k_pcg_per_iter")
    pcg_kernel = ("k_pcg (persistent Jacobi-PCG) and k_pcg_cluster (one cluster per env), every PCG solve"
                  if prof.get("pcg_cluster_solves", 0) else "k_pcg (persistent Jacobi-PCG)")
    roofline = {"bound": "hbm", "kernel": pcg_kernel, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": frac, "peak_source": peak_kind, "traffic": traffic,
                "traffic_unit": "DRAM bytes per CG iteration of the batch (ncu, profiles/traffic.txt)",
                "algorithmic_bytes": prof["pcg_bytes"], "launch_iters": prof["pcg_iters"],
                "share_of_step": prof["pcg_ms"] / head["ms"]}
    if frac_note:
        roofline["note"] = frac_note
    spmv_ms, spmv_bytes = w.bench_spmv(reps=20)
    spmv = {"achieved_gbs": spmv_bytes / (spmv_ms / 1000.0) / 1e9, "ms": spmv_ms, "bytes": spmv_bytes}
    spmv["frac"] = spmv["achieved_gbs"] / peak
    e2e = {"value": world * head["env_steps"] / (e2e_ms / 1000.0), "unit": UNIT,
           "h2d_bytes_per_step": head["h2d_bytes_per_step"], "d2h_bytes_per_step": head["d2h_bytes_per_step"],
           "steps": head["steps"], "warm_start": head_arm,
           "note": ("the same steps as value, through sdx_set_state / sdx_step / sdx_get_state with pinned host "
                    "buffers (u and v both ways every step)")}
    arm_summary = {head_arm: {"value": value, "ms_per_step": ms / head["steps"],
                              "newton_iters_per_env_step": head["newton_per_env_step"],
                              "cg_iters_per_env_step": head["cg_per_env_step"],
                              "converged_frac": head["converged_env_steps"] / head["env_steps"]}}
    for a, rc in comp.items():
        v_a = world * rc["env_steps"] / (rc["ms"] / 1000.0)
        v_h = world * rc["env_steps"] / (head_first / 1000.0)
        arm_summary[a] = {"value": v_a, "ms_per_step": rc["ms"] / rc["steps"], "steps": rc["steps"],
                          "newton_iters_per_env_step": rc["newton_per_env_step"],
                          "cg_iters_per_env_step": rc["cg_per_env_step"],
                          "converged_frac": rc["converged_env_steps"] / rc["env_steps"]}
        # the headline arm's env-steps/s on the same steps (its first n_cmp timed steps) over this arm's
        arm_summary[f"{head_arm}_over_{a}"] = v_h / v_a
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / head["steps"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
        "data": "synthetic (seeded tet grids, random materials and collider trajectories)",
        "config": config,
        "run": {"arms": arms, "headline_arm": head_arm, "compare_steps": n_cmp, "episodes": len(seeds),
                "seeds": f"{seeds[0]}..{seeds[-1]}", "nnzb": w.nnzb,
                "pcg_threads_autotuned": int(prof.get("pcg_threads", 0)),
                "pcg_cluster_size_autotuned": int(prof.get("pcg_cluster_size", 0)),
                "autotune_us": {"grid": prof.get("tune_grid_us", 0.0), "cluster": prof.get("tune_cluster_us", 0.0),
                                "element_hessian": prof.get("tune_elem_us", 0.0),
                                "element_hessian_default_shape": prof.get("tune_elem_default_us", 0.0)},
                "assembly_shapes_autotuned": {"element_threads": int(prof.get("elem_threads", 0)),
                                              "element_aggregated_scatter": bool(prof.get("elem_aggregated", 0)),
                                              "element_residual_threads": int(prof.get("elem_res_threads", 0)),
                                              "contact_threads": int(prof.get("contact_threads", 0))}},
        "converged": {"env_steps": head["converged_env_steps"], "of": head["env_steps"],
                      "frac": head["converged_env_steps"] / head["env_steps"],
                      "note": ("value counts every env-step; an env-step that hit the Newton cap before rel 1e-6 "
                               "is counted too (the CPU oracle stalls on the same envs)")},
        "arms": arm_summary, "training": train_info,
        "roofline": roofline, "spmv": spmv, "e2e": e2e, "gpu_launches": head["launches"],
        "clocks": head["clocks"], "parity": parity,
        "solver": {"newton_iters_per_env_step": head["newton_per_env_step"],
                   "cg_iters_per_env_step": head["cg_per_env_step"],
                   "pcg_launch_iters": prof["pcg_iters"], "pcg_launches": prof["pcg_launches"],
                   "pcg_cluster_solves": int(prof.get("pcg_cluster_solves", 0)),
                   "profile_ms": {k: v for k, v in prof.items() if k.endswith("_ms")},
                   "pcg_gbs_by_kernel": pcg_split(prof)},
    }
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_oracle_run(args, seed0, steps=3, warmup=0, tet_budget=args.cpu_tets)
        pcg_one = reference_pcg_sample(args, seed0)
        if pcg_one:
            line["cpu_baseline"]["one_linear_solve"] = pcg_one
    w.close()
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="cfg2", choices=["cfg0", "cfg1", "cfg2", "cfg3", "cfg4"])
    ap.add_argument("--arms", default=None,
                    help="comma list of solver arms, headline last: plain_fp64, fused_zero, temporal, learned "
                         "(default fused_zero,temporal,learned; single-body workloads add plain_fp64 first)")
    ap.add_argument("--compare-steps", type=int, default=5, dest="compare_steps",
                    help="steps each comparison arm is timed on (the first of the headline's timed steps)")
    ap.add_argument("--train-episodes", type=int, default=None, dest="train_episodes",
                    help="training episodes (default 50 of 16 bodies on the batched workloads; 2 otherwise)")
    ap.add_argument("--train-steps", type=int, default=None, dest="train_steps",
                    help="steps per training episode (default 2; single-body workloads 8)")
    ap.add_argument("--train-epochs", type=int, default=8, dest="train_epochs")
    ap.add_argument("--train-samples", type=int, default=1 << 21, dest="train_samples",
                    help="training vertices kept over all episodes")
    ap.add_argument("--eval-episodes", type=int, default=20, dest="eval_episodes",
                    help="cfg3: held-out episodes each arm is timed on")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--newton-max-iter", type=int, default=0, dest="newton_max_iter")
    ap.add_argument("--cpu-tets", type=int, default=1000000, dest="cpu_tets",
                    help="tets of the envs the CPU baseline steps per step (a bounded sample)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-parity", action="store_true")
    args = ap.parse_args()
    batched = args.workload in ("cfg2", "cfg3")
    if args.arms is None:
        if batched:
            args.arms = "fused_zero,temporal,learned"
        elif args.workload == "cfg4":  # the stiff case compares the refined learned-start solver with plain FP64
            args.arms = "plain_fp64,fused_zero,learned_refined"
        else:
            args.arms = "plain_fp64,fused_zero,temporal,learned"
    if args.train_episodes is None:
        args.train_episodes = 50 if batched else 2
    if args.train_steps is None:
        args.train_steps = 2 if batched else 8
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        # The reference's own implementation of this path is CPU code; its timed stand-in is the CPU
        # restatement in oracle/ (the reference's scene-level step needs its cmake build). Rank 0 only.
        if rank != 0:
            return 0
        from project_superdex_b200.replicas import replica_seed
        seed0 = replica_seed(args.seed, 0)
        (bodies, _), desc = build_workload(args.workload, seed=seed0)
        cb = cpu_oracle_run(args, seed0, steps=args.steps, warmup=args.warmup, tet_budget=args.cpu_tets)
        line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 / cb["value"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded tet grids, random materials and collider trajectories)",
                "config": workload_config(args, seed0, bodies, desc, args.gpus),
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
