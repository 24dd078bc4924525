"""Fixed-length launches of the hot kernels, sized for profiler captures.

    python -m project_superdex_b200.kernel_cases pcg --iters 100
        one backward-Euler step limited to one Newton iteration whose persistent PCG launch runs exactly
        `iters` CG iterations (the tolerance is unreachable), after one untimed warm-up step;
    python -m project_superdex_b200.kernel_cases element
        one full assembly (energy, residual, PSD-projected Hessian) of the current state;
    python -m project_superdex_b200.kernel_cases spmv --reps 3
        `reps` standalone SpMVs of the last assembled matrix;
    python -m project_superdex_b200.kernel_cases mlp --rows 274656 --reps 3
        `reps` tensor-core forwards of the warm-start MLP (random weights) over `rows` feature rows.

The workload is the single-body 64^3-cell grid (274,625 nodes, 1,572,864 tets, 5 capsules) unless
`--cells` says otherwise; `--workload batch` takes the 1,024 uneven bodies (cells per axis U{8..40},
16.2 M nodes, 86 M tets) instead, whose device footprint (~25 GB) is too large for multi-pass profiler
captures: use its CUDA-event timing (`us_per_iter`), or `--envs N` for the first N bodies of the batch
(128: about 3 GB). One JSON line reports the sizes and the algorithmic bytes of one launch (or one
CG iteration), so that DRAM counters from a capture divide into per-unit traffic. Only the measured
launches run between cudaProfilerStart and cudaProfilerStop (capture with `ncu --profile-from-start off`).
"""
from __future__ import annotations

import argparse
import json
import os

from . import scenes
from .soft_body import SoftBodyWorld


def pcg_bytes_per_iter(nnzb: int, n_rows: int, r_in_z: bool) -> int:
    """Algorithmic HBM bytes of one fused Jacobi-PCG iteration: the matrix once (36 B values + 4 B column
    per 3x3 block), the slice pointers, and per row the vector traffic: 228 B with FP64 r (phase 1: own z
    12 + gathered z 12 + p and q read/write 48; phase 2: FP64 x and r read/write 96, p 12, q 12, Jacobi
    diagonal 12, z read/write 24); r carried by z and x by its FP32 increment save 48 + 24. The library
    adds up the same figure per env (sdx_profile.pcg_bytes)."""
    return nnzb * 40 + 4 * (n_rows + 1) + (228 - 72 * r_in_z) * n_rows


def element_bytes(n_tets: int, n_nodes: int, nnzb: int) -> int:
    """Algorithmic HBM bytes of one assembly launch: per tet its 4 row indices 16 B, rest data 64 B and
    16 block positions 64 B; per node u and the inertia target (FP64, 48 B) read and the FP64 gradient
    read/modified/written (48 B); the Hessian values written once (36 B per block)."""
    return n_tets * (16 + 64 + 64) + n_nodes * (48 + 48) + nnzb * 36


def mlp_flops_per_row() -> int:
    """Tensor-core FLOPs of one forward row: 2 x (16 x 128 + 128 x 128 + 128 x 128 + 128 x 16) (the input is
    padded to 16 features and the 3 outputs to 16 columns, as the MMA shapes require)."""
    return 2 * (16 * 128 + 128 * 128 + 128 * 128 + 128 * 16)


def mlp_case(rows: int, reps: int):
    import ctypes as C

    import numpy as np
    import torch

    from . import capi
    from .learned import Mlp
    L = capi.lib()
    ctx = L.sdx_create(0)
    m = Mlp(ctx)
    m.init(0)
    X = np.random.default_rng(0).standard_normal((rows, 16)).astype(np.float32)
    m.forward(X[:1024])  # warm-up (weights to the device, kernel attributes)
    torch.cuda.synchronize()
    torch.cuda.profiler.start()
    for _ in range(reps):
        m.forward(X)
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    L.sdx_destroy(ctx)
    return {"case": "mlp", "rows": rows, "reps": reps, "flops_per_forward": mlp_flops_per_row() * rows}


def step_case(args):
    """Host-driven steps against graph-captured steps (sdx_step_params.newton_graph) on the same workload:
    wall time per step of `--iters` steps after 2 warm-up steps, from the same state, with the Newton and
    CG counts of each."""
    import time
    import torch
    if args.workload == "batch":
        bodies, cfg = scenes.config2(args.seed, n_envs=args.envs)
    elif args.cells <= 10:
        bodies, cfg = scenes.config0(args.seed)
    else:
        bodies, cfg = scenes.config1(args.seed, n=args.cells)
    out = {"case": "step", "workload": args.workload, "cells": args.cells, "n_envs": len(bodies),
           "warm_start": args.warm}
    for graph in (0, 1):
        w = SoftBodyWorld(bodies, cfg, newton_abs_tol=1e-9, newton_max_iter=12 if args.workload == "batch" else 50,
                          warm_start=args.warm, newton_graph=graph)
        w.step(2)
        torch.cuda.synchronize()
        l0 = w.kernel_launches()
        t0 = time.perf_counter()
        newton = cg = 0
        for _ in range(args.iters):
            w.step(1)
            st = w.stats()
            newton += sum(s["newton_iters"] for s in st)
            cg += sum(s["cg_iters"] for s in st)
        torch.cuda.synchronize()
        dt = (time.perf_counter() - t0) / args.iters
        key = "graph" if graph else "host"
        out[key] = {"ms_per_step": dt * 1e3, "newton_per_step": newton / args.iters, "cg_per_step": cg / args.iters,
                    "launches_per_step": (w.kernel_launches() - l0) / args.iters}
        w.close()
    out["graph_over_host"] = out["host"]["ms_per_step"] / out["graph"]["ms_per_step"]
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["pcg", "element", "spmv", "mlp", "step"])
    ap.add_argument("--warm", type=int, default=0, help="step: warm start (SDX_WARM_*: 0 zero, 1 previous, 3 temporal)")
    ap.add_argument("--rows", type=int, default=274656, help="mlp: feature rows per forward")
    ap.add_argument("--workload", choices=["cube", "batch"], default="cube")
    ap.add_argument("--cells", type=int, default=64)
    ap.add_argument("--iters", type=int, default=100)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--envs", type=int, default=1024, help="batch workload: the first N bodies of the batch")
    ap.add_argument("--cta-profile", default=None,
                    help="pcg: also time each CTA's phases over two launches and save them to this .npy")
    args = ap.parse_args(argv)
    if args.case == "mlp":
        print(json.dumps(mlp_case(args.rows, args.reps)))
        return
    if args.case == "step":
        print(json.dumps(step_case(args)))
        return
    if args.workload == "batch":
        bodies, cfg = scenes.config2(args.seed, n_envs=args.envs)
    else:
        bodies, cfg = scenes.config1(args.seed, n=args.cells)
    w = SoftBodyWorld(bodies, cfg, newton_abs_tol=1e-9, newton_max_iter=12)
    w.step(1)  # warm-up: assembles a contact state and the matrix
    import torch
    torch.cuda.synchronize()
    out = {"case": args.case, "workload": args.workload, "cells": args.cells, "n_envs": w.n_envs,
           "n_nodes": w.n_nodes, "n_tets": w.n_tets, "nnzb": w.nnzb}
    if args.case == "pcg":
        w.set_params(newton_max_iter=1, linear_max_iter=args.iters, linear_rel_tol=1e-30, linear_abs_tol=0.0)
        w.set_profiling(True)
        torch.cuda.profiler.start()
        w.step(1)
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
        prof = w.profile()
        st = w.stats()[0]
        # the library's own count for the mode it ran (all envs run the same fixed iteration count)
        bpi = prof["pcg_bytes"] / max(1, prof["pcg_iters"])
        us = prof["pcg_ms"] * 1e3 / max(1, prof["pcg_iters"])
        out.update(cg_iters=st["cg_iters"], bytes_per_iter=bpi, us_per_iter=us,
                   algorithmic_tbs=bpi / (us * 1e-6) / 1e12)
        if args.cta_profile:
            import numpy as np
            n_cta = torch.cuda.get_device_properties(0).multi_processor_count
            runs = []
            for _ in range(2):  # two launches: is the per-CTA spread systematic?
                w.set_profiling(True, cta=True)
                w.step(1)
                torch.cuda.synchronize()
                pr = w.profile()
                cyc = w.pcg_cta_profile(n_cta)
                # cycles -> us: each CTA's four phases add up to the launch's event-timed iteration
                us_it = pr["pcg_ms"] * 1e3 / max(1, pr["pcg_iters"])
                runs.append(cyc / cyc.sum(axis=1, keepdims=True) * us_it)
            prof2 = np.stack(runs)
            np.save(args.cta_profile, prof2)
            spmv = prof2[:, :, 0]
            out.update(cta_spmv_us_mean=float(spmv.mean()), cta_spmv_us_min=float(spmv.min()),
                       cta_spmv_us_max=float(spmv.max()),
                       cta_spmv_run_corr=float(np.corrcoef(spmv[0], spmv[1])[0, 1]),
                       cta_wait1_us_mean=float(prof2[:, :, 1].mean()),
                       cta_update_us_mean=float(prof2[:, :, 2].mean()),
                       cta_wait2_us_mean=float(prof2[:, :, 3].mean()))
    elif args.case == "element":
        torch.cuda.profiler.start()
        w.assemble(hess=True, psd=True, obj=True)
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
        by = element_bytes(w.n_tets, w.n_nodes, w.nnzb)
        out.update(bytes_per_launch=by)
        # every launch shape: Hessian assembly (plain / warp-aggregated scatter) and residual-only assembly,
        # device time per element launch from the library's event timers
        shapes = {}
        for th in (64, 128, 256):
            for agg in (0, 1):
                os.environ.update(SDX_ELEM_THREADS=str(th), SDX_ELEM_RES_THREADS=str(th), SDX_ELEM_AGG=str(agg))
                w.set_profiling(True)
                for _ in range(args.reps):
                    w.assemble(hess=True, psd=True, obj=False)
                    if agg == 0:
                        w.assemble(hess=False, psd=True, obj=False)
                pr = w.profile()
                key = f"{th}{'_agg' if agg else ''}"
                shapes[key] = {"hess_ms": pr["asm_hess_ms"] / max(1, pr["asm_hess_launches"])}
                if agg == 0:
                    shapes[key]["res_ms"] = pr["asm_res_ms"] / max(1, pr["asm_res_launches"])
        for k in ("SDX_ELEM_THREADS", "SDX_ELEM_RES_THREADS", "SDX_ELEM_AGG"):
            os.environ.pop(k, None)
        w.set_profiling(False)
        out.update(shapes=shapes)
    else:
        torch.cuda.profiler.start()
        ms, by = w.bench_spmv(reps=args.reps)
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
        out.update(ms=ms, bytes_per_launch=by)
    w.close()
    print(json.dumps(out))


if __name__ == "__main__":
    main()
