"""Multi-GPU plumbing for the soft-body step: replicas only.

Environments are independent (one island per env, mochi_physics/src/mochi_step.cpp:489-510 runs one task
per island), so the step shards by environment with no data-path exchange. Each rank steps its own
batch on its own GPU; the only collectives are host-side bookkeeping (a barrier before timing and the
max of the per-rank device times).
"""
from __future__ import annotations

from typing import List, Sequence


def shard_envs(n_envs: int, rank: int, world: int) -> range:
    """Contiguous, balanced env range of `rank` (strong scaling of a fixed global batch)."""
    if world <= 0 or not (0 <= rank < world):
        raise ValueError("bad rank/world")
    base, extra = divmod(n_envs, world)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def shard_by_weight(weights: Sequence[float], world: int) -> List[range]:
    """Contiguous env ranges of near-equal total weight (e.g. tets per env) for uneven batches."""
    total = float(sum(weights))
    out, start, acc = [], 0, 0.0
    for r in range(world):
        target = total * (r + 1) / world
        end = start
        while end < len(weights) and (acc + weights[end] <= target or end == start) and \
                len(weights) - end > world - r - 1:
            acc += weights[end]
            end += 1
        if r == world - 1:
            end = len(weights)
        out.append(range(start, end))
        start = end
    return out


def replica_seed(base_seed: int, rank: int) -> int:
    """Weak scaling: every rank steps its own, differently seeded batch of the same size."""
    return base_seed + 1000003 * rank


def max_over_ranks(value: float, device=None) -> float:
    """Max of a per-rank scalar (device time) over the process group; identity without one."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
