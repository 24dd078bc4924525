"""Replica sharding and the max-over-ranks timing reduction, as world_size-2 gloo process groups on CPU."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from project_superdex_b200 import replicas


def test_shard_envs_partition():
    for n in (1, 7, 1024):
        for w in (1, 2, 3, 8):
            if n < w:
                continue
            parts = [replicas.shard_envs(n, r, w) for r in range(w)]
            assert sum(len(p) for p in parts) == n
            assert parts[0].start == 0 and parts[-1].stop == n
            assert all(parts[i].stop == parts[i + 1].start for i in range(w - 1))
            assert max(len(p) for p in parts) - min(len(p) for p in parts) <= 1


def test_shard_by_weight_balances_uneven_envs():
    rng = np.random.default_rng(0)
    w = (rng.integers(8, 41, size=(256, 3)).prod(axis=1) * 6).tolist()
    parts = replicas.shard_by_weight(w, 4)
    assert parts[0].start == 0 and parts[-1].stop == 256 and all(len(p) > 0 for p in parts)
    loads = [sum(w[i] for i in p) for p in parts]
    assert max(loads) / (sum(loads) / 4) < 1.1


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from oracle import oracle as O
    from project_superdex_b200 import scenes
    # each rank steps its own, differently seeded env with the CPU oracle (stand-in for the GPU step)
    rng = np.random.default_rng(replicas.replica_seed(0, rank))
    b = scenes.grid_body(3, 3, 3, 0.01, rng=rng)
    s = O.Scene(b, scenes.SceneConfig())
    u, v, st = s.step(np.zeros(3 * b.n_nodes), np.zeros(3 * b.n_nodes), 1 / 240.0)
    t = replicas.max_over_ranks(float(rank + 1))
    dist.barrier()
    q.put((rank, t, st.convergence, float(np.abs(u).max())))
    dist.destroy_process_group()


def test_two_rank_replicas_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    assert [r[1] for r in res] == [2.0, 2.0]  # max over ranks
    assert all(r[2] == 1 for r in res)
    assert res[0][3] != res[1][3]  # different seeds -> different replicas
