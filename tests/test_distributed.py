"""Host-side multi-rank logic on CPU: LPT sharding and the gather of per-cloud
results over torch.distributed (gloo, world_size 2).  The per-rank solver here
is the CPU oracle, so no GPU is involved; with GPUs the same code runs with
BatchedRidgeDetection over NCCL."""
import os
import socket

import numpy as np
import pytest

import oracle as O
from ridgedetection_b200 import distributed as D
from ridgedetection_b200 import generators as G


def test_shard_lpt_covers_every_cloud_once_and_balances():
    sizes = [int(s[0]) for s in G.batch_spec(200, n_min=100, n_max=5000)]
    for world in (1, 2, 3, 8):
        shards = D.shard_lpt(sizes, world)
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(len(sizes)))
        loads = [sum(sizes[i] for i in s) for s in shards]
        assert max(loads) <= 1.25 * (sum(loads) / world) + max(sizes)
    assert D.shard_lpt(sizes, 4) == D.shard_lpt(sizes, 4)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        spec = G.batch_spec(12, seed_base=501, n_min=200, n_max=1500)
        clouds = [(G.batch_cloud(n, dim, seed), r1, r2) for (n, dim, r1, r2, seed) in spec]

        def solve(part):
            return [O.ridge_bf(P, r1, r2)[0] for (P, r1, r2) in part]

        res = D.solve_sharded(clouds, solve, rank, world)
        q.put((rank, {k: v.tobytes() for k, v in res.items()}))
    finally:
        dist.destroy_process_group()


def test_sharded_solve_gathers_identical_results_on_every_rank():
    import torch.multiprocessing as mp
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    outs = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert outs[0] == outs[1]
    spec = G.batch_spec(12, seed_base=501, n_min=200, n_max=1500)
    for i, (n, dim, r1, r2, seed) in enumerate(spec):
        S, _ = O.ridge_bf(G.batch_cloud(n, dim, seed), r1, r2)
        assert outs[0][i] == S.tobytes()
