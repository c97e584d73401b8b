"""Multi-GPU sharding of the batched workload (one process per GPU).

Clouds are independent, so the batched path shards by cloud with no
collective on the data path: every rank gets a size-balanced subset (greedy
longest-processing-time assignment by n * log n, a proxy for the per-cloud
evolve work), solves it with BatchedRidgeDetection on its own GPU, and the
per-cloud results are gathered on the host at the end (torch.distributed,
NCCL or gloo).  The single-cloud paths do not shard (a per-pass exchange of
centroid sums would break index-order summation and with it bit parity), so
for them each rank runs a replica.
"""
from __future__ import annotations

import heapq
import math
from typing import Callable, Dict, List, Sequence, Tuple


def shard_lpt(sizes: Sequence[int], world: int) -> List[List[int]]:
    """Cloud indices per rank: greedy LPT on cost n*log2(n+1), each rank's list
    kept in ascending cloud order.  Deterministic for equal inputs."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(sizes)), key=lambda c: (-sizes[c] * math.log2(sizes[c] + 2), c))
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    out: List[List[int]] = [[] for _ in range(world)]
    for c in order:
        load, r = heapq.heappop(heap)
        out[r].append(c)
        heapq.heappush(heap, (load + sizes[c] * math.log2(sizes[c] + 2), r))
    return [sorted(x) for x in out]


def solve_sharded(clouds: Sequence[Tuple], solve: Callable[[Sequence[Tuple]], List],
                  rank: int, world: int, group=None) -> Dict[int, object]:
    """Every rank solves its LPT shard with `solve` (a list of clouds -> list of
    results) and receives all ranks' results, keyed by global cloud index."""
    import torch.distributed as dist
    shards = shard_lpt([int(c[0].shape[0]) for c in clouds], world)
    mine = shards[rank]
    local = solve([clouds[i] for i in mine])
    payload = list(zip(mine, local))
    if world == 1:
        gathered = [payload]
    else:
        gathered = [None] * world
        dist.all_gather_object(gathered, payload, group=group)
    result: Dict[int, object] = {}
    for part in gathered:
        for idx, res in part:
            result[idx] = res
    return result
