"""Whole-scene sharding for the batching and serving forms on several GPUs (one process per GPU).

Scenes are independent, so there is no collective on the data path: each rank steps the scenes assigned to
it, and only the per-rank tallies (solves done, device time) are combined at the end (sum and max)."""
from __future__ import annotations

import heapq


def partition(costs, world):
    """Greedy longest-processing-time partition of scene costs over `world` ranks.  Returns one sorted index
    list per rank; every index appears exactly once; deterministic for given costs."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    shards = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        shards[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(s) for s in shards]


def combine(done, seconds, device=None):
    """Sum of `done` and max of `seconds` over the ranks of the default process group (or the local values
    when no group is initialised)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(done), float(seconds)
    d = torch.tensor([float(done)], dtype=torch.float64, device=device)
    t = torch.tensor([float(seconds)], dtype=torch.float64, device=device)
    dist.all_reduce(d, op=dist.ReduceOp.SUM)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(d.item()), float(t.item())
