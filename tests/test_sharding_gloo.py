"""Multi-rank host logic of the batching/serving forms, on CPU with world_size 2 over gloo: the scene
partition covers every scene once and balances cost, and the per-rank tallies combine as sum / max."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from luisacomputesimulator_b200.sharding import combine, partition


def test_partition_covers_and_balances():
    costs = [1000 * (1 + (7 * k) % 13) for k in range(64)]
    for world in (1, 2, 3, 8):
        shards = partition(costs, world)
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(64))
        loads = [sum(costs[i] for i in s) for s in shards]
        assert max(loads) - min(loads) <= max(costs)
    assert partition(costs, 4) == partition(costs, 4)  # deterministic
    with pytest.raises(ValueError):
        partition(costs, 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, costs, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = partition(costs, world)[rank]
        seconds = 1.0 + rank  # stands in for the rank's device time
        total, tmax = combine(len(mine), seconds)
        q.put((rank, sorted(mine), total, tmax))
    finally:
        dist.destroy_process_group()


def test_two_ranks_share_scenes_and_combine_tallies():
    costs = [3, 9, 1, 7, 7, 2, 8, 4]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, costs, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got.sort()
    assert sorted(got[0][1] + got[1][1]) == list(range(len(costs)))
    assert not set(got[0][1]) & set(got[1][1])
    for _, _, total, tmax in got:
        assert total == len(costs) and tmax == 2.0
