"""Rank partitioning and the max-over-ranks timing, with world_size 2 on gloo
(host processes)."""
import os
import socket

import pytest


def test_shard_by_cost_balances_and_covers():
    from napmo_b200.parallel import shard_by_cost
    costs = [5.0, 1.0, 4.0, 3.0, 3.0, 2.0, 2.0, 8.0]
    parts = shard_by_cost(costs, 3)
    assert sorted(i for p in parts for i in p) == list(range(len(costs)))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(costs)
    assert shard_by_cost(costs, 3) == parts
    assert shard_by_cost(costs, 1) == [list(range(len(costs)))]


def _free_port():
    s = socket.socket()
    s.bind(('127.0.0.1', 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    from napmo_b200.parallel import max_over_ranks, shard_by_cost
    os.environ['MASTER_ADDR'] = '127.0.0.1'
    os.environ['MASTER_PORT'] = str(port)
    dist.init_process_group('gloo', rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    costs = [float((7 * i) % 11 + 1) for i in range(20)]
    mine = shard_by_cost(costs, world)[rank]
    dist.barrier()
    t = max_over_ranks(0.5 + rank, dist)
    work = max_over_ranks(sum(costs[i] for i in mine), dist)
    q.put((rank, mine, t, work))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_gloo():
    import multiprocessing as mp
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    out.sort()
    assert out[0][2] == out[1][2] == 1.5           # max over ranks of 0.5 + rank
    assert out[0][3] == out[1][3]
    assert sorted(out[0][1] + out[1][1]) == list(range(20))
    assert not set(out[0][1]) & set(out[1][1])
