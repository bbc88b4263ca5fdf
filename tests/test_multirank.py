"""The multi-rank path on CPU: two gloo ranks shard a batch of worlds by body count, agree that the
shares cover every world once, and reduce the timing as the bench does (max over ranks) and the
work as a sum."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from exgame_b200 import scenarios
from exgame_b200.sharding import max_over_ranks, shard_worlds, sum_over_ranks


def test_shares_cover_every_world_once_and_balance():
    sizes = scenarios.config3_sizes(4096, seed=3)
    for n in (1, 2, 3, 8):
        shares = shard_worlds(sizes, n)
        flat = sorted(k for s in shares for k in s)
        assert flat == list(range(len(sizes)))
        loads = [int(sum(sizes[k] for k in s)) for s in shares]
        assert max(loads) - min(loads) <= int(max(sizes))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world_size, port, out):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world_size, timeout=timedelta(seconds=60))
    sizes = scenarios.config3_sizes(512, seed=5)
    mine = shard_worlds(sizes, world_size)[rank]
    bodies = int(sum(sizes[k] for k in mine))
    total = sum_over_ranks(bodies, dist)
    slowest = max_over_ranks(1.0 + rank, dist)  # rank r "took" 1 + r seconds
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, bodies, total, slowest))


@pytest.mark.timeout(120)
def test_two_gloo_ranks_shard_and_reduce():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=90) for _ in procs)
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    sizes = scenarios.config3_sizes(512, seed=5)
    assert res[0][1] + res[1][1] == int(np.sum(sizes))
    assert res[0][2] == res[1][2] == float(np.sum(sizes))
    assert res[0][3] == res[1][3] == 2.0
