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


def _small_batch():
    from exgame_b200.abi import NEWTON, PRECISION_F64, step_params, LIE_EULER, GRAVITY_PLUMMER, JOINT_DTYPE
    sizes = scenarios.config3_sizes(12, seed=21, lo=4, hi=40)
    worlds = []
    for k, n in enumerate(sizes):
        if k % 2 == 0:
            worlds.append((scenarios.gravity_world(int(n), 10.0, seed=100 + k), np.zeros(0, dtype=JOINT_DTYPE),
                           step_params(integrator=LIE_EULER, gravity_law=GRAVITY_PLUMMER, softening=0.05, dt=1e-3)))
        else:
            b, j = scenarios.tree_world(int(n), seed=200 + k)
            worlds.append((b, j, step_params(integrator=NEWTON, precision=PRECISION_F64, dt=1e-2, tol=1e-10)))
    return sizes, worlds


def _stepping_rank(rank, world_size, port, out, use_gpu):
    """Rank `rank` steps its share of the batch (the oracle on CPU, the library on the GPU) and
    all-gathers every world's final state over gloo."""
    import sys
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world_size, timeout=timedelta(seconds=60))
    sizes, worlds = _small_batch()
    mine = shard_worlds(sizes, world_size)[rank]
    states = {}
    if use_gpu:
        from exgame_b200 import _lib
        dev = _lib.Device(0)
        batch = _lib.DeviceBatch(dev, [worlds[k] for k in mine])
        batch.step(15)
        for i, k in enumerate(mine):
            states[k] = batch.world_bodies(i)
        batch.close()
        dev.close()
    else:
        import oracle_lib
        for k in mine:
            ow = oracle_lib.OracleWorld(*worlds[k])
            ow.step(15)
            states[k] = ow.bodies()
    flat = np.zeros((int(np.sum(sizes)), 14))
    off = np.concatenate([[0], np.cumsum(sizes)])
    for k, b in states.items():
        flat[off[k]:off[k + 1], :8] = b["pose"]
        flat[off[k]:off[k + 1], 8:] = b["momentum"]
    gathered = [torch.zeros(flat.shape, dtype=torch.float64) for _ in range(world_size)]
    dist.all_gather(gathered, torch.from_numpy(flat))
    dist.barrier()
    dist.destroy_process_group()
    total = sum(g.numpy() for g in gathered)  # each world is non-zero on exactly one rank
    out.put((rank, total))


def _run_sharded(use_gpu):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_stepping_rank, args=(r, 2, port, q, use_gpu)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=240) for _ in procs), key=lambda x: x[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert np.array_equal(res[0][1], res[1][1])
    return res[0][1]


@pytest.mark.timeout(300)
def test_sharded_oracle_run_equals_one_process(oracle):
    got = _run_sharded(use_gpu=False)
    sizes, worlds = _small_batch()
    off = np.concatenate([[0], np.cumsum(sizes)])
    for k, w in enumerate(worlds):
        ow = oracle.OracleWorld(*w)
        ow.step(15)
        b = ow.bodies()
        assert np.array_equal(got[off[k]:off[k + 1], :8], b["pose"])
        assert np.array_equal(got[off[k]:off[k + 1], 8:], b["momentum"])


@pytest.mark.gpu
@pytest.mark.timeout(300)
def test_sharded_device_run_equals_one_batch(device):
    """Two processes share cuda:0, each stepping its share of the batch through the library (their
    kernels never wait on each other; the exchange is gloo on the host): every world ends bit for
    bit as in one batch of all worlds."""
    from exgame_b200 import _lib
    got = _run_sharded(use_gpu=True)
    sizes, worlds = _small_batch()
    batch = _lib.DeviceBatch(device, worlds)
    batch.step(15)
    off = np.concatenate([[0], np.cumsum(sizes)])
    for k in range(len(worlds)):
        b = batch.world_bodies(k)
        assert np.array_equal(got[off[k]:off[k + 1], :8], b["pose"])
        assert np.array_equal(got[off[k]:off[k + 1], 8:], b["momentum"])
    batch.close()
