"""Placement of independent worlds over ranks (one process per GPU).

Worlds never interact, so a batch shards by world with no collective in the data path: each rank
builds and steps its own share, and only the timing (the slowest rank's) and the totals are
reduced at the end. Shares are balanced by body count with the longest-processing-time rule
(largest world first onto the least-loaded rank), which keeps every rank within one world's size
of the mean.
"""
import heapq


def shard_worlds(sizes, world_size):
    """List of world-index lists, one per rank; each list ascending."""
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    heap = [(0, r) for r in range(world_size)]
    shares = [[] for _ in range(world_size)]
    for k in sorted(range(len(sizes)), key=lambda k: (-int(sizes[k]), k)):
        load, r = heapq.heappop(heap)
        shares[r].append(k)
        heapq.heappush(heap, (load + int(sizes[k]), r))
    return [sorted(s) for s in shares]


def rank_share(sizes, rank, world_size):
    return shard_worlds(sizes, world_size)[rank]


def max_over_ranks(value, dist=None, device="cpu"):
    """The maximum of a float over the process group (the slowest rank's time); the value itself
    without a group."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value, dist=None, device="cpu"):
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
