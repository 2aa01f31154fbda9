"""Sharding a batch of light curves over processes (one per GPU).

Curves are independent and the periodogram path has no exchange step, so a
multi-GPU run is data parallel over curves with no collective on the data
path: each rank computes the periodograms of its own curves, and the
results are gathered once on the host at the end.  The reference splits
curves evenly by count across devices (periodfind/cuda/ce.cu:459-472); here
the split balances the work, sum of curve length x grid size, which matters
for ragged batches.

Works with any torch.distributed process group (NCCL on GPUs, gloo on CPU);
only `all_gather_object` and a scalar `all_reduce` are used.
"""

from __future__ import annotations

import heapq

import numpy as np


def partition_by_work(lengths, world_size):
    """Greedy longest-first assignment of curves to `world_size` shards so
    that the shards' total points are as even as possible.  Returns a list of
    index arrays (each sorted ascending); every curve appears exactly once."""
    lengths = np.asarray(lengths, dtype=np.int64)
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    heap = [(0, r) for r in range(world_size)]
    buckets = [[] for _ in range(world_size)]
    for i in np.argsort(-lengths, kind="stable"):
        load, r = heapq.heappop(heap)
        buckets[r].append(int(i))
        heapq.heappush(heap, (load + max(int(lengths[i]), 1), r))
    return [np.array(sorted(b), dtype=np.int64) for b in buckets]


def calc_sharded(compute, times, mags, rank, world_size, group=None):
    """Run `compute(times_shard, mags_shard)` on this rank's share of the
    curves and return the per-curve results of ALL curves, in input order,
    on every rank.  `compute` returns a list with one entry per curve (what
    the periodogram classes' calc() returns)."""
    import torch.distributed as dist

    parts = partition_by_work([len(t) for t in times], world_size)
    mine = parts[rank]
    local = compute([times[i] for i in mine], [mags[i] for i in mine]) if len(mine) else []
    if len(local) != len(mine):
        raise RuntimeError("compute() must return one result per curve")
    gathered = [None] * world_size
    dist.all_gather_object(gathered, list(zip(mine.tolist(), local)), group=group)
    out = [None] * len(times)
    for shard in gathered:
        for i, res in shard:
            out[i] = res
    return out


def max_over_ranks(value, device=None, group=None):
    """The maximum of a per-rank scalar (e.g. a step time) over all ranks."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
