"""Host side of the centre-sharded multi-GPU count.

Every triple has one owner hyperedge: its centre when open, its smallest
member when closed (MoCHy-master/main_exact.cpp:114-124). Each rank holds a
replica of the store and counts the triples of its share of the owners
(``Graph.count_static30_shard(rank, world)``); the partial 30-bin vectors
are summed with one all-reduce. Nothing else crosses between ranks.

The helpers here work with any torch.distributed backend: NCCL with tensors
on the rank's GPU, gloo with CPU tensors (the tests run them that way).
"""
from __future__ import annotations

import numpy as np


def allreduce_counts(part: np.ndarray, dist, device=None) -> np.ndarray:
    """Sums uint64 count vectors over all ranks.

    The counts travel as int64 (torch has no uint64 reduction); two's
    complement addition is the same operation modulo 2^64, so the sum is
    exact for any total that fits a uint64.
    """
    import torch

    a = np.ascontiguousarray(part, dtype=np.uint64)
    t = torch.from_numpy(a.view(np.int64).copy())
    if device is not None:
        t = t.to(device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return t.cpu().numpy().view(np.uint64).copy()


def max_over_ranks(seconds: float, dist, device=None) -> float:
    """The slowest rank's time: a sharded step ends when its last rank does."""
    import torch

    t = torch.tensor([float(seconds)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def agree_schedule(schedule, dist, device=None, src: int = 0) -> tuple[int, ...]:
    """Every rank's copy of rank `src`'s launch schedule.

    The GPU shards take every world-th item of one heaviest-first work list,
    and the order of that list follows the schedule (it is split into the
    launch shapes first), so the partials add up to the full count only when
    all ranks use the same schedule: tune on one rank, then agree on it.
    """
    import torch

    t = torch.tensor([int(x) for x in schedule], dtype=torch.int64, device=device)
    dist.broadcast(t, src)
    return tuple(int(x) for x in t.cpu().tolist())


def owner_shard(owner_ids: np.ndarray, world: int) -> np.ndarray:
    """Rank that counts the triples of each owner id under the round-robin
    split the oracle shard uses (a mod world)."""
    return (np.asarray(owner_ids, dtype=np.uint64) % np.uint64(world)).astype(np.int64)
