"""Sharding of independent solves across ranks (one process per GPU).

The ensemble's instances are independent: a rank advances its own shard with no data-path
collective.  Two partitions are provided:

* weak_shard: every rank owns the next `n` instances of the seeded stream (per-GPU work fixed
  as ranks are added -- weak scaling, what the benchmark reports);
* balanced_partition: a fixed set of instances split across ranks by greedy
  longest-processing-time on their cost (points x steps), for strong scaling.

The only cross-rank operation is the max over ranks of a timing, done by the caller's
process group (NCCL on GPUs, gloo in the CPU tests).
"""
from __future__ import annotations

import heapq


def weak_shard(n_per_rank: int, rank: int) -> tuple[int, int]:
    """[first, first + n) of the global instance stream owned by `rank`."""
    if n_per_rank < 0 or rank < 0:
        raise ValueError("negative size or rank")
    return rank * n_per_rank, n_per_rank


def balanced_partition(costs, world: int) -> list[list[int]]:
    """Greedy LPT: assign items (by index) to `world` bins, largest cost first, each to the
    currently lightest bin.  Deterministic: ties break on the lower bin and item index."""
    if world < 1:
        raise ValueError("world must be >= 1")
    bins = [[] for _ in range(world)]
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    for i in sorted(range(len(costs)), key=lambda k: (-costs[k], k)):
        load, r = heapq.heappop(heap)
        bins[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    for b in bins:
        b.sort()
    return bins


def instance_cost(inst) -> float:
    """Work of one instance to t = 2: points x steps."""
    return float(inst.side * inst.side * inst.steps_to_t2)


def max_over_ranks(value: float, dist=None) -> float:
    """Max of a per-rank float over the default process group (identity without one)."""
    if dist is None or not dist.is_available() or not dist.is_initialized():
        return value
    import torch
    backend = dist.get_backend()
    dev = "cuda" if backend == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
