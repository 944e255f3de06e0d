"""Partition of independent instances over ranks (the batched workload's
multi-GPU split: instances are independent, so there is no data-path
collective)."""
from __future__ import annotations


def balanced_shards(costs, world: int) -> list:
    """Greedy longest-processing-time split: instances in decreasing cost,
    each to the rank with the least total so far (ties to the lower rank).
    Returns per-rank lists of instance indices in increasing order; every
    index appears exactly once."""
    if world < 1:
        raise ValueError("world must be >= 1")
    load = [0] * world
    parts = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda k: (-costs[k], k)):
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(i)
        load[r] += costs[i]
    return [sorted(p) for p in parts]
