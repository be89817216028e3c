"""Placement of independent scenes on ranks (one process per GPU).

Scenes of a batch do not interact, so a multi-GPU run needs no collective on the data
path: each rank steps its own batch and only the final metrics are reduced.  A fixed list
of scenes is split by longest-processing-time-first scheduling on an estimated cost per
scene (particles x expected substeps per frame), which keeps the most loaded rank within
4/3 of the optimum.  Every rank computes the same placement from the same inputs.
"""
from __future__ import annotations


def shard_scenes(costs, world: int) -> list[list[int]]:
    """Scene indices per rank: LPT on `costs` (ties broken by index, deterministic)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    loads = [0.0] * world
    out: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (loads[k], k))
        out[r].append(i)
        loads[r] += float(costs[i])
    return [sorted(v) for v in out]


def shard_loads(costs, shards) -> list[float]:
    return [sum(float(costs[i]) for i in s) for s in shards]
