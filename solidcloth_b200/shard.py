"""Partition independent cloth instances over ranks (multi-GPU batches).

Instances never interact, so a batch shards with no collective on the data
path: each rank steps its own instances; only the final metrics are gathered.
Instances are placed by longest-processing-time-first greedy bin packing on an
estimated cost (triangles x iterations, i.e. the constraint-sweep work), which
keeps the most loaded rank within 4/3 of the optimum.
"""
from __future__ import annotations

import heapq


def instance_cost(scene) -> float:
    n = scene.n
    tris = 2 * (n - 1) ** 2
    return float(tris * max(1, scene.params.iterations) * max(1, scene.params.substeps))


def partition(costs, parts: int):
    """list of index lists, one per part; deterministic (ties by index)"""
    if parts < 1:
        raise ValueError("parts must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(parts)]
    out = [[] for _ in range(parts)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    return [sorted(o) for o in out]


def shard(instances, rank: int, world: int):
    """the instances rank `rank` of `world` steps"""
    return [instances[i] for i in partition([instance_cost(s) for s in instances], world)[rank]]
