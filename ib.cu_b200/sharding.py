"""Partition of independent instances over ranks (one process per GPU).

The operators have no exchange step between instances, so a multi-GPU run of
a batch is a set of replicas: each rank runs the batched launch over its own
share of the instances, and the job's time is the slowest rank's.  The
instances are dealt by longest-processing-time first: sorted by decreasing
cost (points plus faces, the two terms of the operators' traffic), each goes
to the rank with the least cost so far, so every rank's load is within one
instance's cost of the mean.
"""
from __future__ import annotations


def instance_cost(points: int, faces: int) -> float:
    """Bytes an instance moves per spread+interpolate: 48 B per point and
    8 B per face, per operator."""
    return 2.0 * (48.0 * points + 8.0 * faces)


def partition(costs, world: int):
    """Instance ids per rank (each list ascending); deterministic, so every
    rank computes the same partition from the same costs."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = [0.0] * world
    shards = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        shards[r].append(i)
        load[r] += float(costs[i])
    return [sorted(s) for s in shards]
