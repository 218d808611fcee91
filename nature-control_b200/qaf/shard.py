"""Placement of ensemble instances on ranks (one process per GPU).

Instances are independent, so an ensemble shards with no exchange while it
steps: each rank advances its own subset and results are gathered at the end.
The cost of an instance is taken as N^2 log2 N (one step's FFT work on an
N x N grid); instances go, largest first, to the rank with the least work so
far (longest-processing-time rule), ties to the lower rank, which keeps every
rank within one largest instance of the mean.
"""
from __future__ import annotations

import math
from typing import List, Sequence


def instance_cost(n: int) -> float:
    return float(n) * n * math.log2(n)


def shard_instances(sizes: Sequence[int], world: int) -> List[List[int]]:
    """Instance ids per rank; every id appears once, in ascending order per rank."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(sizes)), key=lambda k: (-instance_cost(sizes[k]), k))
    load = [0.0] * world
    out: List[List[int]] = [[] for _ in range(world)]
    for k in order:
        r = min(range(world), key=lambda i: (load[i], i))
        out[r].append(k)
        load[r] += instance_cost(sizes[k])
    return [sorted(v) for v in out]


def rank_cost(sizes: Sequence[int], ids: Sequence[int]) -> float:
    return sum(instance_cost(sizes[k]) for k in ids)


def draw_ensemble(count: int, seed: int, sizes=(64, 128, 256), alpha=(0.5, 2.0), rf=(0.01, 0.5)):
    """Seeded instance table: grid size ~ U{sizes}, activity ~ U(alpha), friction ~ U(rf), and a seed each."""
    import numpy as np
    g = np.random.default_rng(seed)
    n = [int(v) for v in g.choice(np.asarray(sizes), size=count)]
    a = [float(v) for v in g.uniform(alpha[0], alpha[1], size=count)]
    m = [float(v) for v in g.uniform(rf[0], rf[1], size=count)]
    seeds = [int(v) for v in g.integers(1, 2**62, size=count)]
    return n, a, m, seeds


def gather_by_instance(ids: Sequence[int], values: Sequence, count: int):
    """All ranks' per-instance results as one list indexed by instance id.

    Every rank passes the ids it advanced and one value per id; the result
    (on every rank) has `count` entries. Uses torch.distributed when it is
    initialised (any backend), else returns the local values in place.
    """
    if len(ids) != len(values):
        raise ValueError("one value per instance id")
    pairs = list(zip(ids, values))
    try:
        import torch.distributed as dist
        parts = [None] * dist.get_world_size() if dist.is_available() and dist.is_initialized() else None
    except ImportError:
        parts = None
    if parts is not None:
        dist.all_gather_object(parts, pairs)
        pairs = [pv for part in parts for pv in part]
    out = [None] * count
    for k, v in pairs:
        if out[k] is not None:
            raise ValueError(f"instance {k} reported by more than one rank")
        out[k] = v
    missing = [k for k, v in enumerate(out) if v is None]
    if missing:
        raise ValueError(f"instances without a result: {missing[:8]}")
    return out
