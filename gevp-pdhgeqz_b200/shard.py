"""Size-balanced sharding of a batch of independent pencils across ranks.

A batch of independent pencils shards with no exchange step: each rank
solves its own subset and only the host gathers results.  The cost of one
pencil grows like n^3, so the subsets are balanced by longest-processing-
time-first assignment: pencils in decreasing size order, each to the rank
with the least accumulated n^3 (ties to the lowest rank).  Deterministic,
so every rank computes the same partition without communication.
"""
from __future__ import annotations

import numpy as np


def balance(sizes, world: int):
    """Partition pencil indices over ``world`` ranks.  Returns (parts, load)
    where parts[r] is the sorted index list of rank r and load[r] its
    summed n^3."""
    sizes = np.asarray(sizes, dtype=np.int64)
    order = sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]), i))
    load = [0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += int(sizes[i]) ** 3
    return [sorted(p) for p in parts], load


def shard(sizes, rank: int, world: int):
    """Indices of the pencils rank ``rank`` solves."""
    return balance(sizes, world)[0][rank]


def imbalance(load) -> float:
    """max / mean of the per-rank loads (1.0 is perfect)."""
    m = float(np.mean(load))
    return float(max(load)) / m if m > 0 else 1.0
