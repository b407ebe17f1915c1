"""Partition of a batch of independent worlds over ranks (one GPU each).

Worlds never interact, so the batched form shards with no data-path
exchange: rank r steps the contiguous world range whose bodies fall in its
share of the cumulative body count, on its own GPU.  The only collectives are
the timing barrier and a max/sum over ranks for reporting.
"""
from __future__ import annotations

from typing import List, Sequence, Tuple

import numpy as np

from .bodies import BodyArrays, take_range


def partition_worlds(world_begin: Sequence[int], nranks: int) -> List[Tuple[int, int]]:
    """Contiguous world ranges [w0, w1) per rank, balanced by body count.

    Rank r takes the worlds whose first body lies in [r*N/R, (r+1)*N/R) of the
    cumulative body count N; every world goes to exactly one rank, in order.
    A rank may get no world when there are fewer worlds than ranks.
    """
    begin = np.asarray(world_begin, dtype=np.int64)
    nworlds = len(begin) - 1
    if nranks < 1:
        raise ValueError("nranks must be >= 1")
    total = int(begin[-1])
    cuts = [0]
    for r in range(1, nranks):
        target = total * r // nranks
        w = int(np.searchsorted(begin[:-1], target, side="left"))
        cuts.append(max(cuts[-1], min(w, nworlds)))
    cuts.append(nworlds)
    return [(cuts[r], cuts[r + 1]) for r in range(nranks)]


def slice_bodies(bodies: BodyArrays, world_begin: Sequence[int], w0: int, w1: int):
    """Bodies of worlds [w0, w1) and their world ranges re-based at 0."""
    begin = np.asarray(world_begin, dtype=np.int64)
    b0, b1 = int(begin[w0]), int(begin[w1])
    return take_range(bodies, b0, b1), (begin[w0:w1 + 1] - b0).astype(np.uint32)
