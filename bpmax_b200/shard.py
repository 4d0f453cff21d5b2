"""Batches across GPUs: pairs are independent objects, so a batch is split over the ranks by
estimated work and every rank fills its own share on its own GPU. The only exchange is the gather
of the scores (and gradients) to every rank at the end, one object all-gather; no collective on
the data path. The reference fills one pair per process run on one node (OpenMP), so this has no
counterpart there.

Work estimate of a pair: the max-plus candidates its fill evaluates at the inner table width the
GPU pads strand 2 to (a multiple of 8 up to 64, then of 64), from the fill's term count
C(M)C(N) + 2T(M)C(N) + 2C(M)T(N) + C(M) + C(N).
"""
from __future__ import annotations

import heapq

import numpy as np

from . import workloads as W


def padded_width(n: int) -> int:
    """The inner table width the GPU uses for a strand-2 length n."""
    return max(8, (n + 7) // 8 * 8) if n <= 64 else (n + 63) // 64 * 64


def pair_cost(m: int, n: int) -> int:
    return int(W.terms(m, padded_width(n))["total"])


def lpt_partition(costs, world: int) -> list[list[int]]:
    """Longest-processing-time-first greedy: pairs in decreasing cost (ties by index) each go to the
    rank with the least work so far (ties by rank). Returns each rank's pair indices, ascending.
    The largest share exceeds the mean by less than the largest single cost."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0, r) for r in range(world)]
    shares: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        shares[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    return [sorted(s) for s in shares]


def shares_of(pairs, world: int) -> list[list[int]]:
    return lpt_partition([pair_cost(len(a), len(b)) for a, b in pairs], world)


def run_sharded(fn, pairs, rank: int, world: int, group=None):
    """Runs ``fn`` (a list of pairs -> an array with one row per pair, e.g. Engine.score_batch) on
    this rank's LPT share of ``pairs`` and gathers every rank's rows into the batch order on every
    rank (torch.distributed all_gather_object over ``group``; every rank must call this with the same
    pairs). Returns (rows of the whole batch, this rank's pair indices)."""
    shares = shares_of(pairs, world)
    mine = shares[rank]
    local = np.asarray(fn([pairs[i] for i in mine])) if mine else None
    if world == 1:
        return local, mine
    import torch.distributed as dist

    got = [None] * world
    dist.all_gather_object(got, (mine, local), group=group)
    out = None
    for idx, rows in got:
        if not idx:
            continue
        if out is None:
            out = np.zeros((len(pairs),) + rows.shape[1:], dtype=rows.dtype)
        out[idx] = rows
    return out, mine
