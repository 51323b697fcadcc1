"""Sharding of independent problems over ranks (one GPU each).

A batch of independent SDPs partitions with no exchange on the data path:
every rank solves its own share and only the timing is reduced.  The share
is a longest-processing-time assignment on the per-iteration work estimate
m^3/3 + sum_l (m^2 n_l^2 + 4 n_l^3 m) (Cholesky of B, Schur pairs, the two
n^3 products per constraint), the same estimate the library's batch uses to
order its queue.  Every rank computes the same assignment from the same
list, so no message is needed to agree on it.
"""
from __future__ import annotations

import heapq


def work_estimate(m: int, blocks) -> float:
    """Per-iteration dd-flop estimate of one problem."""
    w = m ** 3 / 3.0
    for n in blocks:
        w += float(m) * m * n * n + 4.0 * n * n * n * m
    return w


def partition_by_work(works, world: int):
    """Split problem indices into `world` lists: problems in descending
    work, each to the rank with the least work so far (ties to the lower
    rank); each list keeps that descending order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(works)), key=lambda q: (-works[q], q))
    heap = [(0.0, r) for r in range(world)]
    shares = [[] for _ in range(world)]
    for q in order:
        load, r = heapq.heappop(heap)
        shares[r].append(q)
        heapq.heappush(heap, (load + works[q], r))
    return shares
