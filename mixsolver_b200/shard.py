"""Whole cases across GPUs: one process per GPU, no data-path collective.

The batched and served workloads are many independent cases, so a multi-GPU
run assigns whole cases to ranks and each rank advances its own share
(CaseBatch / serve.Server on its GPU). Every rank evaluates the same
deterministic rule on the same inputs, so no rank has to tell another which
cases are its own:

* :func:`assign` -- a fixed set of cases (a batch): longest-processing-time
  first, each case to the least loaded rank (ties to the lower rank);
* :class:`Router` -- a request stream (serving): each arriving request to the
  rank with the least outstanding work, the work of a request leaving its
  rank's account when the request's modelled service time has passed.

The reference splits one case over MPI ranks instead (METIS partition plus
halo exchange); whole-case assignment is the part of its multi-rank design
that applies to many independent cases.
"""
from __future__ import annotations

import heapq


def assign(work, world: int) -> list:
    """Rank of every case: cases in decreasing work (index order among equals),
    each given to the rank with the least work so far (lowest rank among
    equals). The largest rank load exceeds the smallest by at most the largest
    single case's work."""
    order = sorted(range(len(work)), key=lambda i: (-float(work[i]), i))
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    rank_of = [0] * len(work)
    for i in order:
        load, r = heapq.heappop(heap)
        rank_of[i] = r
        heapq.heappush(heap, (load + float(work[i]), r))
    return rank_of


def mine(work, world: int, rank: int) -> list:
    """Indices of the cases assigned to `rank`, in index order."""
    return [i for i, r in enumerate(assign(work, world)) if r == rank]


class Router:
    """Online assignment of a request stream to ranks. route() takes the
    arrival time and the request's modelled service time (its work over the
    rank's throughput) and returns its rank: the rank whose queue drains
    first, i.e. whose accumulated modelled finish time is earliest (lowest
    rank among equals)."""

    def __init__(self, world: int):
        self.world = world
        self.free_at = [0.0] * world

    def route(self, arrival: float, service: float) -> int:
        r = min(range(self.world), key=lambda k: (max(self.free_at[k], arrival), k))
        self.free_at[r] = max(self.free_at[r], arrival) + float(service)
        return r
