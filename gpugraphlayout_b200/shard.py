"""Sharding a batch of independent graphs over ranks (one process per GPU).

Graphs do not interact, so the batch splits with no collective on the data
path: each rank lays out its own share and only the timing is reduced (the
maximum over ranks).  Shares are balanced by a greedy longest-first packing
on nodes + edges, the work of one FA2 iteration being roughly proportional
to both."""
from __future__ import annotations

import heapq


def partition(costs, world: int) -> list[list[int]]:
    """Graph indices per rank: each graph, largest cost first, to the rank
    with the least cost so far (ties to the lower rank).  Deterministic, so
    every rank computes the same split on its own."""
    heap = [(0, r) for r in range(world)]
    parts: list[list[int]] = [[] for _ in range(world)]
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    for p in parts:
        p.sort()
    return parts


def graph_costs(graphs) -> list[int]:
    """nodes + edges of each (n, sources, targets) graph."""
    return [int(n) + len(s) for n, s, _ in graphs]
