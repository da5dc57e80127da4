"""Scenes of a batched run shared out over ranks (one GPU each) by cost.

A scene's substep reads and writes its particles and touches its grid, so its
cost is taken as N_p + N_n: particles plus halo nodes, (cellsX + 3) x
(cellsY + 3).  Scenes are independent: a rank steps its share with no
collective on the data path, and the run's time is the slowest rank's.
`shard_by_cost` balances the shares with the longest-processing-time rule
(largest scene first, each to the rank with the least cost so far), which
keeps every rank within one scene's cost of the mean.  Every rank computes
the same assignment from the same inputs (ties are broken by scene index and
rank index), so no exchange is needed to agree on it.
"""
from __future__ import annotations

import heapq


def scene_cost(particles: int, cells_x: int, cells_y: int) -> int:
    """N_p + N_n of one scene."""
    return int(particles) + (int(cells_x) + 3) * (int(cells_y) + 3)


def shard_by_cost(costs, ranks: int) -> list:
    """Scene indices per rank (each list ascending), largest scenes placed
    first on the least-loaded rank."""
    if ranks < 1:
        raise ValueError("ranks must be positive")
    order = sorted(range(len(costs)), key=lambda k: (-costs[k], k))
    heap = [(0, r) for r in range(ranks)]
    shares = [[] for _ in range(ranks)]
    for k in order:
        load, r = heapq.heappop(heap)
        shares[r].append(k)
        heapq.heappush(heap, (load + costs[k], r))
    return [sorted(s) for s in shares]
