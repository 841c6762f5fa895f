"""Assignment of independent boxes to ranks for a batch spread over several
GPUs (one process per GPU; the boxes never interact, so the data path has no
collective).

Cost model per box: pair work, proportional to the atom count (the density
is the same in every box), plus the FFT work of its PME grid, K^3 log2 K^3,
weighted by one pair-kernel atom per 40 grid points (a grid point costs far
less than an atom's ~100 pair evaluations).  Boxes are dealt largest first to
the least-loaded rank (ties to the lower rank), so every rank computes the
same assignment from the same inputs.
"""

from __future__ import annotations

import heapq
import math


def box_cost(n_atoms: int, grid: int) -> float:
    points = float(grid) ** 3
    return float(n_atoms) + points * math.log2(max(points, 2.0)) / 40.0


def shard(costs: list[float], world: int) -> list[list[int]]:
    """Box indices per rank, each list in increasing order."""
    if world <= 0:
        raise ValueError("world must be positive")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    out: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    return [sorted(x) for x in out]


def imbalance(costs: list[float], parts: list[list[int]]) -> float:
    """Largest rank load over the mean load (1.0 = perfect)."""
    loads = [sum(costs[i] for i in p) for p in parts]
    mean = sum(loads) / len(loads)
    return max(loads) / mean if mean > 0 else 1.0
