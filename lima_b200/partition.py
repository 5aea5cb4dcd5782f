"""Assignment of independent systems to GPUs (config 4 across ranks).

Systems never exchange data, so a multi-GPU batch is a partition with no
collective on the data path: each rank steps its own subset in one batched
engine.  The partition is the longest-processing-time greedy rule on an
estimated per-step cost, computed identically on every rank.
"""
from __future__ import annotations

import heapq


def step_cost(n_atoms: int, pme_points: int = 0) -> float:
    """Relative per-step cost: pair work grows with atoms, PME with grid points."""
    return float(n_atoms) + 0.25 * float(pme_points)


def lpt_partition(costs, n_ranks: int) -> list[list[int]]:
    """Indices of `costs` per rank; largest first onto the least-loaded rank
    (ties broken by rank id, so every rank computes the same answer)."""
    if n_ranks < 1:
        raise ValueError("n_ranks must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(n_ranks)]
    out = [[] for _ in range(n_ranks)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    return [sorted(v) for v in out]
