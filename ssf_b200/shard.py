"""Sharding of independent units (load cases, plates) across ranks.

Batches of independent systems need no exchange between GPUs: each rank takes
a share of the units and solves it alone; only the results are gathered at
the end.  The share is a longest-processing-time assignment: units sorted by
weight (descending, ties by index), each given to the currently least-loaded
rank (ties by rank) -- deterministic, so every rank computes the same plan
without communicating.
"""
from __future__ import annotations

import heapq

import numpy as np


def partition(weights, world: int) -> list[list[int]]:
    """Unit indices per rank (each list ascending)."""
    w = np.asarray(weights, dtype=np.float64)
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(w.size), key=lambda i: (-w[i], i))
    heap = [(0.0, r) for r in range(world)]
    out: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + float(w[i]), r))
    return [sorted(x) for x in out]


def plate_weight(mesh) -> float:
    """Work estimate of one plate solve: equations x iterations, iterations
    of Jacobi-CG growing like the plate's longer side."""
    nx, ny = mesh.meta.get("nx", 1), mesh.meta.get("ny", 1)
    return float(mesh.ndof) * max(nx, ny)


def imbalance(weights, parts) -> float:
    """max rank load / mean rank load of a partition."""
    w = np.asarray(weights, dtype=np.float64)
    loads = [w[p].sum() for p in parts]
    return float(max(loads) / (sum(loads) / len(loads)))
