"""Multi-GPU host logic: one process per GPU, no exchange on the data path.

Two ways to use N GPUs, both without a collective on the data path:

* replicas — every rank estimates its own realisation (``rank_seed``);
  `bench.py --gpus N` measures this (weak scaling);
* triangle sharding — one realisation, its closed triangles split across
  ranks by r1 group (maps are built once per group, so a group is never
  split) with longest-processing-time assignment on the cost
  total_vcp·Ng1² per triangle; each rank computes its groups and the lag
  arrays are gathered on rank 0 (host gather, ≤ 1 MB per triangle).
"""
from __future__ import annotations

import numpy as np


def rank_seed(base: int, rank: int) -> int:
    return int(base) + int(rank)


def plan(tri: np.ndarray, ng1_of, nranks: int):
    """Assign triangles to ranks.  ``tri`` [n, 3] (r1, r2, r3); ``ng1_of(r1)``
    gives the map side.  Returns a list (per rank) of triangle indices."""
    tri = np.asarray(tri).reshape(-1, 3)
    groups = {}
    for t, r1 in enumerate(tri[:, 0].tolist()):
        groups.setdefault(int(r1), []).append(t)
    cost = {r1: len(ts) * float(ng1_of(r1)) ** 2 for r1, ts in groups.items()}
    load = [0.0] * nranks
    out = [[] for _ in range(nranks)]
    for r1 in sorted(groups, key=lambda r: -cost[r]):
        k = int(np.argmin(load))
        out[k].extend(groups[r1])
        load[k] += cost[r1]
    return [sorted(ts) for ts in out]


def estimate_sharded(tri: np.ndarray, ng1_of, compute, rank: int, world: int, gather):
    """Run this rank's share of ``tri`` with ``compute(indices) -> {index: result}``
    and gather everything on rank 0 with ``gather(obj) -> list`` (e.g.
    ``torch.distributed.all_gather_object`` wrapped).  Rank 0 returns the
    results in triangle order; other ranks return None."""
    mine = plan(tri, ng1_of, world)[rank]
    local = compute(mine) if mine else {}
    parts = gather(local)
    if rank != 0:
        return None
    merged = {}
    for p in parts:
        for k, v in p.items():
            if k in merged:
                raise RuntimeError(f"triangle {k} computed twice")
            merged[k] = v
    if len(merged) != len(tri):
        raise RuntimeError(f"gathered {len(merged)} of {len(tri)} triangles")
    return [merged[i] for i in range(len(tri))]
