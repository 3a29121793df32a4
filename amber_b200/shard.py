"""Multi-GPU host logic: one process per GPU, no exchange on the data path.

Two ways to use N GPUs, both without a collective on the data path:

* replicas — every rank estimates its own realisation (``rank_seed``);
  `bench.py --gpus N` measures this (weak scaling);
* triangle sharding — one realisation, its closed triangles split across
  ranks (strong scaling, `bench.py --shard`, `amber_gpu` under RANK /
  WORLD_SIZE).  A triangle is always computed whole on one rank, so every
  lag array is bit-identical to the single-rank one and no partial sums
  cross ranks; the results are gathered on rank 0 (host gather, ≤ 1 MB per
  triangle) or, for the drop-in executable, each rank writes its own
  triangles' files.

The plan.  A triangle costs total_vcp·Ng1(r1)² lag-triple products, and
total_vcp is the same for every triangle of a realisation, so the cost is
Ng1(r1)² per triangle.  Triangles of one r1 group share that group's ring
maps, which a rank builds once for all the group's triangles it holds
(charged as 1/25 of the group's contraction cost: about 4 % on the
single-realisation workload).  A group whose cost is above 1/N of the total is split into
⌈cost / (total/N)⌉ parts of near-equal cost (its triangles dealt round
robin, largest first); every other group stays whole.  The parts are then
placed largest first on the least-loaded rank (LPT), each placement
charging the part's map building to its rank.  On the single-realisation
workload this plans 7.3× on 8 ranks (2.35× with whole groups only).
The library restates the plan in C (amber_cuda_shard_plan) for the drop-in
executable; both use integer arithmetic and plan identically.
"""
from __future__ import annotations

import numpy as np

MAP_FRACTION = 1 / 25  # map building of a group, as a fraction of the group's contraction cost


def rank_seed(base: int, rank: int) -> int:
    return int(base) + int(rank)


def _parts(tri: np.ndarray, ng1_of, nranks: int):
    """(cost, r1, [triangle indices], map cost) of every part: whole groups, or near-equal pieces of
    a group above 1/nranks of the total.  Integer arithmetic throughout (ng1² per triangle), so the
    C restatement in the library (amber_cuda_shard_plan) plans identically."""
    groups = {}
    for t, r1 in enumerate(tri[:, 0].tolist()):
        groups.setdefault(int(r1), []).append(t)
    cost1 = {r1: int(ng1_of(r1)) ** 2 for r1 in groups}
    gcost = {r1: len(ts) * cost1[r1] for r1, ts in groups.items()}
    total = sum(gcost.values())
    parts = []
    for r1 in sorted(groups):
        ts = groups[r1]
        m = max(1, min(len(ts), -(-(gcost[r1] * nranks) // max(total, 1))))
        for j in range(m):
            piece = ts[j::m]
            parts.append((len(piece) * cost1[r1], r1, piece, gcost[r1]))
    return parts


def plan(tri: np.ndarray, ng1_of, nranks: int):
    """Assign triangles to ranks.  ``tri`` [n, 3] (r1, r2, r3); ``ng1_of(r1)`` gives the map side.
    Returns a list (per rank) of sorted triangle indices; every triangle appears exactly once, and
    the plan depends only on ``tri``, ``ng1_of`` and ``nranks`` (every rank computes the same)."""
    tri = np.asarray(tri).reshape(-1, 3)
    load = [0] * nranks  # 25 × contraction cost + map costs (the map charge is 1/25 of a group)
    out = [[] for _ in range(nranks)]
    # largest part first; ties broken by r1 then first triangle, so the order is total
    for cost, r1, piece, map_cost in sorted(_parts(tri, ng1_of, nranks), key=lambda p: (-p[0], p[1], p[2][0])):
        k = min(range(nranks), key=lambda i: (load[i], i))
        out[k].extend(piece)
        load[k] += 25 * cost + map_cost
    return [sorted(ts) for ts in out]


def plan_native(tri: np.ndarray, ng1_of, nranks: int):
    """The same plan from the library (amber_cuda_shard_plan, what the drop-in executable runs)."""
    import ctypes
    from . import load_library
    tri = np.asarray(tri).reshape(-1, 3)
    r1 = np.ascontiguousarray(tri[:, 0], dtype=np.int32)
    ng = np.ascontiguousarray([int(ng1_of(int(r))) for r in r1], dtype=np.int64)
    rank_of = np.zeros(max(len(r1), 1), dtype=np.int32)
    L = load_library()
    rc = L.amber_cuda_shard_plan(len(r1), r1.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                 ng.ctypes.data_as(ctypes.POINTER(ctypes.c_long)), int(nranks),
                                 rank_of.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
    if rc != 0:
        raise ValueError(f"amber_cuda_shard_plan failed ({rc})")
    return [sorted(int(i) for i in np.nonzero(rank_of[:len(r1)] == k)[0]) for k in range(nranks)]


def planned_speedup(tri: np.ndarray, ng1_of, nranks: int) -> float:
    """Single-rank cost over the most loaded rank's cost under ``plan``: contraction ng1² per
    triangle, map building 1/25 of a group's cost on every rank that holds part of the group."""
    tri = np.asarray(tri).reshape(-1, 3)
    cost1 = {r1: int(ng1_of(r1)) ** 2 for r1 in set(tri[:, 0].tolist())}
    gcost = {r1: int((tri[:, 0] == r1).sum()) * c for r1, c in cost1.items()}
    total = sum(gcost.values()) * (1 + MAP_FRACTION)
    worst = 0.0
    for ts in plan(tri, ng1_of, nranks):
        held = {int(tri[t, 0]) for t in ts}
        c = sum(cost1[int(tri[t, 0])] for t in ts) + MAP_FRACTION * sum(gcost[r1] for r1 in held)
        worst = max(worst, c)
    return total / worst if worst > 0 else 1.0


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
