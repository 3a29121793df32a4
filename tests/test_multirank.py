"""N > 1 host path on CPU: two gloo ranks shard one realisation's triangles
(groups above 1/N of the cost split, LPT over the parts) and gather the lag
arrays on rank 0; the compute step is the CPU oracle here (the GPU kernels
are covered by the gpu tests)."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle
from amber_b200 import shard, synth


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _case(kind):
    if kind == "split":
        # the largest ring's group (Ng1 = 104 against 38-72) holds over half the work: on two
        # ranks it is split, so both ranks compute triangles of the same r1 group
        return synth.tiny(32, 8, seed=3, nbins=4, hi=14.0, nc10=3)
    # six bins of milder growth (Ng1 36-92): every group stays whole on two ranks
    return synth.tiny(32, 8, seed=3, nbins=6, hi=12.0, nc10=3)


def _worker(rank, world, port, out_path, kind):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    real = _case(kind)
    gvn, ntn = oracle.normalize(real.gv, real.counts)
    rdata = oracle.calcr(ntn, real.ulow, real.uhigh)
    tri = rdata[:, :3].astype(int)
    ng = lambda r1: oracle.ng1(real.uhigh[r1], real.du)

    def compute(idx):
        _, res = oracle.estimate(real, version=1, tri_subset=idx)
        return {i: r["bldnu"] for i, r in zip(idx, res)}

    def gather(obj):
        parts = [None] * world
        dist.all_gather_object(parts, obj)
        return parts

    got = shard.estimate_sharded(tri, ng, compute, rank, world, gather)
    if rank == 0:
        np.save(out_path, np.stack(got))
    dist.barrier()
    dist.destroy_process_group()


def test_plan_covers_every_triangle_once_and_splits_only_large_groups():
    lo, hi = synth.log_edges(2.0, 120.0, 16)
    tri = oracle.triangles(lo, hi)
    ng = lambda r1: oracle.ng1(hi[r1], 0.5)
    cost = {r1: sum(ng(t[0]) ** 2 for t in tri if t[0] == r1) for r1 in set(tri[:, 0].tolist())}
    total = sum(cost.values())
    for world in (1, 2, 3, 8):
        parts = shard.plan(tri, ng, world)
        assert parts == shard.plan(tri, ng, world)  # deterministic: every rank plans the same
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(tri)))
        for r1, c in cost.items():
            holders = [k for k, p in enumerate(parts) if any(tri[i][0] == r1 for i in p)]
            if c * (1 + shard.MAP_FRACTION) <= total * (1 + shard.MAP_FRACTION) / world:
                assert len(holders) == 1, (world, r1, holders)  # a group within 1/N stays whole
    costs = [sum(ng(tri[i][0]) ** 2 for i in p) for p in shard.plan(tri, ng, 2)]
    assert max(costs) <= 1.1 * min(costs)


def test_planned_strong_scaling_of_the_single_realisation_workload():
    """Closed triangles of the single-realisation workload (256², 16 bins 2-120 cells): the plan
    reaches at least 6.5x on 8 ranks (whole r1 groups alone reach 2.35x: one group holds 43 %
    of the work)."""
    real = synth.config2(seed=1)
    _, ntn = oracle.normalize(real.gv, real.counts)
    tri = oracle.calcr(ntn, real.ulow, real.uhigh)[:, :3].astype(int)
    ng = lambda r1: oracle.ng1(real.uhigh[r1], real.du)
    assert shard.planned_speedup(tri, ng, 8) >= 6.5
    assert shard.planned_speedup(tri, ng, 2) >= 1.9


@pytest.mark.parametrize("kind", ["whole", "split"])
def test_two_gloo_ranks_reassemble_the_single_rank_result(tmp_path, kind):
    real = _case(kind)
    _, ntn = oracle.normalize(real.gv, real.counts)
    tri = oracle.calcr(ntn, real.ulow, real.uhigh)[:, :3].astype(int)
    ng = lambda r1: oracle.ng1(real.uhigh[r1], real.du)
    parts = shard.plan(tri, ng, 2)
    split = [r1 for r1 in set(tri[:, 0].tolist()) if all(any(tri[i][0] == r1 for i in p) for p in parts)]
    assert bool(split) == (kind == "split"), split
    out = str(tmp_path / "lags.npy")
    mp.start_processes(_worker, args=(2, _free_port(), out, kind), nprocs=2, join=True, start_method="spawn")
    got = np.load(out)
    _, res = oracle.estimate(real, version=1)
    ref = np.stack([r["bldnu"] for r in res])
    assert got.shape == ref.shape
    assert np.array_equal(got, ref)


def test_library_plan_equals_the_python_plan():
    """amber_cuda_shard_plan (the C restatement the drop-in executable runs under RANK/WORLD_SIZE)
    and shard.plan assign every triangle to the same rank (host-only call, no GPU)."""
    lo, hi = synth.log_edges(2.0, 120.0, 16)
    cases = [(oracle.triangles(lo, hi), lambda r1: oracle.ng1(hi[r1], 0.5))]
    lo4, hi4 = synth.log_edges(2.0, 240.0, 24)
    cases.append((oracle.triangles(lo4, hi4), lambda r1: oracle.ng1(hi4[r1], 0.5)))
    for tri, ng in cases:
        for world in (1, 2, 3, 5, 8, 16):
            assert shard.plan_native(tri, ng, world) == shard.plan(tri, ng, world), world


def test_library_plan_equals_the_python_plan_on_random_lists():
    """Seeded random triangle lists: uneven r1 groups, map sides with ties and large spreads,
    unsorted input and 1-16 ranks.  The C and Python plans agree triangle for triangle, each covers
    every triangle once, and a group within 1/N of the cost stays on one rank."""
    rng = np.random.default_rng(20261204)
    for case in range(150):
        nr = int(rng.integers(1, 25))
        ntri = int(rng.integers(1, 400))
        side = np.sort(rng.integers(8, 1500, size=nr))
        if case % 3 == 0:
            side[:] = side[0]  # every group the same map side: ties throughout the ordering
        r1 = rng.integers(0, nr, size=ntri)
        tri = np.stack([r1, r1, r1], axis=1)
        ng = lambda r, side=side: int(side[r])
        world = int(rng.integers(1, 17))
        want = shard.plan(tri, ng, world)
        assert shard.plan_native(tri, ng, world) == want, (case, world)
        assert sorted(i for p in want for i in p) == list(range(ntri))
        cost = {}
        for r in r1.tolist():
            cost[r] = cost.get(r, 0) + ng(r) ** 2
        total = sum(cost.values())
        for r, c in cost.items():
            if c * world <= total:
                holders = [k for k, p in enumerate(want) if any(r1[i] == r for i in p)]
                assert len(holders) == 1, (case, r, holders)


def test_library_plan_rejects_bad_arguments():
    import ctypes
    from amber_b200 import load_library
    L = load_library()
    r1 = (ctypes.c_int * 2)(0, 1)
    ng = (ctypes.c_long * 2)(10, 12)
    out = (ctypes.c_int * 2)()
    assert L.amber_cuda_shard_plan(2, r1, ng, 0, out) == -1       # no ranks
    bad = (ctypes.c_long * 2)(10, 0)
    assert L.amber_cuda_shard_plan(2, r1, bad, 2, out) == -1      # a map side of 0
    assert L.amber_cuda_shard_plan(2, r1, ng, 3, out) == 0        # more ranks than triangles: fine
    assert sorted(out) == [0, 1]
    assert L.amber_cuda_shard_plan(0, None, None, 4, None) == 0   # nothing to plan


def test_ranks_get_the_same_ensemble_shapes_with_their_own_seeds():
    """Weak scaling: every rank's 64-realisation ensemble has the same grid sides, channel counts,
    bins and lag windows; only the data seeds (and so the fields, sampling and flags) differ."""
    base = synth.config3_specs()
    for rank in (1, 7):
        other = synth.config3_specs(seed0=100 + 64 * rank)
        shape = lambda sp: (sp["nn"], sp["nc"], sp["nbins"], sp["ring_lo"], sp["ring_hi"], sp["nc10"], sp["flag_frac"])
        assert [shape(a) for a in base] == [shape(b) for b in other]
        assert not {a["seed"] for a in base} & {b["seed"] for b in other}


def test_sharded_gather_rejects_duplicates_and_gaps():
    """estimate_sharded on rank 0 refuses a gather in which a triangle arrives twice or not at all
    (host logic, no process group: the gather is a plain function)."""
    tri = np.array([[2, 1, 1], [2, 2, 1], [3, 1, 1], [3, 3, 2]])
    ng = lambda r1: 40 + 10 * r1
    compute = lambda idx: {i: i * 10 for i in idx}
    assert shard.estimate_sharded(tri, ng, compute, 0, 2, lambda obj: [compute(p) for p in shard.plan(tri, ng, 2)]) \
        == [0, 10, 20, 30]
    assert shard.estimate_sharded(tri, ng, compute, 1, 2, lambda obj: [obj, obj]) is None  # other ranks: nothing
    with pytest.raises(RuntimeError, match="computed twice"):
        shard.estimate_sharded(tri, ng, compute, 0, 2, lambda obj: [compute([0, 1, 2, 3]), compute([0])])
    with pytest.raises(RuntimeError, match="gathered 3 of 4"):
        shard.estimate_sharded(tri, ng, compute, 0, 2, lambda obj: [compute([0, 1]), compute([2])])


def test_rank_seeds_differ():
    assert len({shard.rank_seed(1, r) for r in range(8)}) == 8
