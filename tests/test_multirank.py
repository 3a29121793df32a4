"""N > 1 host path on CPU: two gloo ranks shard one realisation's triangles
(by r1 group, LPT) and gather the lag arrays on rank 0; the compute step is
the CPU oracle here (the GPU kernels are covered by the gpu tests)."""
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


def _worker(rank, world, port, out_path):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    real = synth.tiny(32, 8, seed=3, nbins=4, hi=14.0, nc10=3)
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


def test_plan_covers_every_triangle_once_and_balances():
    lo, hi = synth.log_edges(2.0, 120.0, 16)
    tri = oracle.triangles(lo, hi)
    ng = lambda r1: oracle.ng1(hi[r1], 0.5)
    for world in (1, 2, 3, 8):
        parts = shard.plan(tri, ng, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(tri)))
        for p in parts:  # an r1 group is never split
            for q in parts:
                if p is not q:
                    assert not ({tri[i][0] for i in p} & {tri[i][0] for i in q})
    costs = [sum(ng(tri[i][0]) ** 2 for i in p) for p in shard.plan(tri, ng, 2)]
    assert max(costs) <= 1.6 * min(costs)


def test_two_gloo_ranks_reassemble_the_single_rank_result(tmp_path):
    out = str(tmp_path / "lags.npy")
    mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    got = np.load(out)
    real = synth.tiny(32, 8, seed=3, nbins=4, hi=14.0, nc10=3)
    _, res = oracle.estimate(real, version=1)
    ref = np.stack([r["bldnu"] for r in res])
    assert got.shape == ref.shape
    assert np.array_equal(got, ref)


def test_rank_seeds_differ():
    assert len({shard.rank_seed(1, r) for r in range(8)}) == 8
