"""Batched requests (amber_cuda_enqueue / wait / result): ensembles of realisations of uneven
size and streams of requests run together on one GPU.

* Each request's lag arrays equal the single-realisation path's (same context precision) —
  a job's chunking and reduction grouping depend on the job only, so they are bit-identical.
* A request gives the same result alone and in a mix (the serving contract).
* The mixed-precision results hold the 1e-6 bound against the FP64 oracle, counts are exact.
"""
import numpy as np
import pytest

import oracle
from amber_b200 import synth

pytestmark = pytest.mark.gpu

TOL_MIXED = 1e-6


@pytest.fixture(scope="module")
def lib_built():
    from amber_b200 import build
    build.build()
    return True


def _ensemble():
    # uneven sides, channel counts (BN = 32 and 64 tiles), flag modes and lag widths
    return [
        synth.tiny(48, 16, seed=41, nbins=5, hi=21.0),
        synth.tiny(64, 40, seed=42, nbins=6, hi=28.0, flagged=[0, 1, 38, 39]),
        synth.tiny(32, 12, seed=43, nbins=4, hi=14.0, nc10=11),
        synth.tiny(56, 24, seed=44, nbins=5, hi=25.0, flagged=[3, 17]),
        synth.tiny(80, 72, seed=45, nbins=6, hi=36.0),
    ]


def _single(real, precision):
    import amber_b200
    rdata, res = amber_b200.estimate(real, precision=precision, version=2)
    bl = np.stack([r["bldnu"] for r in res]).reshape(len(res), -1)
    nt = np.stack([r["numtri"] for r in res]).reshape(len(res), -1)
    nd = np.stack([r["numdnu"] for r in res]).reshape(len(res), -1)
    return rdata, bl, nd, nt


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_ensemble_equals_single_realisation_path(precision, lib_built):
    import amber_b200
    reals = _ensemble()
    with amber_b200.Estimator(precision=precision) as est:
        eng = amber_b200.Engine(est)
        tickets = [eng.enqueue(r, want_v2=True) for r in reals]
        outs = [eng.result(t, r) for t, r in zip(tickets, reals)]
        st = eng.stats()
    assert st["requests_done"] == len(reals) and st["queued"] == 0 and st["active"] == 0
    if precision == "mixed":
        assert st["max_active"] >= 2  # requests shared rounds
    for r, (rd, bl, nd, nt, lat) in zip(reals, outs):
        srd, sbl, snd, snt = _single(r, precision)
        np.testing.assert_array_equal(rd[:, :3], srd[:, :3])
        np.testing.assert_allclose(rd[:, 3], srd[:, 3], rtol=1e-12)
        np.testing.assert_array_equal(nd, snd)
        np.testing.assert_array_equal(bl, sbl)
        np.testing.assert_array_equal(nt, snt)
        assert lat > 0


def test_ensemble_mixed_vs_oracle(lib_built):
    import amber_b200
    reals = _ensemble()[:3]
    with amber_b200.Estimator(precision="mixed") as est:
        eng = amber_b200.Engine(est)
        tickets = [eng.enqueue(r, want_v2=True) for r in reals]
        outs = [eng.result(t, r) for t, r in zip(tickets, reals)]
    for r, (rd, bl, nd, nt, _) in zip(reals, outs):
        ordata, ores = oracle.estimate(r, version=2, with_absscale=True)
        np.testing.assert_array_equal(rd[:, :3], ordata[:, :3])
        for i, o in enumerate(ores):
            np.testing.assert_array_equal(nd[i], o["numdnu"].reshape(-1))
            e = np.abs(bl[i] - o["bldnu"].reshape(-1)) / (o["absscale"].reshape(-1) + 1e-300)
            assert e.max() <= TOL_MIXED, e.max()
            ei = np.abs(nt[i] - o["numtri"].reshape(-1)) / (o["absscale_i"].reshape(-1) + 1e-300)
            assert ei.max() <= TOL_MIXED, ei.max()


def test_result_same_alone_and_in_a_mix(lib_built):
    """The serving contract: a request's result does not depend on what shares the GPU with it."""
    import amber_b200
    reals = _ensemble()
    probe = reals[1]
    with amber_b200.Estimator(precision="mixed") as est:
        eng = amber_b200.Engine(est)
        alone = eng.result(eng.enqueue(probe), probe)
        # the same request again, now arriving between others of different sizes
        t_before = [eng.enqueue(r) for r in reals[2:]]
        t_probe = eng.enqueue(probe)
        t_after = [eng.enqueue(r) for r in reals[:1]]
        mixed = eng.result(t_probe, probe)
        for t, r in zip(t_before + t_after, reals[2:] + reals[:1]):
            eng.result(t, r)
    for a, b in zip(alone[:4], mixed[:4]):
        np.testing.assert_array_equal(a, b)


def test_bad_request_and_timeout(lib_built):
    import amber_b200
    bad = synth.tiny(32, 8, seed=5, nbins=3, hi=14.0)
    bad.uhigh = np.array(bad.uhigh, dtype=float)
    bad.uhigh[-1] = 40.0  # beyond N1/2: rejected before any GPU work
    with amber_b200.Estimator(precision="mixed") as est:
        eng = amber_b200.Engine(est)
        with pytest.raises(amber_b200.AmberError) as e:
            eng.enqueue(bad)
        assert e.value.code == -1
        big = synth.tiny(128, 64, seed=6, nbins=8, hi=60.0)
        t = eng.enqueue(big)
        try:
            n = eng.wait(t, timeout_ms=0)  # may already be done on a fast GPU
        except amber_b200.AmberError as ex:
            assert ex.code == -4
        n = eng.wait(t, timeout_ms=-1)
        assert n > 0
        eng.result(t, big)
        with pytest.raises(amber_b200.AmberError):
            eng.wait(t)  # the result has been collected: unknown ticket


def _cyl_reals():
    # nc10 = 19, 35, 11 with the default cut of 8: every folded, cut lag cell has triplets
    e = _ensemble()
    return [e[1], e[4], synth.tiny(48, 24, seed=46, nbins=5, hi=21.0, nc10=11)]


def test_engine_returns_cylindrical_bispectra(lib_built):
    """Requests that ask for cylindrical bispectra get what the single-realisation path's
    amber_cuda_cyl_bs gives (v1: divided by the file Num, v2: mask sums and window), and those
    match the oracle's restatement of the reference's analysis on the same lag arrays."""
    import amber_b200
    reals = _cyl_reals()
    k = amber_b200.reference_cylbs_constants()
    with amber_b200.Estimator(precision="mixed") as est:
        eng = amber_b200.Engine(est)
        t1 = [eng.enqueue(r, want_v2=False, cyl_bs={}) for r in reals]
        t2 = [eng.enqueue(r, want_v2=True, cyl_bs=dict(window=True, denominator="mask")) for r in reals]
        o1 = [eng.result(t, r, want_v2=False) for t, r in zip(t1, reals)]
        o2 = [eng.result(t, r, want_v2=True) for t, r in zip(t2, reals)]
    with amber_b200.Estimator(precision="mixed") as est:
        for r, a, b in zip(reals, o1, o2):
            const = dict(nc10=r.nc10, n_cut=k["n_cut"], mabs_norm=k["mabs_norm"], rc=k["rc"], rc_prime=k["rc_prime"],
                         dnu=k["dnu_mhz"])
            nclen = 2 * r.nc10 + 1
            rdata, _ = amber_b200.estimate(r, version=1, est=est)
            num = est.file_num(rdata)
            single = est.cyl_bs(tri_div=num)
            assert a[5].shape == single.shape
            assert np.abs(a[5] - single).max() <= 1e-12 * np.abs(single).max()
            for i in range(len(rdata)):
                want = oracle.cyl_bs(a[1][i].reshape(nclen, nclen), a[2][i].reshape(nclen, nclen), div=num[i], **const)
                assert np.abs(a[5][i] - want).max() <= 1e-10 * np.abs(want).max()
            amber_b200.estimate(r, version=2, est=est)
            single = est.cyl_bs(window=True, denominator="mask")
            assert np.abs(b[5] - single).max() <= 1e-12 * np.abs(single).max()
            for i in range(len(rdata)):
                want = oracle.cyl_bs(b[1][i].reshape(nclen, nclen), b[3][i].reshape(nclen, nclen), window=True,
                                     **const)
                assert np.abs(b[5][i] - want).max() <= 1e-10 * np.abs(want).max()


def test_engine_rejects_bad_cylindrical_parameters(lib_built):
    import amber_b200
    r = _cyl_reals()[2]
    with amber_b200.Estimator(precision="mixed") as est:
        eng = amber_b200.Engine(est)
        for kw, v2 in ((dict(n_cut=12), True), (dict(denominator="mask"), False), (dict(mabs_norm=0.0), True)):
            with pytest.raises(amber_b200.AmberError) as e:
                eng.enqueue(r, want_v2=v2, cyl_bs=kw)
            assert e.value.code == -1
        assert eng.stats()["queued"] == 0


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_device_resident_cube_equals_host_cube(precision, lib_built):
    """A request whose summed grid and counts already sit in device memory (``inputs_on_device``)
    is read in place: its results equal those of the same request from host buffers, bit for bit,
    and the caller's device buffers come back unchanged."""
    import torch
    import amber_b200
    reals = _ensemble()[:3]
    cubes = [(torch.from_numpy(np.ascontiguousarray(r.gv).view(np.float64)).cuda(),
              torch.from_numpy(np.ascontiguousarray(r.counts, dtype=np.float64)).cuda()) for r in reals]
    before = [(a.clone(), b.clone()) for a, b in cubes]
    with amber_b200.Estimator(precision=precision) as est:
        eng = amber_b200.Engine(est)
        host = [eng.result(eng.enqueue(r), r) for r in reals]
        tickets = [eng.enqueue(r, device_cube=(a.data_ptr(), b.data_ptr())) for r, (a, b) in zip(reals, cubes)]
        dev = [eng.result(t, r) for t, r in zip(tickets, reals)]
    for h, d in zip(host, dev):
        for x, y in zip(h[:4], d[:4]):
            np.testing.assert_array_equal(x, y)
    for (a, b), (a0, b0) in zip(cubes, before):
        assert torch.equal(a, a0) and torch.equal(b, b0)
