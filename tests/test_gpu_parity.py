"""Parity of libamber_cuda against the oracle and the reference's own outputs.

Tolerances (from the contract of this path):
* FP64 plain path: ≤ 1e-10 relative to Σ|products| per lag cell vs the FP64
  oracle (and the reference's FP64 build via the golden fixtures);
* mixed-precision path (int8 digits, exact int32 accumulation): ≤ 1e-6
  relative to Σ|products| per lag cell;
* split-BF16×3 path (FP32 accumulation, kept for comparison): ≤ 3e-5 — it
  cannot hold 1e-6 on the coherent v2 sampling-mask sums;
* triplet counts, the closed-triangle list and gridding: bit-exact.
"""
import glob
import os

import numpy as np
import pytest

import oracle
from amber_b200 import synth

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL = {"fp64": 1e-10, "mixed": 1e-6, "bf16x3": 3e-5}


def _real_from(z):
    return synth.Realisation(nn=z["gv"].shape[0], nc=z["gv"].shape[2], du=float(z["du"]), flag_key=int(z["flag_key"]),
                             gv=z["gv"], counts=z["counts"], uf_chans=z["uf_chans"], ulow=z["ulow"],
                             uhigh=z["uhigh"], nc10=int(z["nc10"]), seed=0)


@pytest.fixture(scope="module")
def lib_built():
    from amber_b200 import build
    build.build()
    return True


def _run(real, precision, version, est_cls):
    from amber_b200 import estimate
    return estimate(real, precision=precision, version=version)


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "est_*.npz"))))
@pytest.mark.parametrize("precision", ["fp64", "mixed", "bf16x3"])
def test_estimator_vs_reference_golden(path, precision, lib_built):
    import amber_b200
    z = np.load(path)
    real = _real_from(z)
    rdata, res = amber_b200.estimate(real, precision=precision, version=2)
    _, ores = oracle.estimate(real, version=2, with_absscale=True)
    np.testing.assert_array_equal(rdata[:, :3], z["rdata"][:, :3])
    np.testing.assert_allclose(rdata[:, 3], z["rdata"][:, 3], rtol=1e-10, atol=1e-10 * np.abs(z["rdata"][:, 3]).max())
    tol = TOL[precision]
    for i, r in enumerate(res):
        np.testing.assert_array_equal(r["numdnu"], z["numdnu"][i])
        e = np.abs(r["bldnu"] - z["bldnu64"][i]) / (ores[i]["absscale"] + 1e-300)
        assert e.max() <= tol, (i, e.max())
        ei = np.abs(r["numtri"] - z["numtri_v2"][i]) / (ores[i]["absscale_i"] + 1e-300)
        assert ei.max() <= tol, (i, ei.max())


@pytest.mark.parametrize("precision", ["fp64", "mixed", "bf16x3"])
@pytest.mark.parametrize("nn,nc,nbins,hi,nc10,flagged,seed", [
    (48, 16, 5, 22.0, 7, None, 31),
    (64, 20, 6, 30.0, 9, [0, 1, 18, 19], 32),
    (56, 12, 4, 26.0, 11, [3], 33),  # nc10 = nc - 1: the widest lag window
    (32, 6, 3, 14.0, 0, None, 34),  # nc10 = 0: the zero lag only
    (36, 12, 3, 16.0, 5, [0, 1, 2, 4, 6, 7, 9, 11], 35),  # most channels flagged
])
def test_estimator_vs_oracle(precision, nn, nc, nbins, hi, nc10, flagged, seed, lib_built):
    import amber_b200
    real = synth.tiny(nn, nc, seed=seed, nbins=nbins, hi=hi, nc10=nc10, flagged=flagged)
    rdata, res = amber_b200.estimate(real, precision=precision, version=2)
    ordata, ores = oracle.estimate(real, version=2, with_absscale=True)
    np.testing.assert_array_equal(rdata[:, :3], ordata[:, :3])
    tol = TOL[precision]
    for r, o in zip(res, ores):
        np.testing.assert_array_equal(r["numdnu"], o["numdnu"])
        e = np.abs(r["bldnu"] - o["bldnu"]) / (o["absscale"] + 1e-300)
        assert e.max() <= tol, e.max()
        ei = np.abs(r["numtri"] - o["numtri"]) / (o["absscale_i"] + 1e-300)
        assert ei.max() <= tol, ei.max()


def test_mixed_vs_fp64_full_size(lib_built):
    """The single-realisation workload (256² grid, 128 channels, 16 bins) at full size: the
    mixed path against the FP64 path on the same GPU, per lag cell, scaled by Σ|products|
    (the FP64 path with |D| maps).  Covers the largest maps (Ng1 = 740, 5.5e5 pixels), where
    the sampling-mask sums are dominated by one peak pixel and the digit errors of every
    other pixel add up; plus a spread of smaller triangles."""
    import amber_b200
    real = synth.config2(seed=1)
    with amber_b200.Estimator(precision="mixed") as est:
        est.load_grid(real.gv, real.counts, real.du, real.flag_key)
        est.set_rings(real.ulow, real.uhigh)
        est.set_channels(real.nc10, real.uf_chans)
        tri = est.calcr()[:, :3].astype(np.int32)
        sample = np.concatenate([tri[::31], tri[-3:]])
        est.run(sample, want_v2=True)
        m_bl, _, m_nt = est.fetch(want_v2=True)
    out = {}
    for prec in ("fp64", "fp64_abs"):
        with amber_b200.Estimator(precision=prec) as e64:
            e64.load_grid(real.gv, real.counts, real.du, real.flag_key)
            e64.set_rings(real.ulow, real.uhigh)
            e64.set_channels(real.nc10, real.uf_chans)
            e64.run(sample, want_v2=True)
            out[prec] = e64.fetch(want_v2=True)
    (bl, _, nt), (abl, _, ant) = out["fp64"], out["fp64_abs"]
    ed = (np.abs(m_bl - bl) / (abl + 1e-300)).reshape(len(sample), -1).max(axis=1)
    ei = (np.abs(m_nt - nt) / (ant + 1e-300)).reshape(len(sample), -1).max(axis=1)
    print("max rel err per triangle, D sums:", ed, "mask sums:", ei)
    assert ed.max() <= TOL["mixed"], (sample[int(ed.argmax())], ed.max())
    assert ei.max() <= TOL["mixed"], (sample[int(ei.argmax())], ei.max())


def test_isosceles_symmetry_full_size(lib_built):
    """A size-independent property at full size: for a triangle with r2 = r3 the two outer maps are
    the same, so T_p1[p2, p3] is symmetric and so are the lag arrays, bldnu[Δ2, Δ3] = bldnu[Δ3, Δ2]
    (and the mask sums).  The plain FP64 path keeps it to rounding; the mixed path forms the two
    operands differently (plain digits and product digits), so there it holds to twice its error
    bound.  Counts are symmetric exactly."""
    import amber_b200
    real = synth.config2(seed=1)
    out = {}
    for prec in ("mixed", "fp64", "fp64_abs"):
        with amber_b200.Estimator(precision=prec) as est:
            est.load_grid(real.gv, real.counts, real.du, real.flag_key)
            est.set_rings(real.ulow, real.uhigh)
            est.set_channels(real.nc10, real.uf_chans)
            tri = est.calcr()[:, :3].astype(np.int32)
            iso = tri[(tri[:, 1] == tri[:, 2]) & (tri[:, 0] != tri[:, 1])]
            sample = iso[-3:]  # the largest maps with r2 = r3 < r1
            est.run(sample, want_v2=True)
            out[prec] = est.fetch(want_v2=True)
    (ab, _, at) = out["fp64_abs"]
    for prec, tol in (("fp64", 1e-10), ("mixed", 2 * TOL["mixed"])):
        bl, nd, nt = out[prec]
        for i in range(len(bl)):
            np.testing.assert_array_equal(nd[i], nd[i].T)
            assert (np.abs(bl[i] - bl[i].T) <= tol * ab[i] + 1e-300).all(), prec
            assert (np.abs(nt[i] - nt[i].T) <= tol * at[i] + 1e-300).all(), prec


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_unit_size_changes_only_rounding(precision, lib_built):
    """The contraction's work units (runs of 256-pixel blocks, each summed into a partial tile of
    its own) set only the FP64 summation grouping.  One-block units (chunk_px = 256) on the
    Ng1 = 354 triangle of the single-realisation workload (490 blocks) against the default units:
    counts identical, lag arrays equal to FP64 rounding."""
    import amber_b200
    real = synth.config2(seed=1)
    out = []
    for chunk_px in (0, 256):
        with amber_b200.Estimator(precision=precision, chunk_px=chunk_px) as est:
            est.load_grid(real.gv, real.counts, real.du, real.flag_key)
            est.set_rings(real.ulow, real.uhigh)
            est.set_channels(real.nc10, real.uf_chans)
            tri = est.calcr()[:, :3].astype(np.int32)
            est.run(tri[[140]], want_v2=True)
            out.append(est.fetch(want_v2=True))
    (b0, n0, t0), (b1, n1, t1) = out
    np.testing.assert_array_equal(n0, n1)
    np.testing.assert_allclose(b1, b0, rtol=0, atol=1e-12 * np.abs(b0).max())
    np.testing.assert_allclose(t1, t0, rtol=0, atol=1e-12 * np.abs(t0).max())


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("nn,nc,nbins,hi,nc10,flagged,seed", [
    (32, 100, 2, 10.0, 40, [5, 50], 54),                         # nclen = 81: one tile, no anchor packing
    (32, 150, 2, 10.0, 70, [3, 77, 149], 53),                    # nclen = 141: 2 × 2 tiles, two anchor blocks
    (32, 140, 2, 10.0, 60, list(range(128, 140)), 55),           # the second anchor block has no anchors
])
def test_estimator_vs_oracle_wide_windows(precision, nn, nc, nbins, hi, nc10, flagged, seed, lib_built):
    """Lag windows wider than one 64-row anchor packing: a single 128-row tile, a 2 × 2 tile grid with
    channels in two anchor blocks, and an anchor block whose channels are all flagged."""
    import amber_b200
    real = synth.tiny(nn, nc, seed=seed, nbins=nbins, hi=hi, nc10=nc10, flagged=flagged)
    rdata, res = amber_b200.estimate(real, precision=precision, version=2)
    ordata, ores = oracle.estimate(real, version=2, with_absscale=True)
    np.testing.assert_array_equal(rdata[:, :3], ordata[:, :3])
    tol = TOL[precision]
    for r, o in zip(res, ores):
        np.testing.assert_array_equal(r["numdnu"], o["numdnu"])
        e = np.abs(r["bldnu"] - o["bldnu"]) / (o["absscale"] + 1e-300)
        assert e.max() <= tol, e.max()
        ei = np.abs(r["numtri"] - o["numtri"]) / (o["absscale_i"] + 1e-300)
        assert ei.max() <= tol, ei.max()


@pytest.mark.skipif(not oracle.ref_available(), reason="reference build (oracle/_ref) not present")
def test_config1_full_vs_reference_build(tmp_path, lib_built):
    """The reference's own CPU-runnable case at full size (128² grid, 32 channels, 8 bins, all 46
    closed triangles, v1): the reference's sources built with FP64 floats (oracle/_ref/ref_amber64)
    run on the host cores, and its bsout files are the standard.  Counts and the triangle list are
    exact, the plain FP64 path is within 1e-10 and the mixed path within 1e-6 of Σ|products| per
    lag cell."""
    import amber_b200
    from amber_b200 import formats
    real = synth.config1()
    _, res_path = oracle.run_ref_amber(real, str(tmp_path), version=1, fp64=True)
    ref_rd = formats.read_closed_rings(res_path)
    nclen = real.nclen
    out = {}
    for prec in ("fp64", "fp64_abs", "mixed"):
        rdata, res = amber_b200.estimate(real, precision=prec, version=1)
        out[prec] = (rdata, res)
    rdata, res64 = out["fp64"]
    np.testing.assert_array_equal(rdata[:, :3], ref_rd[:, :3])
    np.testing.assert_allclose(rdata[:, 3], ref_rd[:, 3], rtol=1e-10)
    assert len(res64) == 46
    for i, r in enumerate(res64):
        name = formats.bsout_name(1, r["r1"], r["r2"], r["r3"], 1)
        ntri, num, bl, nd = formats.read_bsout_v1(f"{res_path}/{name}", nclen, bl_dtype=np.float64)
        scale = out["fp64_abs"][1][i]["bldnu"].reshape(nclen, nclen) + 1e-300
        np.testing.assert_array_equal(r["numdnu"].reshape(nclen, nclen), nd)
        e64 = np.abs(r["bldnu"].reshape(nclen, nclen) - bl) / scale
        assert e64.max() <= TOL["fp64"], (name, e64.max())
        em = np.abs(out["mixed"][1][i]["bldnu"].reshape(nclen, nclen) - bl) / scale
        assert em.max() <= TOL["mixed"], (name, em.max())
        ng = r["ng1"]
        np.testing.assert_allclose(num, (ng / real.nn) ** 2 * r["rdata_num"], rtol=1e-12)
        np.testing.assert_allclose(ntri, num / ng**2, rtol=1e-12)


def test_triangle_v1_v2_file_scalars(lib_built):
    import amber_b200
    z = np.load(os.path.join(GOLDEN, "est_flagged48.npz"))
    real = _real_from(z)
    with amber_b200.Estimator(precision="fp64") as est:
        est.load_grid(real.gv, real.counts, real.du, real.flag_key)
        est.set_rings(real.ulow, real.uhigh)
        est.set_channels(real.nc10, real.uf_chans)
        rdata = est.calcr()
        for rp in (0, len(rdata) // 2, len(rdata) - 1):
            r1, r2, r3 = (int(v) for v in rdata[rp, :3])
            ntri, num, bl, nd = est.triangle_v1(r1, r2, r3, rdata[rp, 3])
            np.testing.assert_allclose(num, z["num"][rp], rtol=1e-10)
            np.testing.assert_allclose(ntri, z["ntri"][rp], rtol=1e-10)
            assert nd.dtype == np.int32 and np.array_equal(nd, z["numdnu"][rp])
            assert np.abs(bl - z["bldnu64"][rp]).max() <= 1e-6 * np.abs(z["bldnu64"][rp]).max()
            inv, bl2, nd2 = est.triangle_v2(r1, r2, r3)
            assert inv == z["inv_ng"][rp]
            assert nd2.dtype == np.float32


def test_pointer_per_cell_load_equals_packed(lib_built):
    import amber_b200
    real = synth.tiny(32, 8, seed=5, nbins=4, hi=14.0, nc10=3)
    outs = []
    for form in ("packed", "cells"):
        with amber_b200.Estimator(precision="fp64") as est:
            if form == "packed":
                est.load_grid(real.gv, real.counts, real.du, real.flag_key)
            else:
                est.load_grid_cells(real.gv, real.counts, real.du, real.flag_key)
            est.set_rings(real.ulow, real.uhigh)
            est.set_channels(real.nc10)
            rdata = est.calcr()
            outs.append(est.triangles(rdata[:, :3].astype(np.int32))[0])
    assert np.array_equal(outs[0], outs[1])


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "grid_*.npz"))))
def test_gridding_bit_exact_vs_reference(path, lib_built):
    import amber_b200
    z = np.load(path)
    n_coll = int(z["n_collapse"]) if "n_collapse" in z.files else 1
    with amber_b200.Estimator(precision="fp64") as est:
        gv, nt = est.grid_vis(int(z["nn"]), z["data"].shape[1], float(z["du"]), float(z["umax"]), z["nu0"],
                              int(z["flag_key"]), z["randpar"], z["data"], n_collapse=n_coll)
    assert np.array_equal(gv.real, z["gv"].real) and np.array_equal(gv.imag, z["gv"].imag)
    assert np.array_equal(nt, z["ntig"])


def test_gridding_edges(lib_built):
    """No records at all (an all-zero grid), and a collapse of every channel into one."""
    import amber_b200
    nn, du, nc = 32, 0.5, 8
    randpar, data = synth.make_visibilities(nn, du, nc, 400, 78)
    nu0 = np.float32(synth.NU0)
    with amber_b200.Estimator() as est:
        g, n = est.grid_vis(nn, nc, du, 7.0, nu0, 1, randpar[:0], data[:0])
        assert g.shape == (nn, nn // 2 + 1, nc) and not g.any() and not n.any()
        g1, n1 = est.grid_vis(nn, nc, du, 7.0, nu0, 0, randpar, data, n_collapse=nc)
    g_o, n_o = oracle.collapse_channels(*oracle.grid_vis(nn, nc, du, 7.0, nu0, 0, randpar, data), nc)
    assert g1.shape[2] == 1 and np.array_equal(g1, g_o) and np.array_equal(n1, n_o)


def test_gridding_bit_exact_vs_oracle_large(lib_built):
    import amber_b200
    nn, du, nc = 128, 0.5, 24
    randpar, data = synth.make_visibilities(nn, du, nc, 60000, 77, dup_frac=0.6)
    for fk in (0, 1):
        g_o, n_o = oracle.grid_vis(nn, nc, du, 0.95 * du * nn / 2, np.float32(synth.NU0), fk, randpar, data)
        with amber_b200.Estimator() as est:
            g, n = est.grid_vis(nn, nc, du, 0.95 * du * nn / 2, np.float32(synth.NU0), fk, randpar, data)
        assert np.array_equal(g, g_o) and np.array_equal(n, n_o)


def test_error_paths(lib_built):
    import amber_b200
    from amber_b200 import AmberError
    real = synth.tiny(32, 8, seed=5, nbins=4, hi=14.0, nc10=3)
    with amber_b200.Estimator(precision="fp64") as est:
        with pytest.raises(AmberError) as e:
            est.calcr()
        assert e.value.code == -6  # no grid yet
        est.load_grid(real.gv, real.counts, real.du, real.flag_key)
        with pytest.raises(AmberError) as e:
            est.set_channels(3, [0, 1, 99])
        assert e.value.code == -1
        with pytest.raises(AmberError):
            est.set_channels(8)  # nc10 must be < nc
        est.set_rings([2.0, 5.0], [5.0, 20.0])  # 20 > N1/2 = 16
        with pytest.raises(AmberError) as e:
            est.calcr()
        assert e.value.code == -1
        with pytest.raises(AmberError):
            est.set_rings([5.0], [4.0])
        est.set_rings(real.ulow, real.uhigh)
        est.set_channels(3)
        with pytest.raises(AmberError):
            est.triangles(np.array([[0, 0, 9]], dtype=np.int32))
        # still usable after errors
        rd = est.calcr()
        assert len(rd) > 0


C2_FIXTURE = os.path.join(GOLDEN, "c2_rp217_ref64.npz")


@pytest.mark.skipif(not os.path.exists(C2_FIXTURE), reason="full-size fixture not generated")
def test_config2_full_size_triangle_vs_reference_build(lib_built):
    """One Ng1 = 740 triangle (rp = 217) of the single-realisation workload at full size — 256² grid,
    128 channels with the block-edge flags, nc10 = 63, 810152 channel triplets × 547600 pixels —
    against the reference's own FP64 build (tests/golden/c2_rp217_ref64.npz, v1 and v2 files).
    FP64 path within 1e-10 and the mixed path within 1e-6 of Σ|products| per lag cell (the FP64
    path on |maps| gives that scale); counts and the file scalars exact."""
    import hashlib
    import amber_b200
    z = np.load(C2_FIXTURE)
    real = synth.config2(seed=1)
    h = hashlib.sha256(np.ascontiguousarray(real.gv).tobytes() + np.ascontiguousarray(real.counts).tobytes())
    assert h.hexdigest() == str(z["inputs_sha256"]), "the seeded generator no longer makes the fixture's inputs"
    rp = int(z["rp"])
    out = {}
    for prec in ("fp64", "mixed", "fp64_abs"):
        with amber_b200.Estimator(precision=prec) as est:
            est.load_grid(real.gv, real.counts, real.du, real.flag_key)
            est.set_rings(real.ulow, real.uhigh)
            est.set_channels(real.nc10, real.uf_chans)
            rd = est.calcr()
            tri = rd[[rp], :3].astype(np.int32)
            assert np.array_equal(tri[0], z["tri"])
            bl, nd, nt = est.triangles(tri, want_v2=True)
            out[prec] = (bl[0].reshape(real.nclen, real.nclen), nd[0].reshape(real.nclen, real.nclen),
                         nt[0].reshape(real.nclen, real.nclen))
            if prec == "fp64":
                r1, r2, r3 = (int(v) for v in z["tri"])
                ntri, num, _, n1 = est.triangle_v1(r1, r2, r3, float(rd[rp, 3]))
                assert np.array_equal(n1, z["numdnu"])
                np.testing.assert_allclose([ntri, num], [float(z["ntri"]), float(z["num"])], rtol=1e-12)
    ab_bl, _, ab_nt = out["fp64_abs"]
    for prec, tol in (("fp64", 1e-10), ("mixed", 1e-6)):
        bl, nd, nt = out[prec]
        np.testing.assert_array_equal(nd, z["numdnu"])
        for ours, ref, scale in ((bl, z["bldnu64"], ab_bl), (bl, z["bldnu_v2"], ab_bl), (nt, z["numtri_v2"], ab_nt)):
            e = np.abs(ours - ref) / (scale + 1e-300)
            assert e.max() <= tol, (prec, e.max())


def _first_with_ng(real, ng_min):
    tri = oracle.triangles(real.ulow, real.uhigh)
    for i, t in enumerate(tri):
        if oracle.ng1(real.uhigh[int(t[0])], real.du) >= ng_min:
            return i
    return len(tri) - 1


@pytest.mark.parametrize("side", [96, 128, 192, 256, 320])
def test_ensemble_realisation_at_real_size_vs_oracle(side, lib_built):
    """The first realisation of each grid side in the 64-realisation ensemble, at its real size
    (its grid, channel count, flags and 12 rings), through the request engine; two of its triangles
    (the smallest map and the first with Ng1 ≥ 70) against the FP64 oracle.  Side 128 has
    nclen = 131, so its lag window spans 2 × 2 tiles."""
    import amber_b200
    specs = synth.config3_specs()
    spec = next(s for s in specs if s["nn"] == side)
    real = synth.from_spec(spec)
    pick = [0, _first_with_ng(real, 70)]
    with amber_b200.Estimator(precision="mixed") as est:
        eng = amber_b200.Engine(est)
        t = eng.enqueue(real, want_v2=True)
        rd, bl, nd, nt, _ = eng.result(t, real, want_v2=True)
    ordata, ores = oracle.estimate(real, version=2, tri_subset=pick, with_absscale=True)
    np.testing.assert_array_equal(rd[:, :3], ordata[:, :3])
    n = real.nclen
    for o in ores:
        i = o["rp"]
        np.testing.assert_array_equal(nd[i].reshape(n, n), o["numdnu"])
        e = np.abs(bl[i].reshape(n, n) - o["bldnu"]) / (o["absscale"] + 1e-300)
        assert e.max() <= 1e-6, (side, i, e.max())
        ei = np.abs(nt[i].reshape(n, n) - o["numtri"]) / (o["absscale_i"] + 1e-300)
        assert ei.max() <= 1e-6, (side, i, ei.max())
