"""Pin the CPU oracle before trusting it (no GPU needed).

The reference ships no tests or golden vectors, so the oracle is pinned
against the reference's OWN code built here from its sources (oracle/_ref):
the fixtures in tests/golden were produced by those builds
(tests/golden/make_golden.py), and when the builds are present the oracle is
also compared against a fresh run on new inputs.
"""
import glob
import os

import numpy as np
import pytest

import oracle
from amber_b200 import formats, synth

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _real_from(z):
    return synth.Realisation(nn=z["gv"].shape[0], nc=z["gv"].shape[2], du=float(z["du"]), flag_key=int(z["flag_key"]),
                             gv=z["gv"], counts=z["counts"], uf_chans=z["uf_chans"], ulow=z["ulow"],
                             uhigh=z["uhigh"], nc10=int(z["nc10"]), seed=0)


@pytest.mark.parametrize("n0,n1", [(20, 18), (38, 38), (74, 74), (45, 30), (16, 17)])
def test_fft_c2r_matches_numpy_on_hermitian_input(n0, n1):
    """fft64_c2r_2d (unnormalised, e^{+i}) equals n0·n1·irfft2 when the input is Hermitian."""
    rng = np.random.default_rng(n0 * 100 + n1)
    full = rng.standard_normal((n0, n1))
    X = np.fft.rfft2(full)  # Hermitian half-plane of a real field
    import ctypes
    lib = oracle.lib()
    lib.fft64_c2r_2d.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                 ctypes.POINTER(ctypes.c_double), ctypes.c_long, ctypes.c_int]
    xin = np.ascontiguousarray(X.astype(np.complex128)).view(np.float64)
    out = np.zeros((n0, n1))
    lib.fft64_c2r_2d(n0, n1, xin.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                     out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), n1, 1)
    np.testing.assert_allclose(out, full * n0 * n1, rtol=0, atol=1e-9 * np.abs(full).max() * n0 * n1)


def test_fft_c2r_ignores_imag_of_dc_column_bin():
    """Documented convention for non-Hermitian input: axis-0 complex DFT, then a
    1D c2r that drops Im of bin 0 — equal to Re of the inverse of the input with
    the j=0 column symmetrised."""
    import ctypes
    n0, n1 = 12, 10
    rng = np.random.default_rng(7)
    X = rng.standard_normal((n0, n1 // 2 + 1)) + 1j * rng.standard_normal((n0, n1 // 2 + 1))
    X[:, n1 // 2] = 0
    lib = oracle.lib()
    lib.fft64_c2r_2d.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                 ctypes.POINTER(ctypes.c_double), ctypes.c_long, ctypes.c_int]
    xin = np.ascontiguousarray(X).view(np.float64)
    out = np.zeros((n0, n1))
    lib.fft64_c2r_2d(n0, n1, xin.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                     out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), n1, 1)
    Y = np.fft.ifft(X, axis=0) * n0
    ref = np.zeros((n0, n1))
    k = np.arange(n1)
    for j in range(n1 // 2 + 1):
        w = 1.0 if j == 0 else 2.0
        yj = Y[:, j].real if j == 0 else Y[:, j]
        ref += w * np.real(np.outer(yj, np.exp(2j * np.pi * j * k / n1)))
    np.testing.assert_allclose(out, ref, atol=1e-10)


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "est_*.npz"))))
def test_oracle_matches_reference_fp64_golden(path):
    z = np.load(path)
    real = _real_from(z)
    rdata, res = oracle.estimate(real, version=2, with_absscale=True)
    ref_rd = z["rdata"]
    assert rdata.shape == ref_rd.shape
    np.testing.assert_array_equal(rdata[:, :3], ref_rd[:, :3])
    np.testing.assert_allclose(rdata[:, 3], ref_rd[:, 3], rtol=1e-12, atol=1e-9 * np.abs(ref_rd[:, 3]).max())
    for i, r in enumerate(res):
        np.testing.assert_array_equal(r["numdnu"], z["numdnu"][i])
        scale = r["absscale"] + 1e-300
        err = np.abs(r["bldnu"] - z["bldnu64"][i]) / scale
        assert err.max() <= 1e-10, (i, err.max())
        erri = np.abs(r["numtri"] - z["numtri_v2"][i]) / (r["absscale_i"] + 1e-300)
        assert erri.max() <= 1e-10, (i, erri.max())
        assert r["total_vcp"] == int(z["total_vcp"])


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "est_*.npz"))))
def test_reference_float_build_within_its_own_rounding(path):
    """The as-shipped float build agrees with its FP64 build to float accuracy
    (a sanity check of the fixture pair, 1e-3 of Σ|products|)."""
    z = np.load(path)
    real = _real_from(z)
    _, res = oracle.estimate(real, version=1, with_absscale=True)
    for i, r in enumerate(res):
        err = np.abs(z["bldnu32"][i].astype(np.float64) - z["bldnu64"][i]) / (r["absscale"] + 1e-300)
        assert err.max() < 1e-3


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "grid_*.npz"))))
def test_oracle_gridding_bit_exact_vs_reference_golden(path):
    """The gridding restatement (and, for the coll_* cases, collapse_channels after it) against the
    reference's gridding stage run on the same records."""
    z = np.load(path)
    n_coll = int(z["n_collapse"]) if "n_collapse" in z.files else 1
    gv, nt = oracle.grid_vis(int(z["nn"]), z["data"].shape[1], float(z["du"]), float(z["umax"]), z["nu0"],
                             int(z["flag_key"]), z["randpar"], z["data"])
    if n_coll > 1:
        gv, nt = oracle.collapse_channels(gv, nt, n_coll)
        assert gv.shape[2] == z["data"].shape[1] // n_coll
    assert np.array_equal(gv.real, z["gv"].real) and np.array_equal(gv.imag, z["gv"].imag)
    assert np.array_equal(nt, z["ntig"])
    assert nt.max() >= 2  # several records share cells: the ordered sum is exercised


def test_triangle_rule_and_ng1():
    lo, hi = synth.log_edges(2.0, 120.0, 16)
    tri = oracle.triangles(lo, hi)
    assert len(tri) == 218
    assert oracle.ng1(120.0, 0.5) == 740 and oracle.ng1(60.0, 0.5) == 380 and oracle.ng1(240.0, 0.5) == 1460
    assert oracle.ng1(270.0, 1.0254384902642049) == 800  # archived run, amber.c:99-103


@pytest.mark.skipif(not oracle.ref_available(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("seed,flagged", [(21, None), (22, [1, 2, 9])])
def test_oracle_matches_fresh_reference_run(seed, flagged):
    real = synth.tiny(36, 10, seed=seed, nbins=4, hi=16.0, nc10=4, flagged=flagged)
    st, rp = oracle.run_ref_amber(real, oracle.tmpdir(), version=2, fp64=True)
    rdata, res = oracle.estimate(real, version=2, with_absscale=True)
    np.testing.assert_array_equal(formats.read_closed_rings(rp)[:, :3], rdata[:, :3])
    for r in res:
        inv, bl, nd = formats.read_bsout_v2(os.path.join(rp, formats.bsout_name(2, r["r1"], r["r2"], r["r3"], 1)),
                                            real.nclen, np.float64)
        # per lag cell, against Σ|products| of that cell; the v2 file's second array is the mask sums
        assert (np.abs(bl - r["bldnu"]) <= 1e-10 * r["absscale"] + 1e-300).all()
        assert (np.abs(nd - r["numtri"]) <= 1e-10 * r["absscale_i"] + 1e-300).all()
        assert inv == 1.0 / (r["ng1"] ** 2)


@pytest.mark.skipif(not oracle.ref_available(), reason="reference build (oracle/_ref) not present")
def test_oracle_gridding_matches_fresh_reference_vcg():
    import math
    fwhm, umax, nc = 1480.73, 20.0, 3
    theta0 = 0.6 * fwhm * math.pi / (180. * 60.)
    du = math.sqrt(math.log(2)) / (math.pi * theta0)
    nn = 2 * int(math.ceil(umax / du))
    randpar, data = synth.make_visibilities(nn, du, nc, 500, 99, umax=umax * 1.05)
    gv, nt, du_ref, nn_ref = oracle.run_ref_vcg(randpar, data, np.float32(synth.NU0), nc, umax, fwhm, 1,
                                                oracle.tmpdir())
    g2, n2 = oracle.grid_vis(nn_ref, nc, du_ref, umax, np.float32(synth.NU0), 1, randpar, data)
    assert np.array_equal(g2, gv) and np.array_equal(n2, nt)


@pytest.mark.skipif(not oracle.ref_available(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("nc,flag_key", [(8, 0), (11, 1)])
def test_oracle_collapse_matches_fresh_reference_vcg(nc, flag_key):
    """The reference's gridding stage run with the collapse key: 4 channels per output channel,
    trailing channels dropped (11 → 2)."""
    import math
    fwhm, umax = 1480.73, 18.0
    theta0 = 0.6 * fwhm * math.pi / (180. * 60.)
    du = math.sqrt(math.log(2)) / (math.pi * theta0)
    nn = 2 * int(math.ceil(umax / du))
    randpar, data = synth.make_visibilities(nn, du, nc, 400, 70 + nc, umax=umax * 1.05)
    gv, nt, du_ref, nn_ref = oracle.run_ref_vcg(randpar, data, np.float32(synth.NU0), nc, umax, fwhm, flag_key,
                                                oracle.tmpdir(), collapse=True)
    g, n = oracle.grid_vis(nn_ref, nc, du_ref, umax, np.float32(synth.NU0), flag_key, randpar, data)
    g2, n2 = oracle.collapse_channels(g, n, 4)
    assert gv.shape[2] == nc // 4
    assert np.array_equal(g2, gv) and np.array_equal(n2, nt)


@pytest.mark.skipif(not oracle.ref_available(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("nn,nc,seed,nc10,flagged", [
    (32, 6, 23, 0, None),                        # only the zero lag
    (32, 7, 24, 6, None),                        # nc10 = nc - 1: the widest window
    (36, 12, 25, 5, [0, 1, 2, 4, 6, 7, 9, 11]),  # most channels flagged
])
def test_oracle_matches_reference_at_edges(nn, nc, seed, nc10, flagged):
    """The FP64 reference build (v1 files) against the oracle per lag cell at the edges of the
    lag window and of the flag set: triangle list, counts exact, lag sums within 1e-10 of
    Σ|products| of the same cell, the file scalars Num and Ntri."""
    real = synth.tiny(nn, nc, seed=seed, nbins=3, hi=0.44 * nn, nc10=nc10, flagged=flagged)
    st, rp = oracle.run_ref_amber(real, oracle.tmpdir(), version=1, fp64=True)
    rdata, res = oracle.estimate(real, version=1, with_absscale=True)
    np.testing.assert_array_equal(formats.read_closed_rings(rp)[:, :3], rdata[:, :3])
    assert len(res) > 0
    for r in res:
        ntri, num, bl, nd = formats.read_bsout_v1(
            os.path.join(rp, formats.bsout_name(1, r["r1"], r["r2"], r["r3"], 1)), real.nclen, bl_dtype=np.float64)
        np.testing.assert_array_equal(nd, r["numdnu"])
        assert (np.abs(bl - r["bldnu"]) <= 1e-10 * r["absscale"] + 1e-300).all()
        np.testing.assert_allclose(num, (r["ng1"] / real.nn) ** 2 * r["rdata_num"], rtol=1e-12)
        np.testing.assert_allclose(ntri, num / r["ng1"] ** 2, rtol=1e-12)


@pytest.mark.skipif(not oracle.ref_available(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("nn,nc,seed,nc10,flagged", [
    (32, 6, 26, 0, None),                        # only the zero lag
    (32, 7, 27, 6, None),                        # nc10 = nc - 1: the widest window
    (36, 12, 28, 5, [0, 1, 2, 4, 6, 7, 9, 11]),  # most channels flagged
])
def test_oracle_v2_matches_reference_at_edges(nn, nc, seed, nc10, flagged):
    """The same edges for the v2 files (4_fbe/amber_v2.c:295-309): lag sums and sampling-mask sums
    per lag cell within 1e-10 of their own Σ|products|, and the 1/Ng1² scalar."""
    real = synth.tiny(nn, nc, seed=seed, nbins=3, hi=0.44 * nn, nc10=nc10, flagged=flagged)
    st, rp = oracle.run_ref_amber(real, oracle.tmpdir(), version=2, fp64=True)
    rdata, res = oracle.estimate(real, version=2, with_absscale=True)
    np.testing.assert_array_equal(formats.read_closed_rings(rp)[:, :3], rdata[:, :3])
    assert len(res) > 0
    for r in res:
        inv, bl, nd = formats.read_bsout_v2(os.path.join(rp, formats.bsout_name(2, r["r1"], r["r2"], r["r3"], 1)),
                                            real.nclen, np.float64)
        assert (np.abs(bl - r["bldnu"]) <= 1e-10 * r["absscale"] + 1e-300).all()
        assert (np.abs(nd - r["numtri"]) <= 1e-10 * r["absscale_i"] + 1e-300).all()
        assert inv == 1.0 / (r["ng1"] ** 2)


@pytest.mark.skipif(not oracle.ref_available(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("version", [1, 2])
def test_oracle_matches_reference_on_an_empty_realisation(version):
    """No sampled cell at all (every count and every visibility zero): the reference still lists
    the geometrically closed triangles, with Num = 0, zero lag and mask sums and the full triplet
    counts; the oracle gives the same files' contents."""
    real = synth.tiny(32, 6, seed=29, nbins=3, hi=14.0, nc10=2)
    real.counts[:] = 0.0
    real.gv[:] = 0.0
    st, rp = oracle.run_ref_amber(real, oracle.tmpdir(), version=version, fp64=True)
    rdata, res = oracle.estimate(real, version=version)
    ref_rings = formats.read_closed_rings(rp)
    np.testing.assert_array_equal(ref_rings, rdata)
    assert len(res) == len(ref_rings) > 0 and (ref_rings[:, 3] == 0).all()
    for r in res:
        name = os.path.join(rp, formats.bsout_name(version, r["r1"], r["r2"], r["r3"], 1))
        if version == 1:
            ntri, num, bl, nd = formats.read_bsout_v1(name, real.nclen, bl_dtype=np.float64)
            assert ntri == 0.0 and num == 0.0
            np.testing.assert_array_equal(nd, r["numdnu"])
            assert nd.max() > 0
        else:
            inv, bl, nd = formats.read_bsout_v2(name, real.nclen, np.float64)
            assert inv == 1.0 / (r["ng1"] ** 2)
            assert not nd.any() and not r["numtri"].any()
        assert not bl.any() and not r["bldnu"].any()


@pytest.mark.skipif(not oracle.ref_available(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("version", [1, 2])
def test_oracle_matches_reference_with_whole_cell_ring_edges(version):
    """Ring edges at whole cells, as the reference's own annular_rings ladder has them
    (4_fbe/amber_funcs.c:2022-2062): cells whose radius falls exactly on an edge belong to the outer
    ring (lo ≤ √(ia²+j²) < hi).  Triangle list, Num and counts exact, sums within 1e-10."""
    import dataclasses
    real = synth.tiny(40, 8, seed=31, nbins=4, hi=17.0, nc10=3, flagged=[2])
    real = dataclasses.replace(real, ulow=np.array([1.0, 5.0, 10.0, 15.0]), uhigh=np.array([5.0, 10.0, 15.0, 17.0]))
    st, rp = oracle.run_ref_amber(real, oracle.tmpdir(), version=version, fp64=True)
    rdata, res = oracle.estimate(real, version=version, with_absscale=True)
    np.testing.assert_array_equal(formats.read_closed_rings(rp), rdata)
    for r in res:
        name = os.path.join(rp, formats.bsout_name(version, r["r1"], r["r2"], r["r3"], 1))
        if version == 1:
            ntri, num, bl, nd = formats.read_bsout_v1(name, real.nclen, bl_dtype=np.float64)
            np.testing.assert_array_equal(nd, r["numdnu"])
        else:
            inv, bl, nd = formats.read_bsout_v2(name, real.nclen, np.float64)
            assert (np.abs(nd - r["numtri"]) <= 1e-10 * r["absscale_i"] + 1e-300).all()
        assert (np.abs(bl - r["bldnu"]) <= 1e-10 * r["absscale"] + 1e-300).all()


@pytest.mark.skipif(not oracle.ref_available(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("version", [1, 2])
def test_oracle_matches_reference_at_the_archived_cell_size(version):
    """Du = 1.0254384902642049, the cell size of the reference's archived run (input_params_ess:7):
    map sides from the Ng1 formula at a non-dyadic Du (amber.c:193-197), the v1 Num scaling and the
    v2 1/Ng1² scalar, counts exact and sums within 1e-10 of Σ|products|."""
    real = synth.make_realisation(36, 8, 33, 4, 2.0, 15.0, 3, flagged=[1, 6], du=1.0254384902642049)
    st, rp = oracle.run_ref_amber(real, oracle.tmpdir(), version=version, fp64=True)
    rdata, res = oracle.estimate(real, version=version, with_absscale=True)
    np.testing.assert_array_equal(formats.read_closed_rings(rp), rdata)
    assert len({r["ng1"] for r in res}) > 1
    for r in res:
        name = os.path.join(rp, formats.bsout_name(version, r["r1"], r["r2"], r["r3"], 1))
        if version == 1:
            ntri, num, bl, nd = formats.read_bsout_v1(name, real.nclen, bl_dtype=np.float64)
            np.testing.assert_array_equal(nd, r["numdnu"])
            np.testing.assert_allclose(num, (r["ng1"] / real.nn) ** 2 * r["rdata_num"], rtol=1e-12)
        else:
            inv, bl, nd = formats.read_bsout_v2(name, real.nclen, np.float64)
            assert inv == 1.0 / (r["ng1"] ** 2)
            assert (np.abs(nd - r["numtri"]) <= 1e-10 * r["absscale_i"] + 1e-300).all()
        assert (np.abs(bl - r["bldnu"]) <= 1e-10 * r["absscale"] + 1e-300).all()
