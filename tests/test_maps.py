"""MAPS two-point function C_ℓ(Δν) (4_fbe/maps.c:179-210 over cl_dnu, amber_funcs.c:1418-1488).

* The oracle's restatement (orc_cl_dnu) is pinned bit for bit to the reference's own cl_dnu,
  run by oracle/_ref/ref_maps: committed golden outputs and, where the build is present, a fresh
  run.
* The device path (amber_cuda_cl_dnu) keeps the reference's summation order and roundings, so it
  is compared bit for bit too.
"""
import os

import numpy as np
import pytest

import oracle
from amber_b200 import synth

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
KEYS = ("cldnu", "numdnu", "binu", "num")


def _golden():
    z = np.load(os.path.join(GOLDEN, "maps_flagged40.npz"))
    real = synth.Realisation(nn=z["gv"].shape[0], nc=z["gv"].shape[2], du=float(z["du"]), flag_key=0, gv=z["gv"],
                             counts=z["counts"], uf_chans=np.arange(z["gv"].shape[2]), ulow=np.array([2.0]),
                             uhigh=np.array([4.0]), nc10=1, seed=0)
    return z, real


def _same(got, z, tag):
    for k in KEYS:
        np.testing.assert_array_equal(got[k], z[f"{tag}_{k}"], err_msg=k)


@pytest.mark.parametrize("tag", ["maps", "fine"])
def test_oracle_matches_reference_golden(tag):
    z, real = _golden()
    nb, umin, umax = z[f"{tag}_bins"]
    _same(oracle.cl_dnu(real, int(nb), umin, umax), z, tag)
    assert (z[f"{tag}_num"] > 0).sum() >= 6


@pytest.mark.skipif(not oracle.ref_available(), reason="reference build (oracle/_ref) not present")
def test_oracle_matches_fresh_reference_run():
    real = synth.tiny(32, 7, seed=52, nbins=3, hi=14.0)
    r, txt = oracle.run_ref_maps(real, oracle.tmpdir(), 10, 0.8, 20.0)
    o = oracle.cl_dnu(real, 10, 0.8, 20.0)
    for k in KEYS:
        np.testing.assert_array_equal(o[k], r[k], err_msg=k)
    lines = open(txt).read().splitlines()
    assert len(lines) == 10 * 7 and lines[0].split("\t")[0] == "0"


@pytest.mark.skipif(not oracle.ref_available(), reason="reference build (oracle/_ref) not present")
def test_oracle_matches_fresh_reference_run_with_the_last_channel_flagged():
    """Flagged channels, the last among them: the reference prints the last pair's bin means, so
    binu and num come out zero, and every value still equals the reference's bit for bit."""
    real = synth.tiny(32, 7, seed=57, nbins=3, hi=14.0, flagged=[2, 6])
    r, _ = oracle.run_ref_maps(real, oracle.tmpdir(), 10, 0.8, 20.0)
    o = oracle.cl_dnu(real, 10, 0.8, 20.0)
    for k in KEYS:
        np.testing.assert_array_equal(o[k], r[k], err_msg=k)
    assert not np.any(r["binu"]) and not np.any(r["num"]) and np.any(r["cldnu"])


def _device(real, nb, umin, umax):
    import amber_b200
    with amber_b200.Estimator(precision="fp64") as est:
        est.load_grid(real.gv, real.counts, real.du, real.flag_key)
        return est.cl_dnu(nb, umin, umax)


@pytest.mark.gpu
@pytest.mark.parametrize("tag", ["maps", "fine"])
def test_device_matches_reference_golden(tag):
    z, real = _golden()
    nb, umin, umax = z[f"{tag}_bins"]
    _same(_device(real, int(nb), umin, umax), z, tag)


@pytest.mark.gpu
@pytest.mark.parametrize("nn,nc,flagged,bins", [
    (96, 37, [0, 5, 36], (15, 1.0, 500.0)),   # nc not a multiple of the 32-channel tile
    (128, 70, None, (20, 0.6, 40.0)),         # three tiles, many cells per bin
])
def test_device_matches_oracle(nn, nc, flagged, bins):
    real = synth.tiny(nn, nc, seed=53, nbins=5, hi=0.4 * nn, flagged=flagged)
    got = _device(real, *bins)
    want = oracle.cl_dnu(real, *bins)
    for k in KEYS:
        np.testing.assert_array_equal(got[k], want[k], err_msg=k)
    assert np.abs(want["cldnu"]).max() > 0


@pytest.mark.gpu
def test_device_argument_errors():
    import amber_b200
    real = synth.tiny(32, 8, seed=54, nbins=3, hi=14.0)
    with amber_b200.Estimator(precision="fp64") as est:
        with pytest.raises(amber_b200.AmberError):
            est.cl_dnu()  # no grid yet
        est.load_grid(real.gv, real.counts, real.du, real.flag_key)
        for bad in ((0, 1.0, 500.0), (15, 0.0, 500.0), (15, 5.0, 5.0)):
            with pytest.raises(amber_b200.AmberError):
                est.cl_dnu(*bad)


@pytest.mark.gpu
def test_maps_driver_writes_the_reference_file(tmp_path):
    """maps_gpu (the MAPS executable): maps.c's arguments and input_params in, results/cldnu out,
    the same text the reference's cl_dnu loop writes (and the oracle's values formatted alike)."""
    import subprocess
    from amber_b200 import build
    build.build()
    real = synth.tiny(40, 10, seed=55, nbins=4, hi=18.0, flagged=[3])
    data = tmp_path / "data"
    real.write(str(data), 1)
    (tmp_path / "input_params").write_text(
        f"{real.gv.shape[0]}\t{real.du!r}\t154.255e6\t40.00e03\t1\t{real.gv.shape[2]}\t{data}\n")
    p = subprocess.run([build.MAPS_DRIVER, "1", "GV_data_1"], capture_output=True, text=True, cwd=tmp_path)
    assert p.returncode == 0, p.stderr
    got = (tmp_path / "results" / "cldnu").read_text()
    o = oracle.cl_dnu(real)
    nc = real.gv.shape[2]
    want = "".join(f"{i}\t{o['binu'][i]:e}\t{j}\t{o['cldnu'][i, j]:e}\t{o['numdnu'][j]:e}\t{o['num'][i]}\n"
                   for i in range(15) for j in range(nc))
    assert got == want
    if oracle.ref_available():
        _, txt = oracle.run_ref_maps(real, oracle.tmpdir())
        assert open(txt).read() == got


def test_cldnu_file_writer_matches_the_reference_text(tmp_path):
    """formats.write_cldnu writes the reference's results/cldnu text (same %e formatting) from the
    golden values; read_cldnu parses it back to the printed precision."""
    from amber_b200 import formats
    z, real = _golden()
    p = tmp_path / "cldnu"
    formats.write_cldnu(p, z["maps_cldnu"], z["maps_numdnu"], z["maps_binu"], z["maps_num"])
    cl, nd, bu, nm = formats.read_cldnu(p)
    np.testing.assert_allclose(cl, z["maps_cldnu"], rtol=1e-6, atol=1e-300)
    np.testing.assert_array_equal(nm, z["maps_num"])
    if oracle.ref_available():
        _, txt = oracle.run_ref_maps(real, oracle.tmpdir())
        assert open(txt).read() == p.read_text()


@pytest.mark.gpu
@pytest.mark.parametrize("bins", [(1, 1.0, 500.0), (6, 400.0, 500.0)])
def test_device_single_bin_and_empty_bins(bins):
    """One bin for every cell, and bins beyond the grid (no cell in any bin: all zeros)."""
    real = synth.tiny(40, 9, seed=56, nbins=4, hi=18.0)
    got = _device(real, *bins)
    want = oracle.cl_dnu(real, *bins)
    for k in KEYS:
        np.testing.assert_array_equal(got[k], want[k], err_msg=k)
