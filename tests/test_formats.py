"""File formats: our writers against the layouts the reference's readers parse."""
import importlib
import os
import sys
import types

import numpy as np
import pytest

from amber_b200 import formats, synth
from oracle import REFERENCE_SOURCES as REF


def test_gv_roundtrip(tmp_path):
    real = synth.tiny(16, 3, seed=1, nbins=2, hi=7.0, nc10=1)
    p = tmp_path / "GV_data_1"
    formats.write_gv(p, real.gv, real.du, 1)
    assert os.path.getsize(p) == 28 + 16 * 9 * 3 * 16  # 28-byte header, no padding
    gv, du, fk = formats.read_gv(p)
    assert np.array_equal(gv, real.gv) and du == real.du and fk == 1


def test_bsout_layouts(tmp_path):
    n = 7
    bl = np.arange(n * n, dtype=np.float32).reshape(n, n)
    nd = (np.arange(n * n, dtype=np.int32) * 3).reshape(n, n)
    p1 = tmp_path / formats.bsout_name(1, 3, 2, 1, 5)
    formats.write_bsout_v1(p1, 0.25, 1234.5, bl, nd)
    assert os.path.getsize(p1) == 16 + n * n * 8
    t, num, b2, n2 = formats.read_bsout_v1(p1, n)
    assert t == 0.25 and num == 1234.5 and np.array_equal(b2, bl) and np.array_equal(n2, nd)
    p2 = tmp_path / formats.bsout_name(2, 3, 2, 1, 5)
    formats.write_bsout_v2(p2, 1.0 / 38 ** 2, bl, nd.astype(np.float32))
    assert os.path.getsize(p2) == 8 + n * n * 8
    assert p1.name == "bsout_final_ra3_rb2_rc1_R5" and p2.name == "bsout_final2_ra3_rb2_rc1_R5"


@pytest.mark.skipif(not os.path.exists(os.path.join(REF, "mabs_funcs.py")), reason="reference sources not present")
def test_reference_python_readers_read_our_files(tmp_path, monkeypatch):
    """mabs_funcs.read_bsout_float / read_bsout_float_v2 (mabs_funcs.py:172-205)
    parse our files unchanged; matplotlib is absent, so a stub module stands in."""
    monkeypatch.setitem(sys.modules, "matplotlib", types.ModuleType("matplotlib"))
    plt = types.ModuleType("matplotlib.pyplot")
    monkeypatch.setitem(sys.modules, "matplotlib.pyplot", plt)
    monkeypatch.syspath_prepend(REF)
    mf = importlib.import_module("mabs_funcs")
    nc10 = 5
    n = 2 * nc10 + 1
    monkeypatch.setattr(mf, "nc10", nc10)
    monkeypatch.setattr(mf, "nclen", n)
    monkeypatch.setattr(mf, "ncsize", n * n)
    rng = np.random.default_rng(0)
    bl = rng.standard_normal((n, n)).astype(np.float32)
    nd = rng.integers(0, 100, (n, n)).astype(np.int32)
    p1 = tmp_path / "v1"
    formats.write_bsout_v1(p1, 0.5, 4.0, bl, nd)
    ntri, bln, ndr = mf.read_bsout_float(str(p1))
    assert ntri == 0.5 and np.allclose(bln, bl / 4.0) and np.array_equal(ndr, nd)
    p2 = tmp_path / "v2"
    formats.write_bsout_v2(p2, 0.125, bl, nd.astype(np.float32))
    _, b2, n2 = mf.read_bsout_float_v2(str(p2))
    assert np.array_equal(b2, bl) and np.array_equal(n2, nd.astype(np.float32))


def test_gv_truncated_file_is_an_error(tmp_path):
    real = synth.tiny(16, 3, seed=1, nbins=2, hi=7.0, nc10=1)
    p = tmp_path / "GV_data_1"
    formats.write_gv(p, real.gv, real.du, 0)
    with open(p, "r+b") as f:
        f.truncate(os.path.getsize(p) - 16)  # one cell-channel short
    with pytest.raises(ValueError, match="truncated grid"):
        formats.read_gv(p)


def test_sampling_roundtrip_and_truncation(tmp_path):
    real = synth.tiny(16, 3, seed=2, nbins=2, hi=7.0, nc10=1)
    p = tmp_path / "sampling"
    formats.write_sampling(p, real.counts)
    assert os.path.getsize(p) == 16 * 9 * 3 * 8  # f64 per cell and channel, no header
    assert np.array_equal(formats.read_sampling(p, 16, 3), real.counts)
    with pytest.raises(ValueError, match="truncated"):
        formats.read_sampling(p, 16, 4)


def test_uf_chans_reads_exactly_the_requested_count(tmp_path):
    """get_uf_chans (4_fbe/amber_funcs.c:2485-2508) reads uf_nc integers: extra values are left
    unread and a short file fails."""
    p = tmp_path / "uf_chans.txt"
    formats.write_uf_chans(p, [0, 3, 3, 7, 11])
    assert formats.read_uf_chans(p, 4).tolist() == [0, 3, 3, 7]
    assert formats.read_uf_chans(p, 5).dtype == np.int32
    with pytest.raises(ValueError, match="expected 6"):
        formats.read_uf_chans(p, 6)


def test_input_params_and_rings_files_roundtrip_exactly(tmp_path):
    p = tmp_path / "input_params_ess"
    formats.write_input_params_ess(p, 154.255, 0.04, 0.1 + 0.2, "data/run1")
    assert formats.read_input_params_ess(p) == (154.255, 0.04, 0.1 + 0.2, "data/run1")
    lo, hi = synth.log_edges(2.0, 120.0, 16)
    r = tmp_path / "rings.txt"
    formats.write_rings_file(r, lo, hi)
    lines = open(r).read().split("\n")
    assert int(lines[0]) == 16
    back = np.array([[float(t) for t in ln.split()] for ln in lines[1:17]])
    assert np.array_equal(back[:, 0], lo) and np.array_equal(back[:, 1], hi)  # 17 digits: bit for bit


def test_closed_rings_roundtrip(tmp_path):
    """closed_rings is rcount × {f64 r1, r2, r3, Num} and rcount an ASCII integer (calCR,
    4_fbe/amber_funcs.c:406-483)."""
    rdata = np.array([[2, 1, 1, 12.5], [3, 3, 2, 7.25e9], [5, 4, 1, 0.0]])
    formats.write_closed_rings(tmp_path / "res", rdata)
    assert os.path.getsize(tmp_path / "res" / "closed_rings") == 3 * 4 * 8
    assert open(tmp_path / "res" / "rcount").read().strip() == "3"
    assert np.array_equal(formats.read_closed_rings(tmp_path / "res"), rdata)


def test_cldnu_file_roundtrip_at_printed_precision(tmp_path):
    """results/cldnu lines "i binu j cldnu numdnu num" with C's %e (4_fbe/maps.c:195-206): the
    reader returns the values to the printed six significant digits."""
    rng = np.random.default_rng(4)
    cl = rng.standard_normal((3, 5)) * 1e3
    nd = rng.integers(1, 1000, 5).astype(float)
    bu = np.array([1.5, 4.25, 11.0])
    nm = np.array([10, 0, 7])
    p = tmp_path / "cldnu"
    formats.write_cldnu(p, cl, nd, bu, nm)
    first = open(p).readline().rstrip("\n").split("\t")
    assert first[0] == "0" and first[2] == "0" and first[1] == f"{bu[0]:e}" and "e" in first[3]
    cl2, nd2, bu2, nm2 = formats.read_cldnu(p)
    assert np.allclose(cl2, cl, rtol=5e-6, atol=0) and np.array_equal(nd2, nd)
    assert np.array_equal(bu2, bu) and np.array_equal(nm2, nm)
