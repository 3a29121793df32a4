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
