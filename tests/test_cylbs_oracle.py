"""The analysis stage's lag→k step (cylindrical bispectrum): the oracle's numpy restatement
against the reference's own Python (mabs_funcs.get_cyl_BS for v1 files, mfunc_winds.cylbs_win
for v2 files), whose outputs on seeded lag arrays are committed in tests/golden/cylbs_ref.npz."""
import os

import numpy as np
import pytest

import oracle

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "cylbs_ref.npz")


def _g():
    g = np.load(GOLD)
    return {k: g[k] for k in g.files}


def _const(g):
    return dict(nc10=int(g["nc10"]), n_cut=int(g["n_cut"]), mabs_norm=float(g["mabs_norm"]), rc=float(g["rc"]),
                rc_prime=float(g["rc_prime"]), dnu=float(g["dnu"]))


def test_v1_counts_normalised_matches_reference():
    g = _g()
    out = oracle.cyl_bs(g["bl"], g["counts"], div=float(g["num"]), **_const(g))
    assert out.shape == g["v1"].shape == (45, 45)
    scale = np.abs(g["v1"]).max()
    assert np.abs(out - g["v1"]).max() <= 1e-13 * scale


def test_v2_windowed_matches_reference_float32_chain():
    g = _g()
    out = oracle.cyl_bs(g["bl"], g["mask"], window=True, float32=True, **_const(g))
    scale = np.abs(g["v2"]).max()
    assert np.abs(out - g["v2"]).max() <= 1e-13 * scale
    # the FP64 chain (what the device computes) differs only by the reference's float32 rounding
    out64 = oracle.cyl_bs(g["bl"], g["mask"], window=True, **_const(g))
    assert np.abs(out64 - g["v2"]).max() <= 1e-5 * scale


def test_reference_constants_match_library_defaults():
    import amber_b200
    g = _g()
    c = amber_b200.reference_cylbs_constants()
    assert c["n_cut"] == int(g["n_cut"])
    for k in ("mabs_norm", "rc", "rc_prime"):
        assert c[k] == float(g[k]), k
    assert c["dnu_mhz"] == float(g["dnu"])


from oracle import REFERENCE_SOURCES as REF  # noqa: E402


@pytest.mark.skipif(not os.path.exists(os.path.join(REF, "mabs_funcs.py")), reason="reference sources not present")
@pytest.mark.parametrize("nc10,seed", [(63, 12), (20, 13)])
def test_oracle_matches_reference_python_fresh(tmp_path, monkeypatch, nc10, seed):
    """The reference's analysis Python run here on fresh seeded files, at the single-realisation
    lag width (nc10 = 63) and a small one; matplotlib is absent, so a stub stands in."""
    import importlib
    import sys
    import types
    from amber_b200 import formats
    monkeypatch.setitem(sys.modules, "matplotlib", types.ModuleType("matplotlib"))
    monkeypatch.setitem(sys.modules, "matplotlib.pyplot", types.ModuleType("matplotlib.pyplot"))
    monkeypatch.syspath_prepend(REF)
    mf = importlib.import_module("mabs_funcs")
    nclen = 2 * nc10 + 1
    monkeypatch.setattr(mf, "nc10", nc10)
    monkeypatch.setattr(mf, "nclen", nclen)
    monkeypatch.setattr(mf, "ncsize", nclen * nclen)
    mw = importlib.import_module("mfunc_winds")
    rng = np.random.default_rng(seed)
    bl = rng.standard_normal((nclen, nclen)).astype(np.float32)
    counts = rng.integers(1, 500, (nclen, nclen)).astype(np.int32)
    mask = rng.uniform(0.1, 3.0, (nclen, nclen)).astype(np.float32)
    formats.write_bsout_v1(tmp_path / formats.bsout_name(1, 4, 3, 2, 1), 0.5, 2.25, bl, counts)
    formats.write_bsout_v2(tmp_path / formats.bsout_name(2, 4, 3, 2, 1), 1.0 / 64, bl, mask)
    v1, _ = mf.get_cyl_BS(4, 3, 2, str(tmp_path), 1)
    v2 = mw.cylbs_win(4, 3, 2, str(tmp_path))
    c = dict(nc10=nc10, n_cut=mf.n_nancut, mabs_norm=mf.mabs_norm, rc=mf.rc, rc_prime=mf.rc_prime, dnu=mf.dnu_mwa)
    o1 = oracle.cyl_bs(bl, counts, div=2.25, **c)
    o2 = oracle.cyl_bs(bl, mask, window=True, float32=True, **c)
    assert np.abs(o1 - v1).max() <= 1e-13 * np.abs(v1).max()
    assert np.abs(o2 - v2).max() <= 1e-13 * np.abs(v2).max()
