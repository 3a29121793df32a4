"""The analysis stage's lag→k step (cylindrical bispectrum): the oracle's numpy restatement
against the reference's own Python (mabs_funcs.get_cyl_BS for v1 files, mfunc_winds.cylbs_win
for v2 files), whose outputs on seeded lag arrays are committed in tests/golden/cylbs_ref.npz."""
import os

import numpy as np

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
