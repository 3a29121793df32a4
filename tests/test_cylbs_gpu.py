"""amber_cuda_cyl_bs (the lag→k step on the device) against the oracle's restatement of
mabs_funcs.get_cyl_BS / mfunc_winds.cylbs_win, applied to the same run's fetched lag arrays.
Both are FP64 from the lag arrays on; the device's direct transforms and numpy's FFT differ by
rounding only, so the bound is 1e-10 of the largest output of each triangle."""
import numpy as np
import pytest

import oracle
from amber_b200 import synth

pytestmark = pytest.mark.gpu

TOL = 1e-10


@pytest.fixture(scope="module")
def lib_built():
    from amber_b200 import build
    build.build()
    return True


def _check(got, want):
    assert got.shape == want.shape
    assert np.isfinite(want).all()
    scale = np.abs(want).max()
    err = np.abs(got - want).max() / scale
    assert err <= TOL, err


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("n_cut", [8, 3])
def test_cyl_bs_matches_oracle(precision, n_cut, lib_built):
    import amber_b200
    # the folded, cut lags span at most 2·(nc10 − n_cut) < nc channels, so no count is zero
    real = synth.tiny(64, 40, seed=21, nbins=5, hi=28.0, nc10=15)
    k = amber_b200.reference_cylbs_constants()
    k["n_cut"] = n_cut
    const = dict(nc10=15, n_cut=n_cut, mabs_norm=k["mabs_norm"], rc=k["rc"], rc_prime=k["rc_prime"],
                 dnu=k["dnu_mhz"])
    with amber_b200.Estimator(precision=precision) as est:
        rdata, res = amber_b200.estimate(real, version=2, est=est)
        num = rdata[:, 3]
        v1 = est.cyl_bs(tri_div=num, n_cut=n_cut)
        v2 = est.cyl_bs(window=True, denominator="mask", n_cut=n_cut)
        plain = est.cyl_bs(n_cut=n_cut)
    n = 2 * (15 + 1 - n_cut) - 1
    assert v1.shape == v2.shape == (len(res), n, n)
    for i, r in enumerate(res):
        _check(v1[i], oracle.cyl_bs(r["bldnu"], r["numdnu"], div=num[i], **const))
        _check(v2[i], oracle.cyl_bs(r["bldnu"], r["numtri"], window=True, **const))
        _check(plain[i], oracle.cyl_bs(r["bldnu"], r["numdnu"], **const))


def test_cyl_bs_state_and_argument_errors(lib_built):
    import amber_b200
    real = synth.tiny(48, 24, seed=22, nbins=4, hi=21.0, nc10=10)
    with amber_b200.Estimator(precision="mixed") as est:
        with pytest.raises(amber_b200.AmberError):
            est.cyl_bs()  # no run yet
        rdata, _ = amber_b200.estimate(real, version=1, est=est)
        with pytest.raises(amber_b200.AmberError):
            est.cyl_bs(denominator="mask")  # v1 run: no mask sums
        with pytest.raises(amber_b200.AmberError):
            est.cyl_bs(n_cut=10)  # nothing left after the cut
        with pytest.raises(amber_b200.AmberError):
            est.cyl_bs(tri_div=np.zeros(len(rdata)))
        assert est.cyl_bs().shape[0] == len(rdata)
        est.calcr()  # overwrites the results buffer: the last run is gone
        with pytest.raises(amber_b200.AmberError):
            est.cyl_bs()
