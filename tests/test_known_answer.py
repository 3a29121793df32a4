"""Known-answer test independent of the reference: the triangle sum in pixel space equals the
closed-triangle sum of the ring coefficients in Fourier space.

Each ring map is the unnormalised inverse transform of the ring's cells,
D(x) = Σ_k F(k) e^{+2πi k·x/Ng1}, with F the Hermitian extension of the half-plane grid values.
The map side Ng1 exceeds three times the largest |k|, so products of three maps do not alias,
and Σ_x D1(x)·D2(x)·D3(x) = Ng1² · Σ_{k1+k2+k3=0} F1(k1)·F2(k2)·F3(k3) holds exactly (up to
rounding).  This pins the oracle's ring filter, transform and triple product together."""
import numpy as np
import pytest
from scipy.signal import convolve2d

import oracle
from amber_b200 import synth


def ring_coefficients(gvn, lo, hi, p, K):
    """Full-plane coefficients F[k0 + K, k1 + K] of ring [lo, hi) for channel p: the stored half
    plane (j >= 0) and its Hermitian mirror; the j = 0 column contributes half of each value at k
    and half of its conjugate at -k (the transform keeps the real part of that column)."""
    nn, h, _ = gvn.shape
    F = np.zeros((2 * K + 1, 2 * K + 1), dtype=np.complex128)
    for ia in range(-(nn // 2) + 1, nn // 2 + 1):
        for j in range(0, h):
            r = np.sqrt(float(ia * ia + j * j))
            if not (r > 0 and lo <= r < hi):
                continue
            g = gvn[ia % nn, j, p]
            if j == 0:
                F[ia + K, K] += g / 2
                F[-ia + K, K] += np.conj(g) / 2
            else:
                F[ia + K, j + K] += g
                F[-ia + K, -j + K] += np.conj(g)
    return F


@pytest.mark.parametrize("seed", [61, 62])
def test_pixel_sum_equals_fourier_closed_triangle_sum(seed):
    real = synth.tiny(40, 4, seed=seed, nbins=4, hi=14.0, nc10=1)
    gvn, _ = oracle.normalize(real.gv, real.counts)
    tri = oracle.triangles(real.ulow, real.uhigh)
    K = int(np.ceil(real.uhigh.max())) + 1
    checked = 0
    for r1, r2, r3 in tri[:: max(1, len(tri) // 6)]:
        ng = oracle.ng1(real.uhigh[r1], real.du)
        maps = [oracle.ring_maps(gvn, real.ulow[r], real.uhigh[r], ng) for r in (r1, r2, r3)]
        for p1, p2, p3 in [(0, 1, 2), (3, 3, 0)]:
            d = maps[0][p1] * maps[1][p2] * maps[2][p3]
            direct, scale = d.sum(), np.abs(d).sum()
            F1, F2, F3 = (ring_coefficients(gvn, real.ulow[r], real.uhigh[r], p, K)
                          for r, p in ((r1, p1), (r2, p2), (r3, p3)))
            C = convolve2d(F1, F2)  # (F1 * F2)[m] at m - 2K = k1 + k2
            S = sum(F3[a, b] * C[2 * K - (a - K), 2 * K - (b - K)]
                    for a in range(2 * K + 1) for b in range(2 * K + 1) if F3[a, b] != 0)
            fourier = ng * ng * S
            assert abs(fourier.imag) <= 1e-9 * scale
            assert abs(direct - fourier.real) <= 1e-10 * scale, (r1, r2, r3, p1, p2, p3, direct, fourier)
            checked += 1
    assert checked >= 4


def _hand_records(nu0, du):
    """Five records placed at cell centres (u, v in units of du), two RR channels each:
    (3, 2) twice (its sums add), (-4, -1) with v < 0 (stored at (4, 1) with Im negated),
    (0, 5) with channel 1 flagged, and one beyond Umax (dropped)."""
    cells = [(3, 2), (3, 2), (-4, -1), (0, 5), (30, 0)]
    randpar = np.zeros((len(cells), 3), dtype=np.float32)
    for g, (a, b) in enumerate(cells):
        randpar[g, 0] = np.float32(a * du / nu0)
        randpar[g, 1] = np.float32(b * du / nu0)
    data = np.zeros((len(cells), 2, 1, 3), dtype=np.float32)
    for g in range(len(cells)):
        for c in range(2):
            data[g, c, 0] = (1.0 + g + 10 * c, 0.5 * (g + 1) - c, 1.0)
    data[3, 1, 0, 2] = -1.0  # flagged
    return randpar, data


def test_gridding_known_answer():
    nu0 = np.float32(150e6)
    nn, du, umax = 32, 0.5, 6.0
    randpar, data = _hand_records(nu0, du)
    gv, nt = oracle.grid_vis(nn, 2, du, umax, nu0, 1, randpar, data)
    want = np.zeros_like(gv)
    cnt = np.zeros_like(nt)
    for g, (i, j, sign) in enumerate([(3, 2, 1), (3, 2, 1), (4 % nn, 1, -1), (0, 5, 1)]):
        for c in range(2):
            if data[g, c, 0, 2] <= 0:
                continue
            want[i, j, c] += data[g, c, 0, 0] + 1j * sign * data[g, c, 0, 1]
            cnt[i, j, c] += 1
    assert np.array_equal(nt, cnt) and np.array_equal(gv, want)
    assert nt.sum() == 7  # 4 records × 2 channels, one flagged; the fifth record is beyond Umax


@pytest.mark.gpu
def test_gridding_known_answer_on_the_device():
    import amber_b200
    from amber_b200 import build
    build.build()
    nu0 = np.float32(150e6)
    randpar, data = _hand_records(nu0, 0.5)
    with amber_b200.Estimator() as est:
        gv, nt = est.grid_vis(32, 2, 0.5, 6.0, nu0, 1, randpar, data)
    g_o, n_o = oracle.grid_vis(32, 2, 0.5, 6.0, nu0, 1, randpar, data)
    assert np.array_equal(gv, g_o) and np.array_equal(nt, n_o) and nt.sum() == 7


def test_oracle_lag_symmetries():
    """Properties of the lag arrays that follow from the estimator's definition: with r2 = r3,
    bldnu[Δ2, Δ3] = bldnu[Δ3, Δ2]; with r1 = r2, swapping the roles of p1 and p2 gives
    bldnu[Δ2, Δ3] = bldnu[−Δ2, Δ3 − Δ2] (flags included: the channel weights are symmetric)."""
    real = synth.tiny(40, 10, seed=71, nbins=4, hi=18.0, nc10=4, flagged=[2, 7])
    _, res = oracle.estimate(real, version=1, with_absscale=True)
    n10 = real.nc10
    seen = set()
    for r in res:
        B, A = r["bldnu"], r["absscale"] + 1e-300
        if r["r2"] == r["r3"]:
            assert (np.abs(B - B.T) <= 1e-12 * A).all()
            seen.add("23")
        if r["r1"] == r["r2"]:
            for d2 in range(-n10, n10 + 1):
                for d3 in range(max(-n10, d2 - n10), min(n10, d2 + n10) + 1):
                    a, b = B[d2 + n10, d3 + n10], B[-d2 + n10, d3 - d2 + n10]
                    assert abs(a - b) <= 1e-12 * A[d2 + n10, d3 + n10]
            seen.add("12")
        np.testing.assert_array_equal(r["numdnu"], r["numdnu"].T)
    assert seen == {"12", "23"}
