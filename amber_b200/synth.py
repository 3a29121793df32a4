"""Seeded synthetic inputs for the estimator path.

No public dataset is involved (the reference ships no UVFITS data): every
workload is generated here with ``numpy.random.default_rng(seed)``.

Field recipe, per uv cell of the half-plane grid ``NN × (NN/2+1)``:
* complex Gaussian amplitude with power ``P(|U|) ∝ |U|^-2.5`` (|U| in cells,
  DC zero), correlated across channels as an AR(1) with ``ρ = e^{-1/8}`` (an
  exponential kernel of 8-channel length);
* iid complex noise of 10 % of the field rms per record;
* sampling counts ``Poisson(λ0 · e^{-|U|/decay})`` per cell and channel,
  zero beyond the outermost ring edge and in flagged channels; ``λ0 = 4``,
  ``decay = 20 cells × NN/128``;
* the stored grid is the SUM over records (``count·field + √count·noise``),
  exactly what the gridding stage writes;
* the j = 0 column is Hermitian (cell −ia is the conjugate of cell ia, with
  the same count), so the c2r transform of a ring sees Hermitian input.

Ring edges are log-spaced with the end points stored exactly.
"""
from __future__ import annotations

import dataclasses
import math
import os

import numpy as np

from . import formats

NU0 = 154.255e6
DNU = 40.0e3


@dataclasses.dataclass
class Realisation:
    """One estimator input: the normalised-to-be grid plus its parameters."""

    nn: int
    nc: int
    du: float
    flag_key: int
    gv: np.ndarray  # complex128 [NN, NN/2+1, nc] — summed visibilities
    counts: np.ndarray  # float64 [NN, NN/2+1, nc]
    uf_chans: np.ndarray  # int32 unflagged channels (all channels when flag_key == 0)
    ulow: np.ndarray
    uhigh: np.ndarray
    nc10: int
    seed: int
    name: str = ""

    @property
    def nclen(self) -> int:
        return 2 * self.nc10 + 1

    def write(self, data_path: str, rlzn: int = 1) -> None:
        """Write the files amber reads: GV_data_<R>, sampling, uf_chans.txt."""
        os.makedirs(data_path, exist_ok=True)
        formats.write_gv(os.path.join(data_path, f"GV_data_{rlzn}"), self.gv, self.du, self.flag_key)
        formats.write_sampling(os.path.join(data_path, "sampling"), self.counts)
        formats.write_uf_chans(os.path.join(data_path, "uf_chans.txt"), self.uf_chans)


def log_edges(lo: float, hi: float, nbins: int):
    e = np.geomspace(lo, hi, nbins + 1)
    e[0] = lo
    e[-1] = hi
    return e[:-1].copy(), e[1:].copy()


def make_realisation(nn: int, nc: int, seed: int, nbins: int, ring_lo: float, ring_hi: float, nc10: int,
                     flagged=None, du: float = 0.5, lam0: float = 4.0, noise_frac: float = 0.1,
                     name: str = "") -> Realisation:
    """Generate one realisation (see module docstring for the recipe).

    ``flagged``: iterable of flagged channel indices (None → flag_key 0)."""
    rng = np.random.default_rng(seed)
    h = nn // 2 + 1
    ia = np.arange(nn)
    ia = np.where(ia > nn // 2, ia - nn, ia)
    jj = np.arange(h)
    u = np.sqrt(ia[:, None].astype(np.float64) ** 2 + jj[None, :].astype(np.float64) ** 2)
    amp = np.zeros_like(u)
    amp[u > 0] = u[u > 0] ** (-2.5 / 2)
    rho = math.exp(-1.0 / 8.0)
    s = math.sqrt(1.0 - rho * rho)
    field = np.empty((nn, h, nc), dtype=np.complex128)
    x = (rng.standard_normal((nn, h)) + 1j * rng.standard_normal((nn, h))) / math.sqrt(2)
    for c in range(nc):
        if c:
            w = (rng.standard_normal((nn, h)) + 1j * rng.standard_normal((nn, h))) / math.sqrt(2)
            x = rho * x + s * w
        field[:, :, c] = x * amp
    live = u > 0
    rms = math.sqrt(float(np.mean(np.abs(field[live]) ** 2)))
    decay = 20.0 * nn / 128.0
    lam = lam0 * np.exp(-u / decay)
    lam[u > ring_hi] = 0.0
    lam[u == 0] = 0.0
    counts = rng.poisson(np.broadcast_to(lam[:, :, None], (nn, h, nc))).astype(np.float64)
    noise = (rng.standard_normal((nn, h, nc)) + 1j * rng.standard_normal((nn, h, nc))) / math.sqrt(2)
    gv = counts * field + np.sqrt(counts) * noise_frac * rms * noise
    flag_key = 0
    uf = np.arange(nc, dtype=np.int32)
    if flagged is not None:
        flagged = np.asarray(sorted(set(int(f) for f in flagged)), dtype=np.int64)
        flag_key = 1
        if flagged.size:
            counts[:, :, flagged] = 0.0
            gv[:, :, flagged] = 0.0
        uf = np.setdiff1d(np.arange(nc), flagged).astype(np.int32)
    # Hermitian j = 0 column: cell (-ia, 0) mirrors (ia, 0).
    for i in range(1, nn // 2):
        gv[nn - i, 0, :] = np.conj(gv[i, 0, :])
        counts[nn - i, 0, :] = counts[i, 0, :]
    gv[0, 0, :] = 0.0
    counts[0, 0, :] = 0.0
    gv[nn // 2, 0, :] = gv[nn // 2, 0, :].real
    ulow, uhigh = log_edges(ring_lo, ring_hi, nbins)
    return Realisation(nn=nn, nc=nc, du=du, flag_key=flag_key, gv=gv, counts=counts, uf_chans=uf,
                       ulow=ulow, uhigh=uhigh, nc10=nc10, seed=seed, name=name)


def block_edge_flags(nc: int, block: int = 32, edge: int = 2):
    """Channels 0..edge-1 and block-edge..block-1 of every block (config 2)."""
    return [c for c in range(nc) if (c % block) < edge or (c % block) >= block - edge]


def random_flags(nc: int, frac: float, seed: int):
    rng = np.random.default_rng(seed + 7919)
    k = int(round(frac * nc))
    return sorted(rng.choice(nc, size=k, replace=False).tolist())


# ---- the workloads -----------------------------------------------------------

def config1(seed: int = 0) -> Realisation:
    """Plain method, CPU-runnable: 128², 32 channels, 8 bins 2→60, nc10 = 31, no flags."""
    return make_realisation(128, 32, seed, 8, 2.0, 60.0, 31, flagged=None, name="config1")


def config2(seed: int = 1) -> Realisation:
    """Single realisation: 256², 128 channels, 16 bins 2→120, nc10 = 63,
    channels 0-1 and 30-31 of every 32-channel block flagged."""
    return make_realisation(256, 128, seed, 16, 2.0, 120.0, 63, flagged=block_edge_flags(128), name="config2")


def config4(seed: int = 2) -> Realisation:
    """Large cube: 512², 384 channels, 24 bins 2→240, nc10 = 191, 15 % random flags."""
    return make_realisation(512, 384, seed, 24, 2.0, 240.0, 191, flagged=random_flags(384, 0.15, seed),
                            name="config4")


ENSEMBLE_SIDES = (96, 128, 192, 256, 320)


def config3_specs(n: int = 64, seed0: int = 100):
    """Shapes of the batched ensemble: side from {96,128,192,256,320}, 24–160
    channels, seeds 100–163, 10 % random flags, 12 bins 2→⌊0.47·side⌋,
    nc10 = nc/2 − 1."""
    rng = np.random.default_rng(12345)
    out = []
    for i in range(n):
        side = int(rng.choice(ENSEMBLE_SIDES))
        nc = int(rng.integers(24, 161))
        out.append(dict(nn=side, nc=nc, seed=seed0 + i, nbins=12, ring_lo=2.0,
                        ring_hi=float(math.floor(0.47 * side)), nc10=nc // 2 - 1, flag_frac=0.10))
    return out


def from_spec(spec) -> Realisation:
    flags = random_flags(spec["nc"], spec["flag_frac"], spec["seed"])
    return make_realisation(spec["nn"], spec["nc"], spec["seed"], spec["nbins"], spec["ring_lo"], spec["ring_hi"],
                            spec["nc10"], flagged=flags, name=f"s{spec['seed']}")


SERVE_SIDES = (64, 128, 256, 384)


def config5_requests(n: int = 2000, rate: float = 50.0, seed: int = 5):
    """Serving stream: Poisson arrivals at ``rate`` req/s; side from
    {64,128,256,384}, 16–256 channels, 6–20 bins, own seed and flag mask."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, size=n))
    reqs = []
    for i in range(n):
        side = int(rng.choice(SERVE_SIDES))
        nc = int(rng.integers(16, 257))
        reqs.append(dict(arrival=float(t[i]), nn=side, nc=nc, seed=10000 + i, nbins=int(rng.integers(6, 21)),
                         ring_lo=2.0, ring_hi=float(math.floor(0.47 * side)), nc10=nc // 2 - 1, flag_frac=0.10))
    return reqs


def tiny(nn: int = 32, nc: int = 8, seed: int = 3, nbins: int = 4, hi: float | None = None, nc10: int | None = None,
         flagged=None) -> Realisation:
    """Small case for parity tests (seconds on the CPU oracle)."""
    hi = float(hi if hi is not None else math.floor(0.45 * nn))
    return make_realisation(nn, nc, seed, nbins, 2.0, hi, nc10 if nc10 is not None else nc // 2 - 1,
                            flagged=flagged, name=f"tiny{nn}x{nc}")


def make_visibilities(nn: int, du: float, nc: int, ngroups: int, seed: int, nu0: float = NU0, nstokes: int = 2,
                      flag_frac: float = 0.1, umax: float | None = None, dup_frac: float = 0.3):
    """Visibility records for the gridding stage: ``randpar`` float32 [G, 3]
    holding (u/ν0, v/ν0, 0) in seconds like UVFITS random parameters, and
    ``data`` float32 [G, nc, nstokes, 3] = (re, im, wt).  About ``dup_frac`` of
    the records reuse an earlier record's (u, v) so that many cells receive
    several records and the ordered accumulation is exercised; ``flag_frac`` of
    the (record, channel) weights are ≤ 0."""
    rng = np.random.default_rng(seed)
    umax = umax if umax is not None else 0.95 * du * (nn // 2)
    r = umax * np.sqrt(rng.uniform(0, 1, ngroups))
    th = rng.uniform(-math.pi, math.pi, ngroups)
    u = r * np.cos(th)
    v = r * np.sin(th)
    ndup = int(dup_frac * ngroups)
    if ngroups > 1 and ndup:
        src = rng.integers(0, ngroups, ndup)
        dst = rng.integers(0, ngroups, ndup)
        u[dst] = u[src] + rng.uniform(-0.2, 0.2, ndup) * du
        v[dst] = v[src] + rng.uniform(-0.2, 0.2, ndup) * du
    randpar = np.zeros((ngroups, 3), dtype=np.float32)
    randpar[:, 0] = (u / nu0).astype(np.float32)
    randpar[:, 1] = (v / nu0).astype(np.float32)
    data = np.empty((ngroups, nc, nstokes, 3), dtype=np.float32)
    data[..., 0] = rng.standard_normal((ngroups, nc, nstokes)) * 10.0
    data[..., 1] = rng.standard_normal((ngroups, nc, nstokes)) * 10.0
    wt = rng.uniform(0.5, 2.0, (ngroups, nc, nstokes))
    wt[rng.uniform(0, 1, (ngroups, nc, nstokes)) < flag_frac] = -1.0
    data[..., 2] = wt
    return randpar, data
