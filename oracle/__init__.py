"""ORACLE / TEST INFRASTRUCTURE ONLY.

CPU checker for the estimator path.  Only tests/, ``__graft_entry__.smoke()``
and bench.py's CPU-baseline leg use this package; the product
(``amber_b200`` / libamber_cuda) never imports it.

* ``liboracle.so`` — our FP64 C restatement (``amber_oracle.c``), wrapped
  below with numpy arrays;
* ``_ref/`` — the reference's own C sources built unchanged against our FFTW
  shim (``Makefile``): ``ref_amber`` (as shipped, float), ``ref_amber_fast``
  (production flags, float), ``ref_amber64`` (``-Dfloat=double``) and
  ``ref_vcg`` (gridding stage).  :func:`run_ref_amber` / :func:`run_ref_vcg`
  drive them through files, exactly as the reference is used.
"""
from __future__ import annotations

import ctypes
import json
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
# Where the reference's own sources are read from (to build _ref/ and to import its Python
# readers in tests); override with AMBER_REF_DIR.  Absent on machines that only run the built files.
REFERENCE_SOURCES = os.environ.get("AMBER_REF_DIR", "/root/reference")
_lib = None

_dp = ctypes.POINTER(ctypes.c_double)
_fp = ctypes.POINTER(ctypes.c_float)
_ip = ctypes.POINTER(ctypes.c_int)
_i64p = ctypes.POINTER(ctypes.c_int64)


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            subprocess.run(["make", "-C", HERE, "oracle"], check=True, capture_output=True)
        L = ctypes.CDLL(path)
        L.orc_grid_vis.restype = ctypes.c_int
        L.orc_grid_vis.argtypes = [ctypes.c_long, ctypes.c_long, ctypes.c_double, ctypes.c_double, ctypes.c_float,
                                   ctypes.c_int, ctypes.c_long, ctypes.c_long, ctypes.c_long, _fp, _fp, _dp, _dp]
        L.orc_normalize.argtypes = [ctypes.c_long, ctypes.c_long, _dp, _dp]
        L.orc_cl_dnu.restype = None
        L.orc_cl_dnu.argtypes = [ctypes.c_long, ctypes.c_long, ctypes.c_double, _dp, _dp, ctypes.c_int, ctypes.c_double,
                                 ctypes.c_double, _dp, _dp, _dp, _dp, _ip]
        L.orc_uavg.argtypes = [ctypes.c_int, _dp, _dp, _dp]
        L.orc_triangles.restype = ctypes.c_int
        L.orc_triangles.argtypes = [ctypes.c_int, _dp, _ip, ctypes.c_int]
        L.orc_ng1.restype = ctypes.c_long
        L.orc_ng1.argtypes = [ctypes.c_double, ctypes.c_double]
        L.orc_calcr.restype = ctypes.c_int
        L.orc_calcr.argtypes = [ctypes.c_long, ctypes.c_long, _dp, ctypes.c_int, _dp, _dp, _dp, _dp, ctypes.c_int,
                                ctypes.c_int]
        for f in (L.orc_ring_map, L.orc_ring_mask_map):
            f.restype = ctypes.c_int
            f.argtypes = [ctypes.c_long, ctypes.c_long, _dp, ctypes.c_double, ctypes.c_double, ctypes.c_long,
                          ctypes.c_int, _dp, ctypes.c_int]
        L.orc_triangle.restype = ctypes.c_long
        L.orc_triangle.argtypes = [ctypes.c_long, ctypes.c_long, ctypes.c_int, ctypes.c_int, _ip, _dp, _dp, _dp,
                                   _dp, _dp, _dp, _dp, _i64p, _dp, ctypes.c_int]
        L.orc_triangle_absscale.argtypes = [ctypes.c_long, ctypes.c_long, ctypes.c_int, ctypes.c_int, _ip, _dp,
                                            _dp, _dp, _dp, ctypes.c_int]
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(t) if a is not None else None


NTHREADS = max(1, min(8, os.cpu_count() or 1))


def grid_vis(nn, nc, du, umax, nu_chan0, flag_key, randpar, data):
    """Gridding restatement; returns (re_im complex128 [NN, H, nc], ntig [NN, H, nc])."""
    randpar = np.ascontiguousarray(randpar, dtype=np.float32)
    data = np.ascontiguousarray(data, dtype=np.float32)
    g, npar = randpar.shape
    nstokes = data.shape[2]
    h = nn // 2 + 1
    re_im = np.zeros((nn, h, nc, 2), dtype=np.float64)
    ntig = np.zeros((nn, h, nc), dtype=np.float64)
    rc = lib().orc_grid_vis(nn, nc, du, umax, np.float32(nu_chan0), flag_key, g, npar, nstokes, _p(randpar, _fp),
                            _p(data, _fp), _p(re_im, _dp), _p(ntig, _dp))
    if rc != 0:
        raise ValueError("record outside the grid")
    return re_im[..., 0] + 1j * re_im[..., 1], ntig


def normalize(gv, counts):
    re_im = np.ascontiguousarray(np.stack([gv.real, gv.imag], axis=-1))
    ntig = np.ascontiguousarray(counts, dtype=np.float64).copy()
    nn, h, nc = counts.shape
    lib().orc_normalize(nn * h, nc, _p(re_im, _dp), _p(ntig, _dp))
    return re_im[..., 0] + 1j * re_im[..., 1], ntig


def uavg(ulow, uhigh):
    lo = np.ascontiguousarray(ulow, dtype=np.float64)
    hi = np.ascontiguousarray(uhigh, dtype=np.float64)
    out = np.zeros_like(lo)
    lib().orc_uavg(len(lo), _p(lo, _dp), _p(hi, _dp), _p(out, _dp))
    return out


def triangles(ulow, uhigh):
    ua = uavg(ulow, uhigh)
    n = lib().orc_triangles(len(ua), _p(ua, _dp), None, 0)
    tri = np.zeros((max(n, 1), 3), dtype=np.int32)
    lib().orc_triangles(len(ua), _p(ua, _dp), _p(tri, _ip), n)
    return tri[:n]


def ng1(uhigh, du):
    return int(lib().orc_ng1(float(uhigh), float(du)))


def calcr(ntig_norm, ulow, uhigh):
    nn, h, nc = ntig_norm.shape
    lo = np.ascontiguousarray(ulow, dtype=np.float64)
    hi = np.ascontiguousarray(uhigh, dtype=np.float64)
    ua = uavg(lo, hi)
    maxtri = int(lib().orc_triangles(len(ua), _p(ua, _dp), None, 0))
    rdata = np.zeros((max(maxtri, 1), 4), dtype=np.float64)
    nt = np.ascontiguousarray(ntig_norm, dtype=np.float64)
    n = lib().orc_calcr(nn, nc, _p(nt, _dp), len(lo), _p(lo, _dp), _p(hi, _dp), _p(ua, _dp), _p(rdata, _dp),
                        maxtri, NTHREADS)
    return rdata[:n]


def ring_maps(gv_norm, lo, hi, ng, mask=False, channels=None):
    """FP64 maps [nc][Ng1·Ng1] of one ring (all channels, or the listed ones)."""
    nn, h, nc = gv_norm.shape
    if mask:
        src = np.ascontiguousarray(gv_norm, dtype=np.float64)
    else:
        src = np.ascontiguousarray(np.stack([gv_norm.real, gv_norm.imag], axis=-1))
    out = np.zeros((nc, ng * ng), dtype=np.float64)
    fn = lib().orc_ring_mask_map if mask else lib().orc_ring_map
    for p in (range(nc) if channels is None else channels):
        row = np.zeros(ng * ng, dtype=np.float64)
        rc = fn(nn, nc, _p(src, _dp), float(lo), float(hi), ng, int(p), _p(row, _dp), 1)
        if rc != 0:
            raise ValueError("ring reaches outside the grid")
        out[p] = row
    return out


def triangle(m1, m2, m3, nc10, uf_chans=None, i1=None, i2=None, i3=None):
    """FP64 lag accumulation; returns (bldnu [nclen,nclen], numdnu int64, numtri or None, total_vcp)."""
    nc, k = m1.shape
    nclen = 2 * nc10 + 1
    uf = None if uf_chans is None else np.ascontiguousarray(uf_chans, dtype=np.int32)
    bl = np.zeros(nclen * nclen)
    nd = np.zeros(nclen * nclen, dtype=np.int64)
    nt = np.zeros(nclen * nclen) if i1 is not None else None
    arrs = [np.ascontiguousarray(a, dtype=np.float64) if a is not None else None for a in (m1, m2, m3, i1, i2, i3)]
    tot = lib().orc_triangle(k, nc, nc10, 0 if uf is None else len(uf), _p(uf, _ip), *[_p(a, _dp) for a in arrs],
                             _p(bl, _dp), _p(nd, _i64p), _p(nt, _dp), NTHREADS)
    return (bl.reshape(nclen, nclen), nd.reshape(nclen, nclen),
            None if nt is None else nt.reshape(nclen, nclen), int(tot))


def triangle_absscale(m1, m2, m3, nc10, uf_chans=None):
    nc, k = m1.shape
    nclen = 2 * nc10 + 1
    uf = None if uf_chans is None else np.ascontiguousarray(uf_chans, dtype=np.int32)
    out = np.zeros(nclen * nclen)
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (m1, m2, m3)]
    lib().orc_triangle_absscale(k, nc, nc10, 0 if uf is None else len(uf), _p(uf, _ip), *[_p(a, _dp) for a in arrs],
                                _p(out, _dp), NTHREADS)
    return out.reshape(nclen, nclen)


def estimate(real, version=1, tri_subset=None, with_absscale=False):
    """Full FP64 oracle pass over a synth.Realisation: normalise, calCR,
    then per closed triangle maps + lag accumulation.  Returns a list of dicts
    in calCR order (optionally restricted to ``tri_subset`` indices)."""
    gvn, ntn = normalize(real.gv, real.counts)
    rdata = calcr(ntn, real.ulow, real.uhigh)
    uf = real.uf_chans if real.flag_key == 1 else None
    out = []
    idxs = range(len(rdata)) if tri_subset is None else tri_subset
    for t in idxs:
        r1, r2, r3 = (int(v) for v in rdata[t, :3])
        ng = ng1(real.uhigh[r1], real.du)
        m = [ring_maps(gvn, real.ulow[r], real.uhigh[r], ng) for r in (r1, r2, r3)]
        im = [ring_maps(ntn, real.ulow[r], real.uhigh[r], ng, mask=True) for r in (r1, r2, r3)] if version == 2 \
            else [None] * 3
        bl, nd, nt, tot = triangle(*m, real.nc10, uf, *im)
        rec = dict(rp=t, r1=r1, r2=r2, r3=r3, ng1=ng, rdata_num=float(rdata[t, 3]), bldnu=bl, numdnu=nd,
                   numtri=nt, total_vcp=tot)
        if with_absscale:
            rec["absscale"] = triangle_absscale(*m, real.nc10, uf)
            if version == 2:
                rec["absscale_i"] = triangle_absscale(*im, real.nc10, uf)
        out.append(rec)
    return rdata, out


# ---- the reference's own code, built from its sources (oracle/_ref) -------------------------

def ref_available():
    return all(os.path.exists(os.path.join(REF_DIR, b)) for b in ("ref_amber", "ref_amber64", "ref_vcg", "ref_maps"))


def run_ref_amber(real, workdir, version=1, fp64=False, fast=False, rp_begin=0, rp_end=-1, nthreads=None,
                  rlzn=1):
    """Write ``real`` as amber input files under ``workdir`` and run the
    reference build.  Returns (json_stats, res_path)."""
    from amber_b200 import formats  # local import: formats is a plain file-format module
    data_path = os.path.join(workdir, "data")
    res_path = os.path.join(workdir, "res")
    os.makedirs(res_path, exist_ok=True)
    real.write(data_path, rlzn)
    params = os.path.join(workdir, "input_params_ess")
    formats.write_input_params_ess(params, 154.255e6, 40.0e3, 1.0, data_path)
    rings = os.path.join(workdir, "rings.txt")
    formats.write_rings_file(rings, real.ulow, real.uhigh)
    exe = "ref_amber64" if fp64 else ("ref_amber_fast" if fast else "ref_amber")
    uf_nc = len(real.uf_chans) if real.flag_key == 1 else 0
    cmd = [os.path.join(REF_DIR, exe), str(rlzn), "v2" if version == 2 else "v1", str(real.nc10), str(uf_nc), rings,
           str(rp_begin), str(rp_end), str(nthreads or NTHREADS), res_path, params]
    p = subprocess.run(cmd, capture_output=True, text=True, cwd=workdir)
    if p.returncode != 0:
        raise RuntimeError(f"{exe} failed: {p.stderr[-2000:]}")
    line = [ln for ln in p.stdout.splitlines() if ln.startswith("AMBER_REF_JSON ")][-1]
    return json.loads(line[len("AMBER_REF_JSON "):]), res_path


def run_ref_vcg(randpar, data, nu_chan0, nc, umax, fwhm, flag_key, workdir, collapse=False):
    """Run the reference's own gridding stage (3_vcg main + tgefuncs) on
    synthetic records; returns (gv complex [NN,H,nc], ntig, dU, NN).  ``collapse``
    runs it with the collapse key set (4 channels per output channel)."""
    from amber_b200 import formats
    vis = os.path.join(workdir, "vis.bin")
    formats.write_vis(vis, randpar, data, nu_chan0, 40.0e3, 1.0)
    params = os.path.join(workdir, "inputparameters")
    with open(params, "w") as f:
        f.write(f"{nc}\t{umax!r}\t{fwhm!r}\t1.\n")
    gvp = os.path.join(workdir, "GV_out")
    smp = os.path.join(workdir, "sampling_out")
    p = subprocess.run([os.path.join(REF_DIR, "ref_vcg"), vis, params, gvp, str(flag_key), "1" if collapse else "0", "1",
                        smp],
                       capture_output=True, text=True, cwd=workdir)
    if p.returncode != 0:
        raise RuntimeError(f"ref_vcg failed: {p.stdout[-1000:]} {p.stderr[-1000:]}")
    gv, du, fk = formats.read_gv(gvp)
    nn = gv.shape[0]
    ntig = formats.read_sampling(smp, nn, gv.shape[2])
    return gv, ntig, du, nn


def tmpdir():
    return tempfile.mkdtemp(prefix="amber_oracle_")


def cl_dnu(real, nb=15, umin=1.0, umax=500.0):
    """MAPS two-point function (orc_cl_dnu: amber_funcs.c:1418-1488 driven as 4_fbe/maps.c:179-210)
    of a synth.Realisation's normalised grid.  Returns dict(cldnu [nb, nc], cldnu_abs, numdnu [nc],
    binu [nb], num [nb]) — binu/num as the last channel pair leaves them."""
    gvn, ntn = normalize(real.gv, real.counts)
    nn, h, nc = ntn.shape
    re_im = np.ascontiguousarray(np.stack([gvn.real, gvn.imag], axis=-1))
    ntn = np.ascontiguousarray(ntn)
    out = dict(cldnu=np.zeros((nb, nc)), cldnu_abs=np.zeros((nb, nc)), numdnu=np.zeros(nc), binu=np.zeros(nb),
               num=np.zeros(nb, dtype=np.int32))
    lib().orc_cl_dnu(nn, nc, float(real.du), _p(re_im, _dp), _p(ntn, _dp), nb, float(umin), float(umax),
                     _p(out["cldnu"], _dp), _p(out["cldnu_abs"], _dp), _p(out["numdnu"], _dp), _p(out["binu"], _dp),
                     _p(out["num"], _ip))
    return out


def run_ref_maps(real, workdir, nb=15, umin=1.0, umax=500.0, rlzn=1):
    """The reference's own cl_dnu over every channel pair (oracle/_ref/ref_maps).  Returns
    (dict(cldnu, numdnu, binu, num at full precision; pairs_s: the pair loop's time), path of the
    maps.c-style text file)."""
    from amber_b200 import formats
    data_path = os.path.join(workdir, "data")
    real.write(data_path, rlzn)
    params = os.path.join(workdir, "input_params_ess")
    formats.write_input_params_ess(params, 154.255e6, 40.0e3, 1.0, data_path)
    txt, binf = os.path.join(workdir, "cldnu"), os.path.join(workdir, "cldnu.bin")
    p = subprocess.run([os.path.join(REF_DIR, "ref_maps"), str(rlzn), params, str(nb), repr(float(umin)),
                        repr(float(umax)), txt, binf], capture_output=True, text=True, cwd=workdir)
    if p.returncode != 0:
        raise RuntimeError(f"ref_maps failed: {p.stdout[-1000:]} {p.stderr[-1000:]}")
    nc = real.gv.shape[2]
    timing = json.loads([ln for ln in p.stdout.splitlines() if ln.startswith("MAPS_REF_JSON ")][-1][14:])
    raw = open(binf, "rb").read()
    d = np.frombuffer(raw, dtype=np.float64, count=nb * nc + nc + nb)
    num = np.frombuffer(raw, dtype=np.int32, offset=8 * (nb * nc + nc + nb), count=nb)
    return dict(cldnu=d[: nb * nc].reshape(nb, nc).copy(), numdnu=d[nb * nc: nb * nc + nc].copy(),
                binu=d[nb * nc + nc:].copy(), num=num.copy(), pairs_s=timing["pairs_s"]), txt


def collapse_channels(gv, ntig, n):
    """collapse_channels (3_vcg/tgefuncs.c:816-838): output channel k of every cell is the sum
    of channels k·n .. k·n + n − 1, added in that order from 0.0; trailing channels dropped.
    gv complex [NN, H, nc], ntig [NN, H, nc]."""
    ncoll = gv.shape[2] // n
    re = np.zeros(gv.shape[:2] + (ncoll,))
    im = np.zeros_like(re)
    nt = np.zeros_like(re)
    for k in range(n):
        sl = slice(k, ncoll * n, n)
        re = re + gv.real[:, :, sl]
        im = im + gv.imag[:, :, sl]
        nt = nt + ntig[:, :, sl]
    return re + 1j * im, nt


# ---- cylindrical bispectrum (analysis stage), restated in numpy ----

def blackman_nuttall(m):
    """Blackman–Nuttall window of length m (mfunc_winds.py:17-31)."""
    n = np.arange(m)
    a0, a1, a2, a3 = 0.3635819, 0.4891775, 0.1365995, 0.0106411
    return a0 - a1 * np.cos(2 * np.pi * n / (m - 1)) + a2 * np.cos(4 * np.pi * n / (m - 1)) - a3 * np.cos(
        6 * np.pi * n / (m - 1))


def cyl_bs(lag, den, nc10, n_cut, mabs_norm, rc, rc_prime, dnu, window=False, div=1.0, float32=False):
    """Cylindrical bispectrum of one lag array [nclen, nclen]:
    fold_quadrants (mabs_funcs.py:210-222) of lag/div and of the normaliser ``den``, the ratio
    over mabs_norm, cut_nan (259-260), optionally the Blackman–Nuttall window of mabs_win
    (mfunc_winds.py:88-103), then Bdnu2Bk_fft (mabs_funcs.py:325-334) / cylbs_win (122-136).

    ``float32`` repeats the v2 chain's rounding: read_bsout_float_v2 (mabs_funcs.py:190-205)
    returns float32 arrays, so the reference folds and divides them in float32 before the
    window (float64) promotes the result.  The v1 chain is float64 from the reader's division
    by Num onwards."""
    dt = np.float32 if float32 else np.float64

    def fold(a):
        a = np.array(a, dtype=dt)
        lower = a[nc10:, :].copy()
        lower[1:, :] += a[:nc10, :][::-1, ::-1]
        return lower
    lag = np.asarray(lag, dtype=dt)
    if div != 1.0:
        lag = lag / np.float64(div)
    # like the reference, divide the whole folded array; empty edge cells (0/0) fall in the cut
    with np.errstate(divide="ignore", invalid="ignore"):
        t = fold(lag) / (dt(mabs_norm) if float32 else mabs_norm) / fold(den)
    d = t[: t.shape[0] - n_cut, n_cut:-n_cut]
    if window:
        m = d.shape[1]
        w2 = np.outer(blackman_nuttall(m), blackman_nuttall(m))
        d = d * w2[m // 2:, :]
    n = d.shape[1]
    res = np.fft.fftshift(np.fft.irfft2(np.fft.ifftshift(d, axes=1), axes=(1, 0), s=(n, n)))
    length = n * dnu * rc_prime
    return res * (rc ** 4 * length * length)
