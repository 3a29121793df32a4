"""amber_b200 — B200-native AMBER estimator hot path.

The product is ``libamber_cuda.so`` (hand-written sm_100a CUDA behind the C
ABI of ``include/amber_cuda.h``).  This module loads it with ctypes and
mirrors the reference's own call sequence (4_fbe/amber.c:40-304):

    est = Estimator(precision="mixed")          # or "fp64": the plain path
    est.load_grid(gv_sums, counts, Du, flag_key) # initialize + ReadGVnAC_gridding + normalize_data
    est.set_rings(ULow, UHigh)                   # annular_rings
    est.set_channels(nc10, uf_chans)             # get_uf_chans + vcp table
    rdata = est.calcr()                          # calCR + read_rings
    Ntri, Num, bldnu, numdnu = est.triangle_v1(r1, r2, r3, rdata[rp, 3])
    inv, bldnu, numdnu = est.triangle_v2(r1, r2, r3)

There is no CPU fallback: without the library or without an sm_100 GPU every
call raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libamber_cuda.so")

AMBER_OK = 0
ERRORS = {-1: "bad argument", -2: "out of device memory / over budget", -3: "CUDA error", -4: "timeout",
          -5: "overflow", -6: "call order", -7: "no sm_100 device"}
PREC = {"fp64": 0, "mixed": 1, "bf16x3": 2, "fp64_abs": 3}

# every entry point include/amber_cuda.h declares
EXPORTS = (
    "amber_cuda_default_opts", "amber_cuda_create", "amber_cuda_destroy", "amber_cuda_last_error",
    "amber_cuda_load_grid_packed", "amber_cuda_load_grid", "amber_cuda_load_grid_device", "amber_cuda_set_rings",
    "amber_cuda_get_uavg",
    "amber_cuda_set_channels", "amber_cuda_calcr", "amber_cuda_ng1", "amber_cuda_triangle_v1",
    "amber_cuda_triangle_v2", "amber_cuda_triangles", "amber_cuda_triangles_run", "amber_cuda_triangles_fetch",
    "amber_cuda_last_run_stats", "amber_cuda_last_run_breakdown", "amber_cuda_last_run_shape", "amber_cuda_grid_vis",
    "amber_cuda_enqueue", "amber_cuda_wait", "amber_cuda_result", "amber_cuda_engine_stats",
    "amber_cuda_tile_choices", "amber_cuda_cyl_bs", "amber_cuda_grid_vis_collapsed", "amber_cuda_cl_dnu",
    "amber_cuda_shard_plan",
)


class AmberError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"libamber_cuda error {code} ({ERRORS.get(code, '?')}): {msg}")
        self.code = code


class CylBsParams(ctypes.Structure):
    _fields_ = [("n_cut", ctypes.c_int), ("window", ctypes.c_int), ("denominator", ctypes.c_int),
                ("mabs_norm", ctypes.c_double), ("rc", ctypes.c_double), ("rc_prime", ctypes.c_double),
                ("dnu_mhz", ctypes.c_double)]


def reference_cylbs_constants():
    """The analysis stage's constants (mabs_funcs.py:4-28), restated by the same formulas:
    n_nancut, mabs_norm = fact·rjfac³ (beam solid angle × Jy→mK cubed), rc, rc_prime, dnu_mwa."""
    import math
    theta_0 = 0.6 * 24.68 * math.pi / 180
    fact = math.pi * theta_0 * theta_0 / 3
    nu0, k_b, c = 154.255e6, 1.38e3, 3e8
    rjfac = 2.0 * k_b * nu0 * nu0 / (c * c) / 1e3
    return dict(n_cut=8, mabs_norm=fact * rjfac ** 3, rc=9210.11291939594, rc_prime=17.0, dnu_mhz=0.04)


def cylbs_params(window=False, denominator="counts", **const) -> CylBsParams:
    """amber_cuda_cylbs_params: the reference's analysis constants, overridden by ``const``;
    ``denominator`` is "counts" (v1 chain) or "mask" (the v2 run's sampling-mask sums)."""
    if denominator not in ("counts", "mask"):
        raise ValueError("denominator is 'counts' or 'mask'")
    k = reference_cylbs_constants()
    unknown = set(const) - set(k)
    if unknown:
        raise TypeError(f"unknown constants {sorted(unknown)}")
    k.update(const)
    return CylBsParams(int(k["n_cut"]), int(bool(window)), 0 if denominator == "counts" else 1, float(k["mabs_norm"]),
                       float(k["rc"]), float(k["rc_prime"]), float(k["dnu_mhz"]))


class Request(ctypes.Structure):
    _fields_ = [("N1", ctypes.c_long), ("nc", ctypes.c_long), ("Du", ctypes.c_double), ("flag_key", ctypes.c_int),
                ("re_im", ctypes.POINTER(ctypes.c_double)), ("ntig", ctypes.POINTER(ctypes.c_double)),
                ("Nr", ctypes.c_int), ("ULow", ctypes.POINTER(ctypes.c_double)),
                ("UHigh", ctypes.POINTER(ctypes.c_double)), ("nc10", ctypes.c_int), ("uf_nc", ctypes.c_int),
                ("uf_chans", ctypes.POINTER(ctypes.c_int)), ("want_v2", ctypes.c_int),
                ("cylbs", ctypes.POINTER(CylBsParams)), ("inputs_on_device", ctypes.c_int)]


class EngineInfo(ctypes.Structure):
    _fields_ = [("requests_done", ctypes.c_long), ("rounds", ctypes.c_long), ("contraction_launches", ctypes.c_long),
                ("max_active", ctypes.c_long), ("queued", ctypes.c_long), ("active", ctypes.c_long),
                ("peak_bytes", ctypes.c_size_t), ("budget_bytes", ctypes.c_size_t), ("products", ctypes.c_double),
                ("busy_ms", ctypes.c_double), ("setup_ms", ctypes.c_double), ("maps_ms", ctypes.c_double),
                ("contract_ms", ctypes.c_double), ("finish_ms", ctypes.c_double), ("kernel_launches", ctypes.c_long),
                ("contract_kernel_ms", ctypes.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Opts(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("precision", ctypes.c_int), ("hbm_budget", ctypes.c_size_t),
                ("stream", ctypes.c_void_p), ("chunk_px", ctypes.c_int), ("tile_n", ctypes.c_int)]


_dp = ctypes.POINTER(ctypes.c_double)
_fp = ctypes.POINTER(ctypes.c_float)
_ip = ctypes.POINTER(ctypes.c_int)
_i32p = ctypes.POINTER(ctypes.c_int32)
_i64p = ctypes.POINTER(ctypes.c_int64)
_vp = ctypes.c_void_p
_lib = None


def load_library():
    """Load libamber_cuda.so (raises if it has not been built: no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m amber_b200.build` "
                          "(there is no CPU fallback)")
    L = ctypes.CDLL(LIB_PATH)
    L.amber_cuda_default_opts.argtypes = [ctypes.POINTER(Opts)]
    L.amber_cuda_create.argtypes = [ctypes.POINTER(Opts), ctypes.POINTER(_vp)]
    L.amber_cuda_destroy.argtypes = [_vp]
    L.amber_cuda_destroy.restype = None
    L.amber_cuda_last_error.argtypes = [_vp]
    L.amber_cuda_last_error.restype = ctypes.c_char_p
    L.amber_cuda_load_grid_packed.argtypes = [_vp, ctypes.c_long, ctypes.c_long, ctypes.c_double, ctypes.c_int, _dp,
                                              _dp]
    L.amber_cuda_load_grid_device.argtypes = L.amber_cuda_load_grid_packed.argtypes
    L.amber_cuda_load_grid.argtypes = [_vp, ctypes.c_long, ctypes.c_long, ctypes.c_double, ctypes.c_int,
                                       ctypes.POINTER(_dp), ctypes.POINTER(_dp), ctypes.POINTER(_dp)]
    L.amber_cuda_set_rings.argtypes = [_vp, ctypes.c_int, _dp, _dp]
    L.amber_cuda_get_uavg.argtypes = [_vp, _dp]
    L.amber_cuda_set_channels.argtypes = [_vp, ctypes.c_int, ctypes.c_int, _ip]
    L.amber_cuda_calcr.argtypes = [_vp, ctypes.c_int, _ip, _dp]
    L.amber_cuda_ng1.argtypes = [_vp, ctypes.c_int]
    L.amber_cuda_ng1.restype = ctypes.c_long
    L.amber_cuda_triangle_v1.argtypes = [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, _fp, _i32p,
                                         _dp, _dp]
    L.amber_cuda_triangle_v2.argtypes = [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, _fp, _fp, _dp]
    L.amber_cuda_triangles.argtypes = [_vp, ctypes.c_int, _ip, ctypes.c_int, _dp, _i64p, _dp]
    L.amber_cuda_triangles_run.argtypes = [_vp, ctypes.c_int, _ip, ctypes.c_int]
    L.amber_cuda_triangles_fetch.argtypes = [_vp, _dp, _i64p, _dp]
    L.amber_cuda_last_run_stats.argtypes = [_vp, _dp, _dp]
    L.amber_cuda_last_run_shape.argtypes = [_vp, _ip, _ip, _ip]
    L.amber_cuda_last_run_breakdown.argtypes = [_vp, _dp, _dp, _dp, ctypes.POINTER(ctypes.c_long),
                                                ctypes.POINTER(ctypes.c_long)]
    L.amber_cuda_grid_vis.argtypes = [_vp, ctypes.c_long, ctypes.c_long, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_float, ctypes.c_int, ctypes.c_long, ctypes.c_long, ctypes.c_long, _fp,
                                      _fp, _dp, _dp]
    L.amber_cuda_enqueue.argtypes = [_vp, ctypes.POINTER(Request), _i64p]
    L.amber_cuda_wait.argtypes = [_vp, ctypes.c_int64, ctypes.c_int, _ip]
    L.amber_cuda_result.argtypes = [_vp, ctypes.c_int64, ctypes.c_int, _dp, _dp, _i64p, _dp, _dp, _dp]
    L.amber_cuda_engine_stats.argtypes = [_vp, ctypes.POINTER(EngineInfo)]
    L.amber_cuda_tile_choices.argtypes = [_vp, ctypes.c_int, _ip, _ip, _fp, _fp]
    L.amber_cuda_shard_plan.argtypes = [ctypes.c_int, _ip, ctypes.POINTER(ctypes.c_long), ctypes.c_int, _ip]
    L.amber_cuda_grid_vis_collapsed.argtypes = [_vp, ctypes.c_long, ctypes.c_long, ctypes.c_double, ctypes.c_double,
                                                ctypes.c_float, ctypes.c_int, ctypes.c_long, ctypes.c_long,
                                                ctypes.c_long, _fp, _fp, ctypes.c_long, _dp, _dp]
    L.amber_cuda_cl_dnu.argtypes = [_vp, ctypes.c_int, ctypes.c_double, ctypes.c_double, _dp, _dp, _dp, _ip]
    L.amber_cuda_cyl_bs.argtypes = [_vp, ctypes.POINTER(CylBsParams), _dp, _dp]
    _lib = L
    return L


def _ptr(a, t):
    return None if a is None else a.ctypes.data_as(t)


class Estimator:
    """One libamber_cuda context (one device, one host thread).

    precision: "mixed" (int8 tensor-core digits, ≤1e-6 of Σ|products| per lag cell), "fp64"
    (plain FP64, ≤1e-10), "fp64_abs" (FP64 over |maps|: the error scale) or "bf16x3"
    (comparison only).  hbm_budget: bytes the context may hold (0: most of the free memory).
    stream: a cudaStream_t to launch on.  chunk_px: pixels per contraction work unit, i.e. per
    FP64 partial lag tile, rounded up to 256-pixel blocks (0: planned); it sets only the summation grouping.
    tile_n: accepted for compatibility and ignored (the lag-space contraction has no tile width).  Every call raises AmberError with the library's message on failure.
    """

    def __init__(self, device: int = 0, precision: str = "mixed", hbm_budget: int = 0, stream: int | None = None,
                 chunk_px: int = 0, tile_n: int = 0):
        self._L = load_library()
        o = Opts(device, PREC[precision], hbm_budget, stream or None, chunk_px, tile_n)
        h = _vp()
        rc = self._L.amber_cuda_create(ctypes.byref(o), ctypes.byref(h))
        if rc != AMBER_OK:
            raise AmberError(rc, "amber_cuda_create failed (an sm_100 GPU is required)")
        self._h = h
        self.precision = precision
        self.nc10 = None
        self.n1 = None
        self.nc = None

    def close(self):
        if getattr(self, "_h", None):
            self._L.amber_cuda_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc):
        if rc != AMBER_OK:
            raise AmberError(rc, self._L.amber_cuda_last_error(self._h).decode(errors="replace"))

    # ---- inputs -----------------------------------------------------------
    def load_grid(self, gv_sums: np.ndarray, counts: np.ndarray, du: float, flag_key: int):
        """Upload summed visibilities (complex [NN, NN/2+1, nc]) and counts; normalised on the device."""
        nn, h, nc = gv_sums.shape
        ri = np.ascontiguousarray(gv_sums, dtype=np.complex128).view(np.float64)
        nt = np.ascontiguousarray(counts, dtype=np.float64)
        self._check(self._L.amber_cuda_load_grid_packed(self._h, nn, nc, float(du), int(flag_key), _ptr(ri, _dp),
                                                        _ptr(nt, _dp)))
        self.n1, self.nc = nn, nc

    def load_grid_raw(self, re_im_ptr: int, ntig_ptr: int, nn: int, nc: int, du: float, flag_key: int):
        """Same as load_grid but from raw host addresses (e.g. pinned buffers)."""
        self._check(self._L.amber_cuda_load_grid_packed(self._h, nn, nc, float(du), int(flag_key),
                                                        ctypes.cast(re_im_ptr, _dp), ctypes.cast(ntig_ptr, _dp)))
        self.n1, self.nc = nn, nc

    def load_grid_device(self, re_im_ptr: int, ntig_ptr: int, nn: int, nc: int, du: float, flag_key: int):
        """Same as load_grid_raw but from device addresses on this context's device (a cube kept
        resident in HBM, e.g. torch tensors): normalised in place, nothing copied in."""
        self._check(self._L.amber_cuda_load_grid_device(self._h, nn, nc, float(du), int(flag_key),
                                                        ctypes.cast(re_im_ptr, _dp), ctypes.cast(ntig_ptr, _dp)))
        self.n1, self.nc = nn, nc

    def load_grid_cells(self, gv_sums, counts, du, flag_key):
        """Pointer-per-cell form (the reference's double** arrays)."""
        nn, h, nc = gv_sums.shape
        ncell = nn * h
        re = np.ascontiguousarray(gv_sums.real.reshape(ncell, nc))
        im = np.ascontiguousarray(gv_sums.imag.reshape(ncell, nc))
        nt = np.ascontiguousarray(counts.reshape(ncell, nc), dtype=np.float64)
        mk = lambda a: (_dp * ncell)(*[a[i].ctypes.data_as(_dp) for i in range(ncell)])
        self._check(self._L.amber_cuda_load_grid(self._h, nn, nc, float(du), int(flag_key), mk(re), mk(im), mk(nt)))
        self.n1, self.nc = nn, nc

    def set_rings(self, ulow, uhigh):
        lo = np.ascontiguousarray(ulow, dtype=np.float64)
        hi = np.ascontiguousarray(uhigh, dtype=np.float64)
        self._check(self._L.amber_cuda_set_rings(self._h, len(lo), _ptr(lo, _dp), _ptr(hi, _dp)))
        self.nr = len(lo)

    def uavg(self):
        out = np.zeros(self.nr)
        self._check(self._L.amber_cuda_get_uavg(self._h, _ptr(out, _dp)))
        return out

    def set_channels(self, nc10: int, uf_chans=None):
        uf = None if uf_chans is None else np.ascontiguousarray(uf_chans, dtype=np.int32)
        self._check(self._L.amber_cuda_set_channels(self._h, int(nc10), 0 if uf is None else len(uf),
                                                    _ptr(uf, _ip)))
        self.nc10 = int(nc10)

    # ---- estimator --------------------------------------------------------
    def calcr(self) -> np.ndarray:
        n = ctypes.c_int(0)
        self._check(self._L.amber_cuda_calcr(self._h, 0, ctypes.byref(n), None))
        out = np.zeros((max(n.value, 1), 4))
        self._check(self._L.amber_cuda_calcr(self._h, n.value, ctypes.byref(n), _ptr(out, _dp)))
        return out[: n.value]

    def ng1(self, r1: int) -> int:
        return int(self._L.amber_cuda_ng1(self._h, int(r1)))

    @property
    def nclen(self):
        return 2 * self.nc10 + 1

    def triangle_v1(self, r1, r2, r3, rdata_num):
        n = self.nclen
        bl = np.zeros((n, n), dtype=np.float32)
        nd = np.zeros((n, n), dtype=np.int32)
        ntri, num = ctypes.c_double(), ctypes.c_double()
        self._check(self._L.amber_cuda_triangle_v1(self._h, r1, r2, r3, float(rdata_num), _ptr(bl, _fp),
                                                   _ptr(nd, _i32p), ctypes.byref(ntri), ctypes.byref(num)))
        return ntri.value, num.value, bl, nd

    def triangle_v2(self, r1, r2, r3):
        n = self.nclen
        bl = np.zeros((n, n), dtype=np.float32)
        nd = np.zeros((n, n), dtype=np.float32)
        inv = ctypes.c_double()
        self._check(self._L.amber_cuda_triangle_v2(self._h, r1, r2, r3, _ptr(bl, _fp), _ptr(nd, _fp),
                                                   ctypes.byref(inv)))
        return inv.value, bl, nd

    def run(self, tri, want_v2=False):
        tri = np.ascontiguousarray(np.asarray(tri, dtype=np.int32).reshape(-1, 3))
        self._check(self._L.amber_cuda_triangles_run(self._h, len(tri), _ptr(tri, _ip), int(bool(want_v2))))

    def last_run_shape(self):
        """(triangles, nclen, has v2 mask sums) of the results the last run left on the device."""
        t, n, v = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self._check(self._L.amber_cuda_last_run_shape(self._h, ctypes.byref(t), ctypes.byref(n), ctypes.byref(v)))
        return t.value, n.value, bool(v.value)

    def fetch(self, want_v2=False):
        ntri, n, _ = self.last_run_shape()
        bl = np.zeros((ntri, n, n))
        nd = np.zeros((ntri, n, n), dtype=np.int64)
        nt = np.zeros((ntri, n, n)) if want_v2 else None
        self._check(self._L.amber_cuda_triangles_fetch(self._h, _ptr(bl, _dp), _ptr(nd, _i64p), _ptr(nt, _dp)))
        return bl, nd, nt

    def triangles(self, tri, want_v2=False):
        """FP64 lag arrays for many triangles: (bldnu, numdnu int64, numtri or None)."""
        self.run(tri, want_v2)
        return self.fetch(want_v2)

    def last_run_stats(self):
        p, ms = ctypes.c_double(), ctypes.c_double()
        self._check(self._L.amber_cuda_last_run_stats(self._h, ctypes.byref(p), ctypes.byref(ms)))
        return p.value, ms.value

    def cl_dnu(self, nb=15, umin=1.0, umax=500.0) -> dict:
        """MAPS two-point function of the loaded grid (amber_cuda_cl_dnu; maps.c's NB = 15, Umin1 = 1,
        Umax1 = 500 by default): dict(cldnu [nb, nc], numdnu [nc], binu [nb], num [nb])."""
        if self.nc is None:
            raise AmberError(-6, "cl_dnu: no grid loaded")
        out = dict(cldnu=np.zeros((nb, self.nc)), numdnu=np.zeros(self.nc), binu=np.zeros(nb),
                   num=np.zeros(nb, dtype=np.int32))
        self._check(self._L.amber_cuda_cl_dnu(self._h, int(nb), float(umin), float(umax), _ptr(out["cldnu"], _dp),
                                              _ptr(out["numdnu"], _dp), _ptr(out["binu"], _dp), _ptr(out["num"], _ip)))
        return out

    def file_num(self, rdata) -> np.ndarray:
        """The Num a v1 file holds for each calCR row, (Ng1/N1)²·rdata[3] (amber.c:193-202); the v1
        reader returns bldnu / Num, so it is the tri_div of the get_cyl_BS chain."""
        rdata = np.asarray(rdata, dtype=np.float64).reshape(-1, 4)
        g = np.array([self.ng1(int(r1)) / self.n1 for r1 in rdata[:, 0]])
        return g * g * rdata[:, 3]

    def cyl_bs(self, window=False, denominator="counts", tri_div=None, **const):
        """Cylindrical bispectra [ntri, N, N] of the last run (amber_cuda_cyl_bs); ``denominator`` is
        "counts" (v1) or "mask" (the sampling-mask sums of a v2 run); ``tri_div`` divides each
        triangle's sums (Num for the v1 chain); constants default to the reference analysis stage's
        (reference_cylbs_constants)."""
        p = cylbs_params(window, denominator, **const)
        ntri, nclen, _ = self.last_run_shape()
        n = max(nclen - 2 * p.n_cut, 1)
        out = np.zeros((max(ntri, 1), n, n))
        td = None
        if tri_div is not None:
            td = np.ascontiguousarray(tri_div, dtype=np.float64).reshape(-1)
            if len(td) != ntri:
                raise ValueError(f"tri_div has {len(td)} entries, the last run {ntri} triangles")
        self._check(self._L.amber_cuda_cyl_bs(self._h, ctypes.byref(p), _ptr(td, _dp), _ptr(out, _dp)))
        return out[:ntri]

    def tile_choices(self) -> dict:
        """Kept for compatibility with the earlier tile-width autotuner: the lag-space contraction has no
        tile width to choose, so this is empty."""
        n = self._L.amber_cuda_tile_choices(self._h, 0, None, None, None, None)
        cls, bn = np.zeros(max(n, 1), np.int32), np.zeros(max(n, 1), np.int32)
        t32, t64 = np.zeros(max(n, 1), np.float32), np.zeros(max(n, 1), np.float32)
        self._L.amber_cuda_tile_choices(self._h, n, _ptr(cls, _ip), _ptr(bn, _ip), _ptr(t32, _fp), _ptr(t64, _fp))
        return {int(cls[i]): (int(bn[i]), float(t32[i]), float(t64[i])) for i in range(n)}

    def last_run_breakdown(self):
        """(ms_maps, ms_contract, ms_reduce, kernel_launches, contract_launches) of the last run."""
        a, b, c = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        n, m = ctypes.c_long(), ctypes.c_long()
        self._check(self._L.amber_cuda_last_run_breakdown(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c),
                                                          ctypes.byref(n), ctypes.byref(m)))
        return a.value, b.value, c.value, n.value, m.value

    def fetch_into(self, bldnu_ptr: int, numtri_ptr: int | None = None):
        """Copy the last run's FP64 lag arrays into caller-owned (e.g. pinned) host memory."""
        self._check(self._L.amber_cuda_triangles_fetch(self._h, ctypes.cast(bldnu_ptr, _dp), None,
                                                       None if numtri_ptr is None else ctypes.cast(numtri_ptr, _dp)))

    # ---- gridding ---------------------------------------------------------
    def grid_vis(self, nn, nc, du, umax, nu_chan0, flag_key, randpar, data, n_collapse=1):
        """Grid visibility records (amber_cuda_grid_vis_collapsed): randpar float32 [G, npar],
        data float32 [G, nchan ≥ nc, nstokes, 3]; the first nc channels are gridded and, with
        n_collapse > 1, summed in groups of n_collapse.  Returns (complex [NN, H, nc // n_collapse],
        counts of the same shape)."""
        randpar = np.ascontiguousarray(randpar, dtype=np.float32)
        data = np.asarray(data, dtype=np.float32)
        if data.ndim != 4 or data.shape[1] < nc or data.shape[3] != 3 or data.shape[0] != randpar.shape[0]:
            raise ValueError("data must be [G, nchan >= nc, nstokes, 3] with G = len(randpar)")
        data = np.ascontiguousarray(data[:, :nc])
        g, npar = randpar.shape
        nstokes = data.shape[2]
        h = nn // 2 + 1
        ncoll = nc // max(int(n_collapse), 1)
        ri = np.zeros((nn, h, max(ncoll, 1), 2))
        nt = np.zeros((nn, h, max(ncoll, 1)))
        self._check(self._L.amber_cuda_grid_vis_collapsed(self._h, nn, nc, float(du), float(umax),
                                                          np.float32(nu_chan0), int(flag_key), g, npar, nstokes,
                                                          _ptr(randpar, _fp), _ptr(data, _fp), int(n_collapse),
                                                          _ptr(ri, _dp), _ptr(nt, _dp)))
        return ri[..., 0] + 1j * ri[..., 1], nt


def _request_of(real, want_v2, cyl=None, with_cube=True):
    """Request struct for a synth.Realisation, with the numpy buffers it points to (keep them alive
    until enqueue returns: the library copies them)."""
    if with_cube:
        ri = np.ascontiguousarray(real.gv, dtype=np.complex128).view(np.float64)
        nt = np.ascontiguousarray(real.counts, dtype=np.float64)
    else:
        ri = np.zeros(2)
        nt = np.zeros(1)
    lo = np.ascontiguousarray(real.ulow, dtype=np.float64)
    hi = np.ascontiguousarray(real.uhigh, dtype=np.float64)
    uf = np.ascontiguousarray(real.uf_chans if real.flag_key == 1 else np.zeros(1), dtype=np.int32)
    q = Request(real.gv.shape[0], real.gv.shape[2], float(real.du), int(real.flag_key), _ptr(ri, _dp), _ptr(nt, _dp),
                len(lo), _ptr(lo, _dp), _ptr(hi, _dp), int(real.nc10), len(uf) if real.flag_key == 1 else 0,
                _ptr(uf, _ip), int(bool(want_v2)), None if cyl is None else ctypes.pointer(cyl), 0)
    return q, (ri, nt, lo, hi, uf, cyl)


class Engine:
    """Batched requests on one context: enqueue realisations (any mix of sizes), wait for them,
    fetch their results.  The library's worker thread admits requests by HBM footprint and runs
    the map-set batches of all admitted requests together (amber_cuda_enqueue)."""

    def __init__(self, est: Estimator):
        self.est = est
        self._L = est._L
        self._cyl_n = {}  # ticket -> N of the cylindrical bispectra it asked for

    def enqueue(self, real, want_v2=True, cyl_bs=None, device_cube=None) -> int:
        """Queue a realisation; ``cyl_bs`` (a dict of cylbs_params arguments, e.g.
        ``dict(window=True, denominator="mask")``) asks for its cylindrical bispectra as well.
        ``device_cube=(re_im_ptr, ntig_ptr)``: the realisation's summed grid and counts are already
        in device memory (packed layout); the request reads them there, so keep them unchanged until
        it is done."""
        cyl = None if cyl_bs is None else cylbs_params(**cyl_bs)
        q, keep = _request_of(real, want_v2, cyl, with_cube=device_cube is None)
        if device_cube is not None:
            q.re_im = ctypes.cast(device_cube[0], _dp)
            q.ntig = ctypes.cast(device_cube[1], _dp)
            q.inputs_on_device = 1
        t = ctypes.c_int64()
        self.est._check(self._L.amber_cuda_enqueue(self.est._h, ctypes.byref(q), ctypes.byref(t)))
        del keep
        if cyl is not None:
            self._cyl_n[t.value] = 2 * (int(real.nc10) + 1 - cyl.n_cut) - 1
        return t.value

    def wait(self, ticket: int, timeout_ms: int = -1) -> int:
        n = ctypes.c_int()
        self.est._check(self._L.amber_cuda_wait(self.est._h, ticket, timeout_ms, ctypes.byref(n)))
        return n.value

    def result(self, ticket: int, real, want_v2=True):
        """(rdata, bldnu, numdnu, numtri, latency_ms) of a finished request; FP64 lag arrays
        [ntri, nclen²], int64 counts.  A request enqueued with ``cyl_bs`` adds its cylindrical
        bispectra [ntri, N, N] as a sixth item."""
        n = self.wait(ticket)
        nclen = 2 * real.nc10 + 1
        rd = np.zeros((max(n, 1), 4))
        bl = np.zeros((max(n, 1), nclen * nclen))
        nd = np.zeros((max(n, 1), nclen * nclen), dtype=np.int64)
        nt = np.zeros((max(n, 1), nclen * nclen)) if want_v2 else None
        lat = ctypes.c_double()
        ncyl = self._cyl_n.get(ticket)
        cy = None if ncyl is None else np.zeros((max(n, 1), ncyl, ncyl))
        self.est._check(self._L.amber_cuda_result(self.est._h, ticket, max(n, 1), _ptr(rd, _dp), _ptr(bl, _dp),
                                                  _ptr(nd, _i64p), _ptr(nt, _dp), ctypes.byref(lat), _ptr(cy, _dp)))
        self._cyl_n.pop(ticket, None)
        out = (rd[:n], bl[:n], nd[:n], (None if nt is None else nt[:n]), lat.value)
        return out if cy is None else out + (cy[:n],)

    def stats(self) -> dict:
        i = EngineInfo()
        self.est._check(self._L.amber_cuda_engine_stats(self.est._h, ctypes.byref(i)))
        return i.as_dict()


def estimate(real, precision="mixed", version=1, tri_subset=None, est: Estimator | None = None):
    """Run the whole estimator on a synth.Realisation; returns (rdata, results)
    where results[i] = dict(r1, r2, r3, bldnu (FP64), numdnu (int64), numtri)."""
    own = est is None
    est = est or Estimator(precision=precision)
    try:
        est.load_grid(real.gv, real.counts, real.du, real.flag_key)
        est.set_rings(real.ulow, real.uhigh)
        est.set_channels(real.nc10, real.uf_chans if real.flag_key == 1 else None)
        rdata = est.calcr()
        idx = list(range(len(rdata))) if tri_subset is None else list(tri_subset)
        tri = rdata[idx, :3].astype(np.int32)
        bl, nd, nt = est.triangles(tri, want_v2=(version == 2))
        out = []
        for i, t in enumerate(idx):
            out.append(dict(rp=t, r1=int(tri[i, 0]), r2=int(tri[i, 1]), r3=int(tri[i, 2]), ng1=est.ng1(int(tri[i, 0])),
                            rdata_num=float(rdata[t, 3]), bldnu=bl[i], numdnu=nd[i],
                            numtri=None if nt is None else nt[i]))
        return rdata, out
    finally:
        if own:
            est.close()
