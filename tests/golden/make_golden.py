"""Regenerate the golden fixtures in this folder from the REFERENCE's own code.

Runs oracle/_ref/ref_amber64 (4_fbe/amber_funcs.c + vars.c built unchanged
with -Dfloat=double), ref_amber (as shipped, float) and ref_vcg (3_vcg/main.c +
tgefuncs.c unchanged) on small seeded synthetic inputs and stores inputs and
outputs as compressed .npz files:

  est_<name>.npz   — grid sums, counts, ring edges, nc10, channels, and the
                     reference's closed_rings plus, per triangle, its v1
                     (FP64 and float builds) and v2 (FP64) lag arrays;
  grid_<name>.npz  — visibility records and the reference's GV/sampling sums
                     (coll_*: with the collapse key set);
  maps_<name>.npz  — a grid and the MAPS two-point function the reference's own
                     cl_dnu computes from it (oracle/_ref/ref_maps);
  cylbs_ref.npz    — seeded lag arrays and the cylindrical bispectra that the
                     reference's analysis Python (mabs_funcs.get_cyl_BS,
                     mfunc_winds.cylbs_win) computes from them;
  c2_rp217_ref64.npz — one Ng1 = 740 triangle of the single-realisation
                     workload at full size, v1 and v2, from the FP64 build
                     (outputs only; the inputs are regenerated from their seed).

Needs the reference sources (make -C oracle ref); run from the repo root:
    python tests/golden/make_golden.py

Reproducibility: the reference's accumulation loop is an OpenMP loop whose
partial sums are added in thread-schedule order, so a fresh run reproduces the
lag arrays to rounding only (within 3e-16 of the largest value for the FP64
build, 1e-7 for the float build); the triangle lists, counts, gridding, MAPS and
cylindrical-bispectrum outputs come out bit-identical.  The tests compare with
tolerances far above that (1e-10 of the per-cell sum of |products| for FP64).
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from amber_b200 import formats, synth  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

EST_CASES = {
    # name: (nn, nc, seed, nbins, hi, nc10, flagged)
    "unflagged32": (32, 8, 3, 4, 14.0, 3, None),
    "flagged48": (48, 12, 4, 5, 21.0, 5, [0, 5, 11]),
    "dup40": (40, 10, 6, 4, 18.0, 6, None),  # uf_chans with a repeated channel, see below
}


def est_case(name, nn, nc, seed, nbins, hi, nc10, flagged):
    real = synth.tiny(nn, nc, seed=seed, nbins=nbins, hi=hi, nc10=nc10, flagged=flagged)
    if name == "dup40":
        real.flag_key = 1
        real.uf_chans = np.array([0, 1, 2, 3, 3, 5, 6, 8, 9], dtype=np.int32)  # channel 3 twice, 4 and 7 absent
    nclen = real.nclen
    rec = dict(gv=real.gv, counts=real.counts, ulow=real.ulow, uhigh=real.uhigh, nc10=real.nc10,
               uf_chans=real.uf_chans, flag_key=real.flag_key, du=real.du)
    st64, rp64 = oracle.run_ref_amber(real, oracle.tmpdir(), version=1, fp64=True)
    rdata = formats.read_closed_rings(rp64)
    rec["rdata"] = rdata
    st32, rp32 = oracle.run_ref_amber(real, oracle.tmpdir(), version=1, fp64=False)
    sv2, rpv2 = oracle.run_ref_amber(real, oracle.tmpdir(), version=2, fp64=True)
    b64, n64, b32, ntri, num, bv2, nv2, inv = [], [], [], [], [], [], [], []
    for r1, r2, r3, _ in rdata:
        r1, r2, r3 = int(r1), int(r2), int(r3)
        t, nu, bl, nd = formats.read_bsout_v1(os.path.join(rp64, formats.bsout_name(1, r1, r2, r3, 1)), nclen,
                                              np.float64)
        b64.append(bl); n64.append(nd); ntri.append(t); num.append(nu)
        _, _, bl32, nd32 = formats.read_bsout_v1(os.path.join(rp32, formats.bsout_name(1, r1, r2, r3, 1)), nclen)
        assert (nd32 == nd).all()
        b32.append(bl32)
        iv, blv, ndv = formats.read_bsout_v2(os.path.join(rpv2, formats.bsout_name(2, r1, r2, r3, 1)), nclen,
                                             np.float64)
        bv2.append(blv); nv2.append(ndv); inv.append(iv)
    rec.update(bldnu64=np.array(b64), numdnu=np.array(n64), bldnu32=np.array(b32), ntri=np.array(ntri),
               num=np.array(num), bldnu_v2=np.array(bv2), numtri_v2=np.array(nv2), inv_ng=np.array(inv),
               total_vcp=st64["total_vcp"])
    np.savez_compressed(os.path.join(OUT, f"est_{name}.npz"), **rec)
    print(name, "triangles", len(rdata), "total_vcp", st64["total_vcp"])


def c2_full_case(rp=217):
    """One Ng1 = 740 triangle of the single-realisation workload (256² grid, 128 channels with the
    block-edge flags, 16 bins, nc10 = 63) at full size, through the reference's FP64 build, v1 and
    v2.  Only outputs are stored: the inputs are regenerated by synth.config2(seed=1) (seeded), and
    a SHA-256 of the grid and the counts guards against the generator drifting."""
    import hashlib
    real = synth.config2(seed=1)
    nclen = real.nclen
    st1, rp1 = oracle.run_ref_amber(real, oracle.tmpdir(), version=1, fp64=True, rp_begin=rp, rp_end=rp + 1)
    st2, rp2 = oracle.run_ref_amber(real, oracle.tmpdir(), version=2, fp64=True, rp_begin=rp, rp_end=rp + 1)
    rdata = formats.read_closed_rings(rp1)
    r1, r2, r3 = (int(v) for v in rdata[rp, :3])
    t, nu, bl, nd = formats.read_bsout_v1(os.path.join(rp1, formats.bsout_name(1, r1, r2, r3, 1)), nclen, np.float64)
    iv, blv, ndv = formats.read_bsout_v2(os.path.join(rp2, formats.bsout_name(2, r1, r2, r3, 1)), nclen, np.float64)
    h = hashlib.sha256(np.ascontiguousarray(real.gv).tobytes() + np.ascontiguousarray(real.counts).tobytes())
    np.savez_compressed(os.path.join(OUT, f"c2_rp{rp}_ref64.npz"), rp=rp, tri=np.array([r1, r2, r3]),
                        rdata_num=rdata[rp, 3], ntri=t, num=nu, bldnu64=bl, numdnu=nd, bldnu_v2=blv, numtri_v2=ndv,
                        inv_ng=iv, total_vcp=st1["total_vcp"], inputs_sha256=h.hexdigest())
    print("c2 rp", rp, (r1, r2, r3), "total_vcp", st1["total_vcp"], "v1", st1["accum_s"], "s, v2", st2["accum_s"], "s")


GRID_CASES = {
    # name: (nc, ngroups, seed, flag_key, fwhm_arcmin, umax_wavelengths)
    "flag1": (5, 2000, 11, 1, 1480.73, 30.0),
    "flag0": (4, 1200, 12, 0, 1480.73, 25.0),
}
# the same, run with the collapse key (4 channels per output channel; 9 → 2, one dropped)
GRID_COLL_CASES = {
    "coll_flag1": (9, 600, 13, 1, 1480.73, 25.0),
}


def grid_case(name, nc, ngroups, seed, flag_key, fwhm, umax, collapse=False):
    # dU the reference derives from the beam (tgefuncs.c:306-309)
    import math
    theta0 = 0.6 * fwhm * math.pi / (180. * 60.)
    du = math.sqrt(math.log(2)) / (math.pi * theta0)
    nn = 2 * int(math.ceil(umax / du))
    randpar, data = synth.make_visibilities(nn, du, nc, ngroups, seed, umax=umax * 1.02)
    gv, ntig, du_ref, nn_ref = oracle.run_ref_vcg(randpar, data, np.float32(synth.NU0), nc, umax, fwhm, flag_key,
                                                  oracle.tmpdir(), collapse=collapse)
    np.savez_compressed(os.path.join(OUT, f"grid_{name}.npz"), randpar=randpar, data=data, nu0=np.float32(synth.NU0),
                        du=du_ref, nn=nn_ref, umax=umax, flag_key=flag_key, gv=gv, ntig=ntig, fwhm=fwhm,
                        n_collapse=4 if collapse else 1)
    print(name, "NN", nn_ref, "dU", du_ref, "cells hit", int((ntig.sum(axis=2) > 0).sum()))


def cylbs_case(nc10=30, seed=11):
    """The analysis stage's lag→k step, computed by the reference's own Python functions:
    mabs_funcs.get_cyl_BS (v1 file: counts normalise, the reader divides by Num) and
    mfunc_winds.cylbs_win (v2 file: mask sums normalise, Blackman–Nuttall window), on seeded lag
    arrays written in the reference's file formats.  matplotlib is absent here, so a stub stands in
    for the modules' unused plotting import."""
    import importlib
    import types
    sys.modules.setdefault("matplotlib", types.ModuleType("matplotlib"))
    sys.modules.setdefault("matplotlib.pyplot", types.ModuleType("matplotlib.pyplot"))
    sys.path.insert(0, oracle.REFERENCE_SOURCES)
    mf = importlib.import_module("mabs_funcs")
    nclen = 2 * nc10 + 1
    mf.nc10, mf.nclen, mf.ncsize = nc10, nclen, nclen * nclen
    mw = importlib.import_module("mfunc_winds")
    rng = np.random.default_rng(seed)
    bl = rng.standard_normal((nclen, nclen)).astype(np.float32)
    counts = rng.integers(50, 400, (nclen, nclen)).astype(np.int32)
    mask = rng.uniform(0.5, 2.0, (nclen, nclen)).astype(np.float32)
    ntri, num = 0.25, 3.5
    d = oracle.tmpdir()
    formats.write_bsout_v1(os.path.join(d, formats.bsout_name(1, 3, 2, 1, 1)), ntri, num, bl, counts)
    formats.write_bsout_v2(os.path.join(d, formats.bsout_name(2, 3, 2, 1, 1)), 1.0 / 64, bl, mask)
    v1, _ = mf.get_cyl_BS(3, 2, 1, d, 1)
    v2 = mw.cylbs_win(3, 2, 1, d)
    np.savez_compressed(os.path.join(OUT, "cylbs_ref.npz"), nc10=nc10, bl=bl, counts=counts, mask=mask, num=num,
                        n_cut=mf.n_nancut, mabs_norm=mf.mabs_norm, rc=mf.rc, rc_prime=mf.rc_prime, dnu=mf.dnu_mwa,
                        v1=v1, v2=v2)
    print("cylbs", v1.shape, v2.shape)


def maps_case(name="maps_flagged40", seed=51):
    """The reference's own cl_dnu over every channel pair (ref_maps: amber_funcs.c unchanged, driven
    as 4_fbe/maps.c drives it) on a small flagged realisation, with maps.c's bins (15, 1, 500) and a
    finer set (24 bins from 0.7 to 30)."""
    real = synth.tiny(40, 10, seed=seed, nbins=4, hi=18.0, flagged=[3, 8])
    out = dict(gv=real.gv, counts=real.counts, du=real.du)
    for tag, (nb, umin, umax) in {"maps": (15, 1.0, 500.0), "fine": (24, 0.7, 30.0)}.items():
        r, _ = oracle.run_ref_maps(real, oracle.tmpdir(), nb, umin, umax)
        out.update({f"{tag}_{k}": v for k, v in r.items()})
        out[f"{tag}_bins"] = np.array([nb, umin, umax])
    np.savez_compressed(os.path.join(OUT, f"{name}.npz"), **out)
    print(name, "nonempty bins", int((out["maps_num"] > 0).sum()), int((out["fine_num"] > 0).sum()))


if __name__ == "__main__":
    if not oracle.ref_available():
        raise SystemExit("build the reference first: make -C oracle ref")
    for k, v in EST_CASES.items():
        est_case(k, *v)
    for k, v in GRID_CASES.items():
        grid_case(k, *v)
    for k, v in GRID_COLL_CASES.items():
        grid_case(k, *v, collapse=True)
    cylbs_case()
    maps_case()
    c2_full_case()  # ~10 min on 8 host threads
