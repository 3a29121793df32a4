"""Benchmark of the AMBER estimator hot path on B200.

Workload (one "step"): the single-realisation case — a 256² uv grid, 128
channels (channels 0-1 and 30-31 of every 32-channel block flagged), 16
log-spaced annular bins from 2 to 120 cells, all lag pairs |Δν| < 64
(nc10 = 63), v2 output — pushed through the whole estimator: calCR, then for
all 218 closed triangles the ring maps and the triple-product lag
accumulation of both the visibility maps (bldnu) and the sampling-mask maps
(numdnu).  Inputs are seeded synthetic data of that shape (there is no
public dataset for this path).

Metric: lag-triple products per second, one product being one term
D_r1(x,p1)·D_r2(x,p2)·D_r3(x,p3) of the reference's loop (4_fbe/amber.c:261-263);
per triangle total_vcp·Ng1², counted for the D and the I (mask) sums.

* value — device time of the run with the grid already resident in HBM;
* e2e   — the same through the C ABI from pinned host buffers: grid upload and
  normalisation, rings, channels, calCR, the run, and the copy of every lag
  array back to the host, all inside the timed region;
* fp64_plain — the plain FP64 GPU path on the same GPU over a bounded sample;
* roofline — the contraction kernel, algorithmic flops (2 per product) per
  launch over its CUDA-event time, against the measured bf16 dense peak;
* cpu_baseline — the reference's own OpenMP loop (oracle/_ref/ref_amber_fast,
  its sources built unchanged) on the host cores over a bounded sample;
* ensemble — 64 realisations of uneven size through the request engine
  (amber_cuda_enqueue), end to end, with mixed vs plain FP64 on a subset;
* serving — a prefix of the Poisson request stream enqueued at its arrival
  times: p50/p99 latency and throughput, FP64 one-at-a-time beside it.

`--impl reference` times that same reference build as the reference arm.
Multi-GPU: one process per GPU (torchrun), each rank runs its own realisation
(seed 1 + rank): weak scaling, no collective on the data path; timing is the
max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "lag-triple products/s vs plain FP64 on same GPU @<=1e-6 rel err; p50/p99 latency"
UNIT = "lag-triple products/s"
WORKLOAD = dict(workload="single realisation: 256^2 grid, 128 channels (4 of every 32 flagged), "
                         "16 log bins 2-120 cells, nc10=63, v2 (D and mask sums), all 218 closed triangles",
                grid=256, channels=128, bins=16, nc10=63, du=0.5, version=2)


# DRAM bytes per lag-triple product of contract_i8_kernel, from one ncu capture of a full launch
# (triangle rp=140 of the single-realisation workload: 227.51 MB for 810152 * 125316 products).
# Every map row is read once per launch, so traffic grows with products.
DRAM_BYTES_PER_PRODUCT = 227.51e6 / (810152 * 125316)


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return p, "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        if not shutil.which("nvidia-smi"):
            return
        fd, self.path = tempfile.mkstemp(prefix="clocks_", suffix=".csv")
        os.close(fd)
        self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                      "-i", str(self.index), "-lms", "200"], stdout=open(self.path, "w"),
                                     stderr=subprocess.DEVNULL)

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        loaded = [s for s in sm if mx and s > 0.3 * max(mx)] or sm
        return {"sm_mhz": float(np.median(loaded)) if loaded else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def cpu_reference_sample(real, nthreads=None, rp_pick=None, version=1, fast=True):
    """Time the reference's own accumulation loop (ref_amber_fast) on one triangle."""
    import oracle  # the reference build and its driver live in oracle/
    from amber_b200 import formats
    wd = tempfile.mkdtemp(prefix="amber_ref_")
    try:
        nthreads = nthreads or os.cpu_count() or 1
        if rp_pick is None:
            # the last triangle: largest ring r1 = 15, Ng1 = 740 — the kind of triangle that dominates the step
            rp_pick = len(oracle.triangles(real.ulow, real.uhigh)) - 1
        st, _ = oracle.run_ref_amber(real, wd, version=version, fp64=False, fast=fast, rp_begin=rp_pick,
                                     rp_end=rp_pick + 1, nthreads=nthreads)
        return st, rp_pick
    finally:
        shutil.rmtree(wd, ignore_errors=True)


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import oracle
    from amber_b200 import synth
    if not oracle.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "reference build oracle/_ref missing (make -C oracle ref)"}))
        return 0
    real = synth.config2()
    rates, times = [], []
    st = None
    for i in range(args.warmup + args.steps):
        st, rp = cpu_reference_sample(real)
        rate = st["products"] / st["accum_s"]
        if i >= args.warmup:
            rates.append(rate)
            times.append(st["accum_s"])
    value = float(np.median(rates))
    sample = (f"triangle rp={rp} of the workload (Ng1=740, total_vcp={st['total_vcp']}), v1 accumulation loop "
              f"timed like amber.c:230,285; maps excluded")
    out = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * float(np.median(times)),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
           "config": WORKLOAD,
           "cpu_baseline": {"value": value, "unit": UNIT, "cores": st["threads"], "kind": "reference",
                            "sample": sample},
           "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))
    return 0


def _engine_run(amber_b200, reals, precision, dev):
    """All realisations through one context's request engine; returns (wall s, products, results, stats)."""
    with amber_b200.Estimator(device=dev, precision=precision) as est:
        eng = amber_b200.Engine(est)
        p0 = eng.stats()["products"]
        t0 = time.perf_counter()
        tickets = [eng.enqueue(r, want_v2=True) for r in reals]
        res = [eng.result(t, r, want_v2=True) for t, r in zip(tickets, reals)]
        wall = time.perf_counter() - t0
        st = eng.stats()
    return wall, st["products"] - p0, res, st


def ensemble_section(amber_b200, synth, dev):
    """Batched ensemble: the 64 realisations of uneven size (sides 96-320, 24-160 channels, 10 %
    flags, 12 bins) through the request engine, end to end (inputs from host memory, every lag
    array back); plus mixed vs plain FP64 on a fixed subset of the same ensemble."""
    specs = synth.config3_specs()
    t_gen = time.perf_counter()
    reals = [synth.from_spec(s) for s in specs]
    t_gen = time.perf_counter() - t_gen
    _engine_run(amber_b200, reals[48:49], "mixed", dev)  # warm-up (allocations, twiddles)
    wall, prod, _, st = _engine_run(amber_b200, reals, "mixed", dev)
    sub = [0, 16, 48]
    sreals = [reals[i] for i in sub]
    w_m, p_m, r_m, _ = _engine_run(amber_b200, sreals, "mixed", dev)
    w_f, p_f, r_f, _ = _engine_run(amber_b200, sreals, "fp64", dev)
    _, _, r_a, _ = _engine_run(amber_b200, sreals, "fp64_abs", dev)
    err = 0.0
    for m, f, a in zip(r_m, r_f, r_a):
        err = max(err, float((np.abs(m[1] - f[1]) / (a[1] + 1e-300)).max()),
                  float((np.abs(m[3] - f[3]) / (a[3] + 1e-300)).max()))
        assert np.array_equal(m[2], f[2])  # counts exact
    return {"workload": "ensemble: 64 realisations, sides {96,128,192,256,320}, 24-160 channels, 10 % flags, "
                        "12 log bins 2..0.47*side, nc10=nc/2-1, v2, all closed triangles, seeds 100-163",
            "value": prod / wall, "unit": UNIT, "products": prod, "wall_s": wall,
            "timing": "end to end through amber_cuda_enqueue/wait/result from host memory (wall clock)",
            "engine": {k: st[k] for k in ("rounds", "contraction_launches", "max_active", "peak_bytes", "busy_ms",
                                          "setup_ms", "maps_ms", "contract_ms", "finish_ms")},
            "fp64_plain": {"sample": "realisations 0, 16, 48 of the ensemble (sides 256/192/96), same engine",
                           "value": p_f / w_f, "mixed_same_sample": p_m / w_m, "speedup": (p_m / w_m) / (p_f / w_f),
                           "max_rel_err_vs_fp64": err, "err_scale": "sum of |products| per lag cell"},
            "generation_s": t_gen}


def serving_section(amber_b200, synth, dev, n=8):
    """Serving stream: the first n requests of the Poisson stream (50 req/s; sides {64..384},
    16-256 channels, 6-20 bins) enqueued at their arrival times; latency = arrival to result
    ready.  The stream as specified is far beyond one GPU's capacity (~1.5e17 products arriving
    in 39 s), so only a prefix runs; the plain FP64 one-at-a-time path is timed on two small
    requests of the prefix."""
    reqs = synth.config5_requests()[:n]
    reals = [synth.from_spec(q) for q in reqs]
    _engine_run(amber_b200, [synth.from_spec(dict(reqs[4], nn=64))], "mixed", dev)  # warm-up
    with amber_b200.Estimator(device=dev, precision="mixed") as est:
        eng = amber_b200.Engine(est)
        p0 = eng.stats()["products"]
        t0 = time.perf_counter()
        tickets = []
        for q, r in zip(reqs, reals):
            delay = (q["arrival"] - reqs[0]["arrival"]) - (time.perf_counter() - t0)
            if delay > 0:
                time.sleep(delay)
            tickets.append(eng.enqueue(r, want_v2=True))
        lat = [eng.result(t, r, want_v2=True)[4] for t, r in zip(tickets, reals)]
        wall = time.perf_counter() - t0
        st = eng.stats()
        prod = st["products"] - p0
    small = sorted(range(n), key=lambda i: reqs[i]["nn"] ** 2 * reqs[i]["nc"] * reqs[i]["nbins"])[:2]
    f_prod, f_wall, f_lat = 0.0, 0.0, []
    for i in small:
        with amber_b200.Estimator(device=dev, precision="fp64") as e64:
            t = time.perf_counter()
            amber_b200.estimate(reals[i], precision="fp64", version=2, est=e64)
            f_lat.append(1e3 * (time.perf_counter() - t))
            f_prod += e64.last_run_stats()[0]
            f_wall += time.perf_counter() - t
    return {"workload": f"serving: first {n} requests of the Poisson stream (50 req/s), sides/channels/bins as drawn",
            "requests": n, "value": prod / wall, "unit": UNIT, "products": prod, "wall_s": wall,
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "latency_ms": [round(x, 1) for x in lat],
            "engine": {k: st[k] for k in ("rounds", "contraction_launches", "max_active", "peak_bytes")},
            "fp64_one_at_a_time": {"requests": small, "value": f_prod / f_wall, "latency_ms": f_lat,
                                   "sizes": [(reqs[i]["nn"], reqs[i]["nc"], reqs[i]["nbins"]) for i in small]}}


def config4_section(amber_b200, synth, dev, args):
    """The large cube (512^2 grid, 384 channels, 15 % flags, 24 bins 2-240, nc10=191): too large
    for a default run (~4.7e15 products), so a fixed sample of its closed triangles: the four with
    the largest maps (Ng1 = 1460) and two small ones, mixed precision, plus plain FP64 and its
    error on one mid-size triangle."""
    t_gen = time.perf_counter()
    real = synth.config4()
    t_gen = time.perf_counter() - t_gen
    res = {}
    for prec in ("mixed", "fp64", "fp64_abs"):
        with amber_b200.Estimator(device=dev, precision=prec) as est:
            est.load_grid(real.gv, real.counts, real.du, real.flag_key)
            est.set_rings(real.ulow, real.uhigh)
            est.set_channels(real.nc10, real.uf_chans)
            tri = est.calcr()[:, :3].astype(np.int32)
            mid = len(tri) // 3
            sample = np.concatenate([tri[:2], tri[-4:]]) if prec == "mixed" else tri[[mid]]
            if prec == "mixed":
                est.run(tri[[mid]], want_v2=True)  # the FP64 comparison triangle, also warms up
                ref = est.fetch(want_v2=True)
            est.run(sample, want_v2=True)
            p, ms = est.last_run_stats()
            res[prec] = dict(products=p, ms=ms, out=est.fetch(want_v2=True), ntri=len(tri),
                             ng1=[est.ng1(int(t[0])) for t in sample])
            if prec == "mixed":
                res["mixed_mid"] = ref
    (mb, _, mt) = res["mixed_mid"]
    (fb, _, ft), (ab, _, at) = res["fp64"]["out"], res["fp64_abs"]["out"]
    err = max(float((np.abs(mb - fb) / (ab + 1e-300)).max()), float((np.abs(mt - ft) / (at + 1e-300)).max()))
    m = res["mixed"]
    return {"workload": "large cube: 512^2 grid, 384 channels, 15 % random flags, 24 log bins 2..240, nc10=191, v2",
            "sample": f"6 of its {m['ntri']} closed triangles (the first two and the four with Ng1=1460)",
            "value": m["products"] / (m["ms"] * 1e-3), "unit": UNIT, "products": m["products"], "device_ms": m["ms"],
            "ng1": m["ng1"],
            "fp64_plain": {"sample": "one mid-list triangle", "value": res["fp64"]["products"] / (res["fp64"]["ms"] * 1e-3),
                           "max_rel_err_vs_fp64": err, "err_scale": "sum of |products| per lag cell"},
            "generation_s": t_gen}


def config1_section(amber_b200, synth, dev, reps=5):
    """The reference's own CPU-runnable case, whole (128^2 grid, 32 channels, 8 bins 2-60, nc10=31,
    all 46 closed triangles, v1): the C ABI from host buffers (grid upload, rings, channels, calCR,
    every triangle, lag arrays back) against the reference's complete run on all host threads
    (oracle/_ref/ref_amber_fast: its sources built unchanged with the production flags)."""
    real = synth.config1()
    out = {"workload": "config 1, whole run: 128^2 grid, 32 channels, 8 log bins 2-60, nc10=31, v1, 46 triangles"}
    for prec in ("mixed", "fp64"):
        with amber_b200.Estimator(device=dev, precision=prec) as est:
            times, products = [], 0.0
            for r in range(reps + 1):
                t0 = time.perf_counter()
                est.load_grid(real.gv, real.counts, real.du, real.flag_key)
                est.set_rings(real.ulow, real.uhigh)
                est.set_channels(real.nc10)
                rd = est.calcr()
                bl, nd, _ = est.triangles(rd[:, :3].astype(np.int32), want_v2=False)
                if r:  # the first pass warms up (autotuner, allocations)
                    times.append(time.perf_counter() - t0)
                products = est.last_run_stats()[0]
        out[prec] = {"wall_ms_median": 1e3 * float(np.median(times)), "triangles": int(len(rd)), "products": products,
                     "value": products / float(np.median(times)), "unit": UNIT}
    try:
        import oracle
        if oracle.ref_available():
            wd = tempfile.mkdtemp(prefix="amber_c1_")
            try:
                st, _ = oracle.run_ref_amber(real, wd, version=1, fast=True, nthreads=os.cpu_count())
            finally:
                shutil.rmtree(wd, ignore_errors=True)
            out["reference"] = {"total_s": st["total_s"], "accum_s": st["accum_s"], "maps_s": st["maps_s"],
                                "threads": st["threads"], "products": st["products"],
                                "value_accum": st["products"] / st["accum_s"], "unit": UNIT,
                                "note": "accum_s is the reference's own timer scope (amber.c:230,285); maps_s runs "
                                        "its map builder on the oracle's FP64 DFT in place of FFTW, which is slower"}
            out["speedup_vs_reference_accum"] = st["accum_s"] / (out["mixed"]["wall_ms_median"] * 1e-3)
    except Exception as e:  # the comparison is a report, not the measurement
        out["reference_error"] = str(e)[:200]
    return out


def stages_section(amber_b200, synth, dev, reps=5):
    """The stages either side of the contraction, on the single-realisation workload: the
    cylindrical bispectra of all 218 triangles after a v2 run (both analysis chains), and the
    gridding of 100k visibility records (128 channels) without and with the 4-channel collapse.
    Each figure is the median wall time of a synchronous C-ABI call, host copies included."""
    real = synth.config2(seed=1)
    res = {"workload": "stages beside the contraction: cylindrical bispectra of the single-realisation run "
                       "(218 triangles, nc10=63, n_cut=8, N=111); gridding of 100k records x 128 channels "
                       "onto the 256^2 grid"}

    def med(f):
        f()
        ts = []
        for _ in range(reps):
            t0 = time.perf_counter()
            f()
            ts.append(time.perf_counter() - t0)
        return 1e3 * float(np.median(ts))

    with amber_b200.Estimator(device=dev, precision="mixed") as est:
        est.load_grid(real.gv, real.counts, real.du, real.flag_key)
        est.set_rings(real.ulow, real.uhigh)
        est.set_channels(real.nc10, real.uf_chans)
        rd = est.calcr()
        est.run(rd[:, :3].astype(np.int32), want_v2=True)
        num = est.file_num(rd)
        res["cyl_bs_v1_ms"] = med(lambda: est.cyl_bs(tri_div=num))
        res["cyl_bs_v2_window_ms"] = med(lambda: est.cyl_bs(window=True, denominator="mask"))
        res["triangles"] = int(len(rd))
        nn, du, nc = 256, 0.5, 128
        randpar, data = synth.make_visibilities(nn, du, nc, 100000, 91)
        umax = 0.95 * du * nn / 2
        res["grid_ms"] = med(lambda: est.grid_vis(nn, nc, du, umax, np.float32(synth.NU0), 1, randpar, data))
        res["grid_collapse4_ms"] = med(lambda: est.grid_vis(nn, nc, du, umax, np.float32(synth.NU0), 1, randpar, data,
                                                            n_collapse=4))
        res["records"] = int(len(randpar))
        res["record_bytes"] = int(randpar.nbytes + data.nbytes)
    return res


def gridding_section(amber_b200, synth, dev, reps=5):
    """Gridding alone (amber_cuda_grid_vis, 3_vcg's group_loop_gridding): 100k visibility records x 128
    channels x 2 Stokes onto the 256^2 grid, flag_key 1.  Reports the median wall time of the
    synchronous call (records up, grid down) and the algorithmic bytes of the device work: the
    RR payload read once (12 B per record-channel) plus u, v (8 B per record), and the grid written
    once (24 B per cell-channel: re, im, count)."""
    nn, du, nc, nrec = 256, 0.5, 128, 100000
    randpar, data = synth.make_visibilities(nn, du, nc, nrec, 91)
    umax = 0.95 * du * nn / 2
    ts = []
    with amber_b200.Estimator(device=dev, precision="fp64") as est:
        for _ in range(reps + 1):
            t0 = time.perf_counter()
            est.grid_vis(nn, nc, du, umax, np.float32(synth.NU0), 1, randpar, data)
            ts.append(time.perf_counter() - t0)
    h = nn // 2 + 1
    return {"workload": f"gridding: {nrec} records x {nc} channels x 2 Stokes onto the {nn}^2 grid (flag_key 1)",
            "grid_call_ms_median": 1e3 * float(np.median(ts[1:])),
            "algorithmic_bytes": int(nrec * (8 + 12 * nc) + nn * h * nc * 24),
            "record_bytes_copied_in": int(randpar.nbytes + data.nbytes)}


def maps_section(amber_b200, synth, dev):
    """The MAPS two-point function (amber_cuda_cl_dnu; maps.c's 15 bins from 1 to 500) of the
    single-realisation grid, against the reference's own cl_dnu pair loop (oracle/_ref/ref_maps,
    one host thread as maps.c runs it) on the same grid."""
    real = synth.config2(seed=1)
    with amber_b200.Estimator(device=dev, precision="fp64") as est:
        est.load_grid(real.gv, real.counts, real.du, real.flag_key)
        out = est.cl_dnu()  # warm-up
        times = []
        for _ in range(5):
            t0 = time.perf_counter()
            out = est.cl_dnu()
            times.append(time.perf_counter() - t0)
    nc = real.gv.shape[2]
    res = {"workload": "MAPS C_l(dnu) of the single-realisation grid: 256^2 cells, 128 channels, 15 log bins 1-500",
           "pairs": nc * (nc + 1) // 2, "call_ms_median": 1e3 * float(np.median(times)),
           "call_ms_min": 1e3 * float(min(times))}
    try:
        import oracle
        if oracle.ref_available():
            wd = tempfile.mkdtemp(prefix="amber_maps_")
            try:
                ref, _ = oracle.run_ref_maps(real, wd)
            finally:
                shutil.rmtree(wd, ignore_errors=True)
            res["reference_pairs_s"] = ref["pairs_s"]
            res["speedup_vs_reference"] = ref["pairs_s"] / (res["call_ms_median"] * 1e-3)
            res["bit_identical"] = all(np.array_equal(out[k], ref[k]) for k in ("cldnu", "numdnu", "binu", "num"))
    except Exception as e:  # the comparison is a report, not the measurement
        res["reference_error"] = str(e)[:200]
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="amber_b200", choices=["amber_b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--tri-subset", default="", help="comma-separated triangle indices (profiling runs only)")
    ap.add_argument("--tile-n", type=int, default=0, choices=[0, 32, 64, 128],
                    help="fix the contraction's p3 tile width instead of the autotuner's choice (profiling runs: "
                         "under a profiler the tuner's trial timings are not representative)")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the batched-ensemble measurement")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving-stream measurement")
    ap.add_argument("--config1", action="store_true",
                    help="measure the reference's whole CPU-runnable case (config 1) beside the reference's own run")
    ap.add_argument("--stages", action="store_true",
                    help="time the stages beside the contraction (cylindrical bispectra, gridding with collapse)")
    ap.add_argument("--maps", action="store_true",
                    help="measure the MAPS two-point function (amber_cuda_cl_dnu) instead of the default step")
    ap.add_argument("--gridding", action="store_true",
                    help="time the gridding stage alone (100k records x 128 channels onto 256^2)")
    ap.add_argument("--config4", action="store_true",
                    help="measure a fixed sample of the large cube (512^2, 384 channels) instead of the default step")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)

    import torch
    import torch.distributed as dist
    import amber_b200
    from amber_b200 import build, synth

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    build.build()

    if args.config4:
        if rank == 0:
            c4 = config4_section(amber_b200, synth, local, args)
            print(json.dumps(dict(metric=METRIC, impl="amber_b200", n_gpus=1, higher_is_better=True,
                                  dtype="int8 tensor-core digits, int32 accumulate, fp64 reduce", data="synthetic",
                                  config={"workload": c4["workload"]}, **{k: v for k, v in c4.items() if k != "workload"})))
        return 0

    if args.config1:
        if rank == 0:
            c1 = config1_section(amber_b200, synth, local)
            print(json.dumps(dict(metric=METRIC, impl="amber_b200", n_gpus=1, higher_is_better=True, data="synthetic",
                                  config={"workload": c1["workload"]}, **{k: v for k, v in c1.items() if k != "workload"})))
        return 0

    if args.stages:
        if rank == 0:
            st = stages_section(amber_b200, synth, local)
            print(json.dumps(dict(impl="amber_b200", n_gpus=1, data="synthetic", config={"workload": st["workload"]},
                                  **{k: v for k, v in st.items() if k != "workload"})))
        return 0

    if args.gridding:
        if rank == 0:
            gr = gridding_section(amber_b200, synth, local)
            print(json.dumps(dict(impl="amber_b200", n_gpus=1, dtype="f64 sums of f32 records", data="synthetic",
                                  config={"workload": gr["workload"]}, **{k: v for k, v in gr.items() if k != "workload"})))
        return 0

    if args.maps:
        if rank == 0:
            m = maps_section(amber_b200, synth, local)
            print(json.dumps(dict(impl="amber_b200", n_gpus=1, dtype="f64", data="synthetic",
                                  config={"workload": m["workload"]}, **{k: v for k, v in m.items() if k != "workload"})))
        return 0

    real = synth.config2(seed=1 + rank)
    stream = torch.cuda.current_stream(dev)
    est = amber_b200.Estimator(device=local, precision="mixed", stream=stream.cuda_stream, tile_n=args.tile_n)
    est.load_grid(real.gv, real.counts, real.du, real.flag_key)
    est.set_rings(real.ulow, real.uhigh)
    est.set_channels(real.nc10, real.uf_chans)
    rdata = est.calcr()
    tri = rdata[:, :3].astype(np.int32)
    if args.tri_subset:
        tri = tri[[int(t) for t in args.tri_subset.split(",")]]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # 256 MB > 126 MB L2

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def sum_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        return float(t.item())

    # ---- device-resident throughput (value) ----
    for _ in range(args.warmup):
        flush.zero_()
        est.run(tri, want_v2=True)
    clocks = Clocks(local)
    clocks.start()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    products = 0.0
    contract_ms = maps_ms = reduce_ms = 0.0
    launches = contracts = 0
    step_ms = []
    for _ in range(args.steps):
        flush.zero_()
        est.run(tri, want_v2=True)
        p, ms = est.last_run_stats()
        a, b, c, n, m = est.last_run_breakdown()
        products += p
        step_ms.append(ms)
        maps_ms += a
        contract_ms += b
        reduce_ms += c
        launches += n + 1  # + the L2 flush kernel
        contracts += m
    e1.record(stream)
    barrier()
    clk = clocks.stop()
    total_ms = max_over_ranks(e0.elapsed_time(e1))
    all_products = sum_over_ranks(products)
    value = all_products / (total_ms * 1e-3)

    # ---- end to end through the C ABI from pinned host buffers (e2e) ----
    ri_host = torch.from_numpy(np.ascontiguousarray(real.gv).view(np.float64)).pin_memory()
    nt_host = torch.from_numpy(np.ascontiguousarray(real.counts)).pin_memory()
    nclen = real.nclen
    out_bl = torch.empty((len(tri), nclen, nclen), dtype=torch.float64).pin_memory()
    out_nt = torch.empty((len(tri), nclen, nclen), dtype=torch.float64).pin_memory()
    h2d = ri_host.numel() * 8 + nt_host.numel() * 8
    d2h = out_bl.numel() * 8 + out_nt.numel() * 8 + rdata.size * 8

    def e2e_step():
        est.load_grid_raw(ri_host.data_ptr(), nt_host.data_ptr(), real.nn, real.nc, real.du, real.flag_key)
        est.set_rings(real.ulow, real.uhigh)
        est.set_channels(real.nc10, real.uf_chans)
        rd = est.calcr()
        est.run(rd[:, :3].astype(np.int32) if not args.tri_subset else tri, want_v2=True)
        est.fetch_into(out_bl.data_ptr(), out_nt.data_ptr())
        return est.last_run_stats()[0]

    for _ in range(max(1, args.warmup - 1)):
        e2e_step()
    barrier()
    lat = []
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    e2e_products = 0.0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        e2e_products += e2e_step()
        lat.append(time.perf_counter() - t0)
    f1.record(stream)
    barrier()
    e2e_ms = max_over_ranks(f0.elapsed_time(f1))
    e2e_value = sum_over_ranks(e2e_products) / (e2e_ms * 1e-3)

    # ---- plain FP64 GPU path and the mixed path's error on a bounded sample ----
    fp64 = None
    if rank == 0 and not args.no_fp64:
        sample = tri[-3:]  # the three triangles with the largest map (r1 = 15, Ng1 = 740)
        est.run(sample, want_v2=True)
        mixed_bl, _, mixed_nt = est.fetch(want_v2=True)
        p_mixed, ms_mixed = est.last_run_stats()
        res = {}
        for prec in ("fp64", "fp64_abs"):
            with amber_b200.Estimator(device=local, precision=prec, stream=stream.cuda_stream) as e64:
                e64.load_grid(real.gv, real.counts, real.du, real.flag_key)
                e64.set_rings(real.ulow, real.uhigh)
                e64.set_channels(real.nc10, real.uf_chans)
                e64.run(sample, want_v2=True)
                res[prec] = (e64.fetch(want_v2=True), e64.last_run_stats())
        (bl64, _, nt64), (p64, ms64) = res["fp64"]
        (ab_bl, _, ab_nt), _ = res["fp64_abs"]
        err = max(float((np.abs(mixed_bl - bl64) / (ab_bl + 1e-300)).max()),
                  float((np.abs(mixed_nt - nt64) / (ab_nt + 1e-300)).max()))
        fp64 = {"value": p64 / (ms64 * 1e-3), "unit": UNIT,
                "sample": "the 3 triangles with r1=15 (Ng1=740), v2, same GPU",
                "mixed_same_sample": p_mixed / (ms_mixed * 1e-3), "speedup": (p64 / ms64) / (p_mixed / ms_mixed),
                "max_rel_err_vs_fp64": err, "err_scale": "sum of |products| per lag cell"}
        fp64["speedup"] = fp64["mixed_same_sample"] / fp64["value"]

    # ---- CPU baseline: the reference's own loop on the host cores ----
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        try:
            import oracle
            if oracle.ref_available():
                st, rp = cpu_reference_sample(real)
                cpu = {"value": st["products"] / st["accum_s"], "unit": UNIT, "cores": st["threads"],
                       "kind": "reference",
                       "sample": f"one triangle (rp={rp}, Ng1=740) of this workload, v1 accumulation loop of the "
                                 f"reference's own sources (oracle/_ref/ref_amber_fast), {st['accum_s']:.1f} s"}
        except Exception as ex:  # reported, not fatal
            cpu = {"value": None, "unit": UNIT, "error": str(ex)[:200]}

    pk, pk_kind = peaks()
    # algorithmic flops of one contraction launch = 2 per product; products per launch = p/(launches)
    per_launch_products = products / max(contracts, 1)
    avg_launch_ms = contract_ms / max(contracts, 1)
    achieved = 2.0 * per_launch_products / (avg_launch_ms * 1e-3) / 1e12
    peak = pk.get("bf16_tflops_sustained", pk.get("bf16_tflops"))
    # the digit scheme runs 9 int8 MACs per lag-triple product (3 x 4 digits, classes i+j <= 3)
    int8_tops = 2.0 * 9 * per_launch_products / (avg_launch_ms * 1e-3) / 1e12
    roof = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
            "traffic": DRAM_BYTES_PER_PRODUCT * per_launch_products, "kernel": "contract_i8_kernel",
            "traffic_source": "ncu dram__bytes_read+write of one launch (profiles/"
                              "contract_i8_kernel_config2_one_triangle.txt), scaled by products per launch",
            "peak_kind": f"{pk_kind} bf16 dense, sustained (int8 MMA nominal rate is 2x this)",
            "int8_digit_mmas": {"macs_per_product": 9, "tops": int8_tops, "frac_of_2x_bf16_peak": int8_tops / (2 * peak)},
            "per_launch_products": per_launch_products, "avg_launch_ms": avg_launch_ms,
            "share_of_step": contract_ms / max(sum(step_ms), 1e-9),
            "phase_ms_per_step": {"maps": maps_ms / args.steps, "contract": contract_ms / args.steps,
                                  "lag_reduce": reduce_ms / args.steps}}
    lat_ms = sorted(1e3 * x for x in lat)
    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "int8 tensor-core digits, int32 accumulate, fp64 reduce",
           "data": "synthetic (seeded Gaussian field, Poisson sampling, per-rank seed)",
           "config": dict(WORKLOAD, parallelism=f"replicas x{world}", l2="256 MB flush between steps; working set "
                                                                          "(maps) > L2"),
           "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                   "p50_ms": float(np.percentile(lat_ms, 50)), "p99_ms": float(np.percentile(lat_ms, 99))},
           "fp64_plain": fp64, "roofline": roof, "cpu_baseline": cpu, "clocks": clk,
           "gpu_launches": int(launches), "products_per_step": products / args.steps}
    out["autotuner"] = {f"nclen<={k}": {"tile_n": v[0], "trial_ms_32": round(v[1], 3), "trial_ms_64": round(v[2], 3)}
                        for k, v in est.tile_choices().items()}
    est.close()
    # batched ensemble and serving stream: 1 GPU only (the scaling runs measure the step above)
    if rank == 0 and world == 1 and not args.tri_subset:
        for key, flag, fn in (("ensemble", args.no_ensemble, ensemble_section),
                              ("serving", args.no_serving, serving_section)):
            if flag:
                continue
            try:
                out[key] = fn(amber_b200, synth, local)
            except Exception as ex:  # reported, not fatal
                out[key] = {"error": str(ex)[:300]}
    if rank == 0:
        print(json.dumps(out))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
