"""Benchmark of the AMBER estimator hot path on B200.

Workload (the headline): the batched ensemble — 64 realisations of uneven size,
grid side drawn from {96, 128, 192, 256, 320}, 24-160 channels, random 10 %
channel flags, 12 log-spaced annular bins from 2 to 0.47·side cells, all lag
pairs |Δν| ≤ nc/2 − 1, v2 output (visibility sums bldnu and sampling-mask sums
numtri), seeds 100-163.  Every realisation goes through the whole estimator:
calCR, then for all closed triangles the ring maps and the triple-product lag
accumulation.  Inputs are seeded synthetic data of that shape (there is no
public dataset for this path).

One step = one batch of 8 realisations (realisations j, j+8, …, j+56 for batch
j, so every batch mixes grid sizes) through the request engine; the default
K = 8 steps time the whole ensemble exactly once after W = 3 warm-up batches.

Metric: lag-triple products per second, one product being one term
D_r1(x,p1)·D_r2(x,p2)·D_r3(x,p3) of the reference's loop (4_fbe/amber.c:261-263);
per triangle total_vcp·Ng1², counted for the D and the I (mask) sums.

* value — device time (CUDA events) of the steps with every cube already in HBM
  (amber_cuda_enqueue with inputs_on_device);
* e2e   — the same steps through the public API from host memory: each request's
  cube copied in, every lag array (bldnu, numdnu, numtri) copied back;
* fp64_plain — the plain FP64 GPU path over the whole ensemble, its contraction
  kernel's rate against the measured FP64 GEMM peak, and the mixed path's error
  against it on three realisations;
* roofline — the int8 contraction kernel, algorithmic flops (2 per product) over
  its CUDA-event time, against the measured bf16 dense peak;
* cpu_baseline — the reference's own OpenMP loop (oracle/_ref/ref_amber_fast,
  its sources built unchanged) on the host cores, one triangle of the ensemble;
* single_realisation — the 256², 128-channel, 16-bin realisation on the
  device-resident path;
* config4_sample — six triangles of the 512², 384-channel cube (all four with
  Ng1 = 1460), with the plain FP64 path and its error on one more.

`--impl reference` times that same reference build as the reference arm.
`--serving N`, `--config4`, `--config1`, `--stages`, `--maps`, `--gridding` run
the other measurements instead of the headline.
Multi-GPU: one process per GPU (torchrun); each rank runs its own ensemble
(seeds 100 + 64·rank onwards): weak scaling, no collective on the data path;
timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "lag-triple products/s vs plain FP64 on same GPU @<=1e-6 rel err; p50/p99 latency"
UNIT = "lag-triple products/s"
WORKLOAD = dict(workload="batched ensemble: 64 realisations, sides {96,128,192,256,320}, 24-160 channels, "
                         "10 % random channel flags, 12 log bins 2..0.47*side cells, nc10=nc/2-1, v2 (D and mask "
                         "sums), all closed triangles, seeds 100-163; step = 8 realisations",
                realisations=64, batch=8, bins=12, version=2)
SINGLE = "single realisation: 256^2 grid, 128 channels (4 of every 32 flagged), 16 log bins 2-120 cells, nc10=63, v2"


# DRAM bytes per lag-triple product of the int8 lag-space kernel (ls_i8_kernel), from one ncu capture
# of a full launch (profiles/ls_i8_kernel_config2_one_triangle.txt): every staged map slice is read
# once per unit, so traffic grows with the products of a launch.
DRAM_BYTES_PER_PRODUCT = (493.735e6 + 26.335e6) / 4.436392352e11
CPU_SAMPLE_REALISATION = 3  # side 256, 116 channels: its last (largest-ring) triangle is ~15 s of reference CPU


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
    wd = tempfile.mkdtemp(prefix="amber_ref_")
    try:
        nthreads = nthreads or os.cpu_count() or 1
        if rp_pick is None:
            # the last closed triangle of the build being timed (its own calCR: the float build's
            # list can be one shorter than the FP64 one), found by a run over no triangles: the
            # largest ring r1, the kind of triangle that dominates a realisation
            st0, _ = oracle.run_ref_amber(real, wd, version=version, fp64=False, fast=fast, rp_begin=0, rp_end=0,
                                          nthreads=nthreads)
            rp_pick = int(st0["rcount"]) - 1
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
    real = synth.from_spec(synth.config3_specs()[CPU_SAMPLE_REALISATION])
    rates, times = [], []
    st = None
    for i in range(args.warmup + args.steps):
        st, rp = cpu_reference_sample(real)
        rate = st["products"] / st["accum_s"]
        if i >= args.warmup:
            rates.append(rate)
            times.append(st["accum_s"])
    value = float(np.median(rates))
    sample = (f"ensemble realisation {CPU_SAMPLE_REALISATION} (side {real.nn}, {real.nc} channels), its last triangle "
              f"rp={rp} (total_vcp={st['total_vcp']}), v1 accumulation loop timed like amber.c:230,285; maps excluded")
    out = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * float(np.median(times)),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
           "config": WORKLOAD,
           "cpu_baseline": {"value": value, "unit": UNIT, "cores": st["threads"], "kind": "reference",
                            "sample": sample},
           "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))
    return 0


def ensemble_batches(n=64, b=8):
    """Batch j holds realisations j, j+b, j+2b, …: every batch mixes grid sizes."""
    return [list(range(j, n, b)) for j in range(b)]


def run_batch(eng, reals, idx, cubes=None):
    """Enqueue the realisations ``idx`` (device-resident when ``cubes`` is given), wait for all of
    them and read their results back; returns the results in ``idx`` order."""
    tickets = [eng.enqueue(reals[i], want_v2=True, device_cube=None if cubes is None else cubes[i]) for i in idx]
    return [eng.result(t, reals[i], want_v2=True) for t, i in zip(tickets, idx)]


def device_cubes(torch, reals, dev):
    """Each realisation's summed grid and counts as device tensors (the packed layout the engine reads)."""
    keep, ptrs = [], []
    for r in reals:
        ri = torch.from_numpy(np.ascontiguousarray(r.gv).view(np.float64)).to(dev)
        nt = torch.from_numpy(np.ascontiguousarray(r.counts, dtype=np.float64)).to(dev)
        keep.append((ri, nt))
        ptrs.append((ri.data_ptr(), nt.data_ptr()))
    return keep, ptrs


def fp64_peak(torch, dev, n=8192, reps=5):
    """Measured FP64 dense rate of the GPU: a float64 n³ matmul, best of ``reps`` (TFLOP/s)."""
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    torch.matmul(a, b)
    best = 0.0
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize(dev)
        best = max(best, 2.0 * n ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    del a, b
    return best


def fp64_section(amber_b200, torch, reals, cubes, dev, mixed_sub):
    """The plain FP64 path over the whole ensemble (same engine, device-resident cubes), its
    contraction kernel's rate against the measured FP64 GEMM peak, and the mixed path's error
    against it on the realisations ``mixed_sub`` (a dict index -> mixed result)."""
    peak = fp64_peak(torch, dev)
    with amber_b200.Estimator(device=dev, precision="fp64") as est:
        eng = amber_b200.Engine(est)
        run_batch(eng, reals, [min(range(len(reals)), key=lambda i: reals[i].nn * reals[i].nc)], cubes)  # warm-up
        s0 = eng.stats()
        t0 = time.perf_counter()
        res = run_batch(eng, reals, list(range(len(reals))), cubes)
        wall = time.perf_counter() - t0
        s1 = eng.stats()
    prod = s1["products"] - s0["products"]
    kms = s1["contract_kernel_ms"] - s0["contract_kernel_ms"]
    achieved = 2.0 * prod / (kms * 1e-3) / 1e12 if kms > 0 else None
    err = 0.0
    with amber_b200.Estimator(device=dev, precision="fp64_abs") as est:
        eng = amber_b200.Engine(est)
        for i, m in mixed_sub.items():
            a = run_batch(eng, reals, [i], cubes)[0]
            f = res[i]
            err = max(err, float((np.abs(m[1] - f[1]) / (a[1] + 1e-300)).max()),
                      float((np.abs(m[3] - f[3]) / (a[3] + 1e-300)).max()))
            assert np.array_equal(m[2], f[2])  # counts exact
    return {"value": prod / wall, "unit": UNIT, "products": prod, "wall_s": wall,
            "sample": "the whole ensemble (64 realisations), same engine, device-resident cubes",
            "kernel": {"name": "ls_fp64_kernel", "achieved_tflops": achieved, "peak_tflops": peak,
                       "frac": None if achieved is None else achieved / peak,
                       "peak_kind": "measured here: torch float64 8192^3 matmul, best of 5",
                       "flops": "2 per lag-triple product (useful products only; lag-window padding excluded)"},
            "max_rel_err_vs_fp64": err, "err_scale": "sum of |products| per lag cell",
            "err_sample": sorted(mixed_sub)}


def serving_section(amber_b200, synth, dev, n=200, rate=0.3):
    """Serving stream: ``n`` requests of the config-5 size distribution (sides {64,128,256,384},
    16-256 channels, 6-20 bins, own seed and flags) arriving as a Poisson process at ``rate``
    req/s (the stream's 50 req/s inter-arrival times rescaled), enqueued at their arrival times;
    latency = arrival to result ready.  The plain FP64 path one request at a time runs on the ten
    smallest requests of the same sample."""
    reqs = synth.config5_requests()[:n]
    t_gen = time.perf_counter()
    reals = [synth.from_spec(q) for q in reqs]
    t_gen = time.perf_counter() - t_gen
    scale = 50.0 / rate
    with amber_b200.Estimator(device=dev, precision="mixed") as est:
        eng = amber_b200.Engine(est)
        run_batch(eng, [synth.from_spec(dict(reqs[0], nn=64, nc=32, nc10=15, ring_hi=30.0))], [0])  # warm-up
        s0 = eng.stats()
        t0 = time.perf_counter()
        tickets = []
        for q, r in zip(reqs, reals):
            delay = scale * (q["arrival"] - reqs[0]["arrival"]) - (time.perf_counter() - t0)
            if delay > 0:
                time.sleep(delay)
            tickets.append(eng.enqueue(r, want_v2=True))
        lat = [eng.result(t, r, want_v2=True)[4] for t, r in zip(tickets, reals)]
        wall = time.perf_counter() - t0
        s1 = eng.stats()
    prod = s1["products"] - s0["products"]
    small = sorted(range(n), key=lambda i: reqs[i]["nn"] ** 2 * reqs[i]["nc"] ** 3 * reqs[i]["nbins"])[:10]
    f_prod, f_wall, f_lat = 0.0, 0.0, []
    with amber_b200.Estimator(device=dev, precision="fp64") as e64:
        amber_b200.estimate(reals[small[0]], precision="fp64", version=2, est=e64)  # warm-up
        for i in small:
            t = time.perf_counter()
            amber_b200.estimate(reals[i], precision="fp64", version=2, est=e64)
            f_lat.append(1e3 * (time.perf_counter() - t))
            f_prod += e64.last_run_stats()[0]
            f_wall += time.perf_counter() - t
    return {"workload": f"serving: {n} requests of the config-5 size distribution, Poisson arrivals at {rate} req/s",
            "requests": n, "rate_req_s": rate, "value": prod / wall, "unit": UNIT, "products": prod, "wall_s": wall,
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mixed_latency_ms_of_fp64_sample": [round(lat[i], 1) for i in small],
            "engine": {k: s1[k] - s0[k] if k in ("rounds", "contraction_launches") else s1[k]
                       for k in ("rounds", "contraction_launches", "max_active", "peak_bytes")},
            "fp64_one_at_a_time": {"requests": small, "value": f_prod / f_wall, "latency_ms": [round(x, 1) for x in f_lat],
                                   "p50_ms": float(np.percentile(f_lat, 50))},
            "generation_s": t_gen}


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


def single_section(amber_b200, synth, dev, stream, reps=2):
    """The single-realisation case on the device-resident path: all 218 closed triangles of the
    256² realisation, one warm-up run and ``reps`` timed runs (CUDA events)."""
    import torch
    real = synth.config2(seed=1)
    with amber_b200.Estimator(device=dev, precision="mixed", stream=stream.cuda_stream) as est:
        est.load_grid(real.gv, real.counts, real.du, real.flag_key)
        est.set_rings(real.ulow, real.uhigh)
        est.set_channels(real.nc10, real.uf_chans)
        tri = est.calcr()[:, :3].astype(np.int32)
        est.run(tri, want_v2=True)
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        prod, cms = 0.0, 0.0
        for _ in range(reps):
            est.run(tri, want_v2=True)
            prod += est.last_run_stats()[0]
            cms += est.last_run_breakdown()[1]
        e1.record(stream)
        torch.cuda.synchronize(dev)
        ms = e0.elapsed_time(e1)
    return {"workload": SINGLE, "value": prod / (ms * 1e-3), "unit": UNIT, "ms_per_run": ms / reps,
            "contract_ms_per_run": cms / reps, "products_per_run": prod / reps}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=8, help="timed batches of 8 realisations (8 = the whole ensemble)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="amber_b200", choices=["amber_b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-single", action="store_true", help="skip the single-realisation section")
    ap.add_argument("--no-config4", action="store_true", help="skip the large-cube sample section")
    ap.add_argument("--serving", type=int, default=0, metavar="N",
                    help="run N requests of the serving stream instead of the headline")
    ap.add_argument("--rate", type=float, default=0.3,
                    help="Poisson arrival rate of --serving (req/s); one B200 serves ~0.41/s of the stream's sizes")
    ap.add_argument("--config1", action="store_true",
                    help="measure the reference's whole CPU-runnable case (config 1) beside the reference's own run")
    ap.add_argument("--stages", action="store_true",
                    help="time the stages beside the contraction (cylindrical bispectra, gridding with collapse)")
    ap.add_argument("--maps", action="store_true",
                    help="measure the MAPS two-point function (amber_cuda_cl_dnu) instead of the headline")
    ap.add_argument("--gridding", action="store_true",
                    help="time the gridding stage alone (100k records x 128 channels onto 256^2)")
    ap.add_argument("--config4", action="store_true",
                    help="measure a fixed sample of the large cube (512^2, 384 channels) instead of the headline")
    ap.add_argument("--shard", action="store_true",
                    help="strong scaling: the single-realisation case's triangles split across the ranks "
                         "(amber_cuda_shard_plan), instead of the headline")
    ap.add_argument("--profile-triangle", type=int, default=-1, metavar="RP",
                    help="profiling runs: triangle RP of the single-realisation case, twice, v1, on --precision")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
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
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    build.build()

    if args.profile_triangle >= 0:
        real = synth.config2(seed=1)
        with amber_b200.Estimator(device=local, precision=args.precision) as est:
            est.load_grid(real.gv, real.counts, real.du, real.flag_key)
            est.set_rings(real.ulow, real.uhigh)
            est.set_channels(real.nc10, real.uf_chans)
            tri = est.calcr()[[args.profile_triangle], :3].astype(np.int32)
            for _ in range(2):  # a profiler captures the second launch (-s 1)
                est.run(tri, want_v2=False)
            p, ms = est.last_run_stats()
        print(json.dumps({"profile_triangle": args.profile_triangle, "precision": args.precision,
                          "products": p, "ms": ms}))
        return 0

    modes = (("config4", lambda: config4_section(amber_b200, synth, local, args)),
             ("config1", lambda: config1_section(amber_b200, synth, local)),
             ("stages", lambda: stages_section(amber_b200, synth, local)),
             ("gridding", lambda: gridding_section(amber_b200, synth, local)),
             ("maps", lambda: maps_section(amber_b200, synth, local)),
             ("serving", lambda: serving_section(amber_b200, synth, local, n=args.serving, rate=args.rate)))
    for name, fn in modes:
        if getattr(args, name):
            if rank == 0:
                r = fn()
                print(json.dumps(dict(metric=METRIC, impl="amber_b200", n_gpus=1, data="synthetic",
                                      config={"workload": r["workload"]},
                                      **{k: v for k, v in r.items() if k != "workload"})))
            return 0

    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    def reduce(x, op):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=op)
        return float(t.item())

    if args.shard:
        from amber_b200 import shard
        real = synth.config2(seed=1)
        stream = torch.cuda.current_stream(dev)
        with amber_b200.Estimator(device=local, precision="mixed", stream=stream.cuda_stream) as est:
            est.load_grid(real.gv, real.counts, real.du, real.flag_key)
            est.set_rings(real.ulow, real.uhigh)
            est.set_channels(real.nc10, real.uf_chans)
            tri = est.calcr()[:, :3].astype(np.int32)
            mine = shard.plan_native(tri, est.ng1, world)[rank]
            sub = tri[mine]
            for _ in range(args.warmup):
                est.run(sub, want_v2=True)
            clocks = Clocks(local)
            clocks.start()
            barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            prod = 0.0
            for _ in range(args.steps):
                est.run(sub, want_v2=True)
                prod += est.last_run_stats()[0]
            e1.record(stream)
            barrier()
            clk = clocks.stop()
            ms = reduce(e0.elapsed_time(e1), dist.ReduceOp.MAX if world > 1 else None)
            total = reduce(prod, dist.ReduceOp.SUM if world > 1 else None)
            planned = {str(n): shard.planned_speedup(tri, est.ng1, n) for n in (1, 2, 4, 8)}
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": total / (ms * 1e-3), "unit": UNIT, "n_gpus": world,
                              "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
                              "higher_is_better": True, "scaling": "strong", "impl": "amber_b200",
                              "dtype": "int8 tensor-core digits, int32 accumulate, fp64 reduce", "data": "synthetic",
                              "config": {"workload": SINGLE, "parallelism": f"triangles sharded x{world}"},
                              "triangles_per_rank_0": len(mine), "planned_speedup": planned, "clocks": clk}))
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return 0

    # ---- this rank's ensemble, its cubes resident in HBM ----
    t_gen = time.perf_counter()
    specs = synth.config3_specs(seed0=100 + 64 * rank)
    reals = [synth.from_spec(sp) for sp in specs]
    t_gen = time.perf_counter() - t_gen
    keep, cubes = device_cubes(torch, reals, dev)
    batches = ensemble_batches(len(reals), 8)
    order = [batches[(args.warmup + k) % len(batches)] for k in range(args.steps)]
    stream = torch.cuda.current_stream(dev)
    est = amber_b200.Estimator(device=local, precision="mixed")
    eng = amber_b200.Engine(est)

    # ---- device-resident throughput (value) ----
    for k in range(args.warmup):
        run_batch(eng, reals, batches[k % len(batches)], cubes)
    clocks = Clocks(local)
    clocks.start()
    barrier()
    s0 = eng.stats()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    mixed = {}
    for idx in order:
        for i, r in zip(idx, run_batch(eng, reals, idx, cubes)):
            mixed[i] = r
    e1.record(stream)
    barrier()
    clk = clocks.stop()
    s1 = eng.stats()
    total_ms = reduce(e0.elapsed_time(e1), dist.ReduceOp.MAX if world > 1 else None)
    products = s1["products"] - s0["products"]
    all_products = reduce(products, dist.ReduceOp.SUM if world > 1 else None)
    value = all_products / (total_ms * 1e-3)
    kms = s1["contract_kernel_ms"] - s0["contract_kernel_ms"]
    launches = s1["contraction_launches"] - s0["contraction_launches"]
    gpu_launches = s1["kernel_launches"] - s0["kernel_launches"]

    # ---- end to end through the public API from host memory (e2e) ----
    run_batch(eng, reals, batches[0])  # warm-up of the host-input path
    barrier()
    h2d = d2h = 0
    path_diff, counts_equal = 0.0, True
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    q0 = eng.stats()
    f0.record(stream)
    lat = []
    for idx in order:
        t0 = time.perf_counter()
        res = run_batch(eng, reals, idx)
        lat.append(time.perf_counter() - t0)
        for i, r in zip(idx, res):
            h2d += reals[i].gv.nbytes + reals[i].counts.size * 8
            d2h += sum(a.nbytes for a in r[:4] if a is not None)
            # the host-input path computes what the device-resident path did (to FP64 rounding: the
            # engine may group the realisations into other launches)
            for a, b in ((r[1], mixed[i][1]), (r[3], mixed[i][3])):
                path_diff = max(path_diff, float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)))
            counts_equal = counts_equal and np.array_equal(r[2], mixed[i][2])
    f1.record(stream)
    barrier()
    q1 = eng.stats()
    e2e_ms = reduce(f0.elapsed_time(f1), dist.ReduceOp.MAX if world > 1 else None)
    e2e_value = reduce(q1["products"] - q0["products"], dist.ReduceOp.SUM if world > 1 else None) / (e2e_ms * 1e-3)
    est.close()

    pk, pk_kind = peaks()
    peak = pk.get("bf16_tflops_sustained", pk.get("bf16_tflops"))
    per_launch = products / max(launches, 1)
    avg_launch_ms = kms / max(launches, 1)
    achieved = 2.0 * per_launch / (avg_launch_ms * 1e-3) / 1e12 if avg_launch_ms > 0 else None
    # digit MMAs per product: 6 int8 MACs for the D sums (classes 0-2 of 3x3 digits), 9 for the mask
    # sums (classes 0-3 of 3x4 digits); a v2 run has as many products of each
    int8_tops = None if achieved is None else achieved * 7.5
    roof = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": None if achieved is None else achieved / peak,
            "traffic": None if DRAM_BYTES_PER_PRODUCT is None else DRAM_BYTES_PER_PRODUCT * per_launch,
            "kernel": "ls_i8_kernel", "launches": int(launches), "avg_launch_ms": avg_launch_ms,
            "per_launch_products": per_launch,
            "timing": "CUDA events around every contraction launch (engine phase events), summed",
            "traffic_source": "ncu dram__bytes_read+write of one launch (profiles/ls_i8_kernel_config2_one_triangle"
                              ".txt), scaled by products per launch",
            "peak_kind": f"{pk_kind} bf16 dense, sustained (int8 MMA nominal rate is 2x this)",
            "int8_digit_mmas": {"macs_per_product": 7.5, "tops": int8_tops,
                                "frac_of_2x_bf16_peak": None if int8_tops is None else int8_tops / (2 * peak)},
            "share_of_busy": kms / max(s1["busy_ms"] - s0["busy_ms"], 1e-9)}

    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "int8 tensor-core digits, int32 accumulate, fp64 reduce",
           "data": "synthetic (seeded Gaussian fields, Poisson sampling, random flags; per-rank seeds)",
           "config": dict(WORKLOAD, parallelism=f"replicas x{world}",
                          l2="inputs larger than L2: every step streams 8 realisations' maps (GBs) through HBM"),
           "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d / args.steps),
                   "d2h_bytes_per_step": int(d2h / args.steps),
                   "p50_ms": 1e3 * float(np.percentile(lat, 50)), "p99_ms": 1e3 * float(np.percentile(lat, 99)),
                   "path": "amber_cuda_enqueue / amber_cuda_result with host buffers (cube in, lag arrays out)",
                   "max_rel_diff_vs_device_resident": path_diff, "counts_equal": counts_equal},
           "roofline": roof, "clocks": clk, "gpu_launches": int(gpu_launches),
           "products_per_step": products / args.steps, "generation_s": t_gen,
           "engine": {k: s1[k] - s0[k] for k in ("rounds", "setup_ms", "maps_ms", "contract_ms", "finish_ms")}}

    if rank == 0 and world == 1 and not args.no_fp64:
        try:
            out["fp64_plain"] = fp64_section(amber_b200, torch, reals, cubes, local,
                                             {i: mixed[i] for i in (0, 16, 48) if i in mixed})
            out["fp64_plain"]["mixed_whole_ensemble"] = value
            out["fp64_plain"]["speedup"] = value / out["fp64_plain"]["value"]
        except Exception as ex:  # reported, not fatal
            out["fp64_plain"] = {"error": str(ex)[:300]}
    if rank == 0 and world == 1 and not args.no_single:
        try:
            out["single_realisation"] = single_section(amber_b200, synth, local, stream)
        except Exception as ex:
            out["single_realisation"] = {"error": str(ex)[:300]}
    if rank == 0 and world == 1 and not args.no_config4:
        try:
            out["config4_sample"] = config4_section(amber_b200, synth, local, args)
        except Exception as ex:
            out["config4_sample"] = {"error": str(ex)[:300]}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            import oracle
            if oracle.ref_available():
                st, rp = cpu_reference_sample(reals[CPU_SAMPLE_REALISATION])
                r = reals[CPU_SAMPLE_REALISATION]
                out["cpu_baseline"] = {
                    "value": st["products"] / st["accum_s"], "unit": UNIT, "cores": st["threads"], "kind": "reference",
                    "sample": f"ensemble realisation {CPU_SAMPLE_REALISATION} (side {r.nn}, {r.nc} channels), its last "
                              f"triangle rp={rp}, v1 accumulation loop of the reference's own sources "
                              f"(oracle/_ref/ref_amber_fast), {st['accum_s']:.1f} s"}
        except Exception as ex:  # reported, not fatal
            out["cpu_baseline"] = {"value": None, "unit": UNIT, "error": str(ex)[:200]}
    del keep
    if rank == 0:
        print(json.dumps(out))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
