"""The allocation-free entry point, amber_cuda_contract_fp64_noalloc.

It serves callers that own every device allocation themselves (a process
that reserves its HBM budget up front, or an application whose own caching
allocator must stay the only one) and so cannot let the library allocate.
Here the test plays that caller: it owns the device buffers (through torch),
calls the entry point through the C ABI twice in a row, and checks each
result against the context-based entry point (amber_cuda_triangles in FP64)
within the FP64 path's tolerance, 1e-10 of Σ|products| per lag cell.
This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

import oracle
from amber_b200 import synth

pytestmark = pytest.mark.gpu
TOL64 = 1e-10


def _entry():
    import amber_b200
    from amber_b200 import build
    build.build()
    L = amber_b200.load_library()
    f = L.amber_cuda_contract_fp64_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_long, ctypes.c_long, ctypes.c_long,
                  ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_char_p,
                  ctypes.c_size_t]
    return f


def _case(seed, flagged):
    real = synth.tiny(48, 12, seed=seed, nbins=5, hi=22.0, nc10=5, flagged=flagged)
    gvn, _ = oracle.normalize(real.gv, real.counts)
    rdata = oracle.calcr(oracle.normalize(real.gv, real.counts)[1], real.ulow, real.uhigh)
    r1, r2, r3 = (int(v) for v in rdata[-1, :3])  # the triangle with the largest map
    ng = oracle.ng1(real.uhigh[r1], real.du)
    maps = [oracle.ring_maps(gvn, real.ulow[r], real.uhigh[r], ng) for r in (r1, r2, r3)]
    w = np.zeros(real.nc, dtype=np.int32)
    for c in (real.uf_chans if real.flag_key == 1 else range(real.nc)):
        w[c] += 1
    return real, (r1, r2, r3), maps, w


def _via_context(real, tri):
    import amber_b200
    with amber_b200.Estimator(precision="fp64") as est:
        est.load_grid(real.gv, real.counts, real.du, real.flag_key)
        est.set_rings(real.ulow, real.uhigh)
        est.set_channels(real.nc10, real.uf_chans if real.flag_key == 1 else None)
        bl, _, _ = est.triangles(np.array([tri], dtype=np.int32))
    return bl[0]


def test_noalloc_matches_context_entry_point_twice():
    import torch
    f = _entry()
    real, tri, maps, w = _case(41, [0, 7])
    ref = _via_context(real, tri)
    scale = oracle.triangle_absscale(*maps, real.nc10, real.uf_chans) + 1e-300
    nc, k = maps[0].shape
    kp = (k + 63) // 64 * 64
    dev = torch.device("cuda", 0)
    d_maps = []
    for m in maps:
        t = torch.zeros((nc, kp), dtype=torch.float64, device=dev)
        t[:, :k] = torch.from_numpy(m)
        d_maps.append(t)
    nclen = 2 * real.nc10 + 1
    err = ctypes.create_string_buffer(256)
    for call in range(2):  # the scratch keeps the last call's contents between calls
        lag = torch.full((nclen, nclen), float("nan"), dtype=torch.float64, device=dev)
        rc = f(d_maps[0].data_ptr(), d_maps[1].data_ptr(), d_maps[2].data_ptr(), nc, k, kp, real.nc10,
               w.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), lag.data_ptr(),
               torch.cuda.current_stream(dev).cuda_stream, err, len(err))
        assert rc == 0, err.value
        torch.cuda.synchronize(dev)
        got = lag.cpu().numpy()
        e = np.abs(got - ref) / scale
        assert e.max() <= TOL64, (call, e.max())


def _random_case(nc, nc10, k, seed, flagged=()):
    """Seeded FP64 maps of an nc-channel triangle with k pixels (no pipeline needed: the entry point
    contracts whatever maps it is given) and the oracle's lag array and Σ|products| for them."""
    rng = np.random.default_rng(seed)
    maps = [rng.standard_normal((nc, k)) for _ in range(3)]
    uf = np.setdiff1d(np.arange(nc), np.asarray(flagged, dtype=np.int64)).astype(np.int32)
    w = np.zeros(nc, dtype=np.int32)
    w[uf] = 1
    bl, _, _, _ = oracle.triangle(*maps, nc10, uf if len(flagged) else None)
    scale = oracle.triangle_absscale(*maps, nc10, uf if len(flagged) else None) + 1e-300
    return maps, w, bl, scale


def _call_noalloc(f, maps, w, nc10, dev):
    import torch
    nc, k = maps[0].shape
    kp = (k + 63) // 64 * 64
    d_maps = []
    for m in maps:
        t = torch.zeros((nc, kp), dtype=torch.float64, device=dev)
        t[:, :k] = torch.from_numpy(m)
        d_maps.append(t)
    nclen = 2 * nc10 + 1
    lag = torch.full((nclen, nclen), float("nan"), dtype=torch.float64, device=dev)
    err = ctypes.create_string_buffer(256)
    torch.cuda.synchronize(dev)
    free0 = torch.cuda.mem_get_info(dev)[0]
    rc = f(d_maps[0].data_ptr(), d_maps[1].data_ptr(), d_maps[2].data_ptr(), nc, k, kp, nc10,
           w.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), lag.data_ptr(), torch.cuda.current_stream(dev).cuda_stream,
           err, len(err))
    assert rc == 0, err.value
    torch.cuda.synchronize(dev)
    free1 = torch.cuda.mem_get_info(dev)[0]
    return lag.cpu().numpy(), free0, free1


@pytest.mark.parametrize("nc,nc10,k,seed,flagged", [
    # nclen = 301: eleven anchors' partial tiles fill the scratch, so 160 anchors run in 15
    # batches and every batch after the first adds its sum to the lag array
    (160, 150, 96, 3, (0, 5, 77)),
    # few anchors and 8192 pixels: the pixel range is split 8 ways within one batch
    (12, 5, 8192, 4, (2,)),
])
def test_noalloc_batches_and_pixel_split_vs_oracle(nc, nc10, k, seed, flagged):
    """The batch accumulation and the pixel split, each checked against the oracle's FP64 lag array
    on two calls in a row; the device's free memory is the same before and after each call (the
    calls after the first: the first may load the library's device code, which maps the array)."""
    import torch
    f = _entry()
    dev = torch.device("cuda", 0)
    maps, w, want, scale = _random_case(nc, nc10, k, seed, flagged)
    frees = []
    for call in range(3):
        got, free0, free1 = _call_noalloc(f, maps, w, nc10, dev)
        e = np.abs(got - want) / scale
        assert e.max() <= TOL64, (call, e.max())
        if call:
            frees.append((free0, free1))
    for free0, free1 in frees:
        assert free0 == free1, "device memory was allocated during the call"


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    f = _entry()
    dev = torch.device("cuda", 0)
    t = torch.zeros(64, dtype=torch.float64, device=dev)
    w = np.ones(5000, dtype=np.int32)
    err = ctypes.create_string_buffer(256)
    p = t.data_ptr()
    rc = f(p, p, p, 5000, 8, 8, 3, w.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), p, None, err, len(err))
    assert rc == -1 and b"nc outside" in err.value  # more channels than the scratch tables hold
    w = np.ones(1100, dtype=np.int32)
    rc = f(p, p, p, 1100, 8, 8, 600, w.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), p, None, err, len(err))
    assert rc == -1 and b"too large" in err.value  # nclen² beyond the partial-tile scratch


def test_noalloc_refuses_a_capturing_stream():
    """Each call uploads its channel tables from host memory when it is made; a stream that is being
    captured would record that copy for later instead, so the call refuses it (and leaves the capture
    untouched)."""
    import torch
    f = _entry()
    dev = torch.device("cuda", 0)
    t = torch.zeros(64, dtype=torch.float64, device=dev)
    w = np.ones(4, dtype=np.int32)
    err = ctypes.create_string_buffer(256)
    p = t.data_ptr()
    s = torch.cuda.Stream(dev)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(s):
        g.capture_begin()
        rc = f(p, p, p, 4, 8, 8, 1, w.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), p, s.cuda_stream, err, len(err))
        t.add_(1.0)  # the capture is still valid after the refusal
        g.capture_end()
    assert rc == -1 and b"captured" in err.value
    g.replay()
    torch.cuda.synchronize(dev)
    assert float(t[0]) == 1.0
