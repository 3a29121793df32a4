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
