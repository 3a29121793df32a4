"""Build libamber_cuda.so in-tree for sm_100a (nvcc, no JIT cache).

``python -m amber_b200.build`` or ``amber_b200.build.build()``; also builds
the C drivers ``amber_gpu`` (estimator stage), ``vcg_gpu`` (gridding stage)
and ``maps_gpu`` (the MAPS two-point function) next to the library.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libamber_cuda.so")
DRIVER = os.path.join(HERE, "amber_gpu")
VCG_DRIVER = os.path.join(HERE, "vcg_gpu")
MAPS_DRIVER = os.path.join(HERE, "maps_gpu")
SOURCES = ["api.cu", "maps.cu", "lagspace.cu", "contract64.cu", "contract_tc.cu", "contract_i8.cu", "grid.cu", "noalloc.cu", "engine.cu", "cylbs.cu", "cldnu.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    deps = srcs + [os.path.join(CSRC, "common.cuh"), os.path.join(ROOT, "include", "amber_cuda.h")]
    deps += [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    if force or _stale(LIB, deps):
        objdir = os.path.join(ROOT, "_build", "obj")
        os.makedirs(objdir, exist_ok=True)
        objs = []
        for s in srcs:
            o = os.path.join(objdir, os.path.basename(s) + ".o")
            cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-fvisibility=hidden",
                   "-I", os.path.join(ROOT, "include"), "-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
            objs.append(o)
        cmd = [nvcc(), *ARCH, "-shared", "-o", LIB, *objs, "-lcuda"]
        subprocess.run(cmd, check=True)
    for exe, name in ((DRIVER, "amber_gpu.c"), (VCG_DRIVER, "vcg_gpu.c"), (MAPS_DRIVER, "maps_gpu.c")):
        drv_src = os.path.join(HERE, "driver", name)
        if os.path.exists(drv_src) and (force or _stale(exe, [drv_src, LIB, os.path.join(ROOT, "include", "amber_cuda.h")])):
            cc = shutil.which("gcc") or "cc"
            subprocess.run([cc, "-O2", "-std=gnu11", "-Wall", "-I", os.path.join(ROOT, "include"), drv_src, "-o", exe,
                            "-L", HERE, "-lamber_cuda", "-Wl,-rpath,$ORIGIN", "-lm"], check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
