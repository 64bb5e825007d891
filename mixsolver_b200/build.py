"""Build libmixgpu.so in-tree with nvcc for sm_100a.

    python -m mixsolver_b200.build

The FP64 parity kernels are compiled with -fmad=false: the reference's gfortran
-O2 x86-64 build issues no fused multiply-add, and the element-wise kernels
reproduce its arithmetic exactly.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libmixgpu.so")
BUILD = os.path.join(HERE, "_build")

SOURCES = ["case.cu", "assembly.cu", "krylov.cu", "krylov_mixed.cu", "krylov_poly64.cu", "batch.cu", "standalone.cu", "noalloc.cu", "device_topo.cu",
           "mesh_host.cpp", "cas_reader.cpp"]
# the mixed-precision form needs no bit-parity and may contract into FMA
FMA_OK = {"krylov_mixed.cu", "krylov_poly64.cu"}
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-ffp-contract=off", "--expt-relaxed-constexpr"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.exists(c) or c == "nvcc"):
            return c
    return "nvcc"


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    hdrs = [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".cuh", ".h"))]
    hdrs.append(os.path.join(os.path.dirname(HERE), "include", "mixgpu.h"))
    newest_hdr = max(os.path.getmtime(h) for h in hdrs)
    objs, cmds = [], []
    for s in srcs:
        o = os.path.join(BUILD, os.path.basename(s) + ".o")
        objs.append(o)
        if not force and os.path.exists(o) and os.path.getmtime(o) > max(os.path.getmtime(s), newest_hdr):
            continue
        flags = [("-fmad=true" if f == "-fmad=false" and os.path.basename(s) in FMA_OK else f) for f in NVCC_FLAGS]
        cmds.append([nvcc()] + ARCH + flags + ["-c", s, "-o", o])
    # the translation units compile side by side (the mixed-precision kernels
    # alone take about a minute)
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as pool:
        for cmd in cmds:
            if verbose:
                print(" ".join(cmd))
        list(pool.map(subprocess.check_call, cmds))
    if force or not os.path.exists(OUT) or os.path.getmtime(OUT) < max(os.path.getmtime(o) for o in objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", OUT] + objs + ["-cudart", "static", "-lpthread"]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
    return OUT


if __name__ == "__main__":
    print(build(verbose=True, force="--force" in sys.argv))
