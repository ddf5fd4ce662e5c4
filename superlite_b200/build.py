"""Builds libslg.so (the sm_100a CUDA library behind include/slg.h) in-tree.

    python -m superlite_b200.build        # or superlite_b200.build.build()

nvcc cross-compiles for sm_100a without a GPU.  The FP64 translation units are
compiled with -fmad=false so that products and sums round separately, as in
the reference's Fortran; the mixed-precision unit keeps FMA contraction.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT, "libslg.so")

FP64_SOURCES = ["opacity.cu", "grid.cu", "transport.cu", "source.cu", "capi.cu", "noalloc.cu", "eos.cu",
                "adjoint.cu", "peaks.cu"]
MIXED_SOURCES = ["transport_mixed.cu"]
HEADERS = ["slg_device.cuh", "slg_internal.h", "transport_impl.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _host_cxx():
    for c in ("/usr/bin/g++", shutil.which("g++")):
        if c and os.path.exists(c):
            return c
    return None


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OUT, exist_ok=True)
    nvcc = _nvcc()
    cxx = _host_cxx()
    inc = ["-I", os.path.join(ROOT, "include"), "-I", CSRC]
    common = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC"]
    if cxx:
        common += ["-ccbin", cxx]
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "slg.h")]
    objs = []
    for src, fmad in [(s, False) for s in FP64_SOURCES] + [(s, True) for s in MIXED_SOURCES]:
        path = os.path.join(CSRC, src)
        obj = os.path.join(OUT, src.replace(".cu", ".o"))
        if force or _stale(obj, [path] + hdrs):
            cmd = [nvcc, "-c", path, "-o", obj] + common + inc + [f"--fmad={'true' if fmad else 'false'}"]
            if verbose:
                print(" ".join(cmd))
            subprocess.run(cmd, check=True)
        objs.append(obj)
    if force or _stale(LIB, objs):
        cmd = [nvcc, "-shared", "-o", LIB] + objs + ARCH + ["-lcudart"]
        if cxx:
            cmd += ["-ccbin", cxx]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
