"""Measured throughput of the pipes that bound the hot path's kernels.

    python -m superlite_b200.peaks [--out profiles/measured_pipe_peaks.json]

Runs slg_pipe_throughput (csrc/peaks.cu) for FP64 FMA, FP64 exp, FP32 FMA
and 32-bit integer multiply-add on cuda:0 while sampling the SM clock with
nvidia-smi, and writes one JSON record.  The FP32 FMA rate, divided by the 64
flops of a warp-wide FMA, is the sustained warp-instruction issue rate (one
instruction per cycle per scheduler); the bench normalises the particle
loop's instruction rate by it, and the opacity kernels' line-shell terms per
second by the FP64 exp rate.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import tempfile
import time

from . import capi

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
DEFAULT_OUT = os.path.join(ROOT, "profiles", "measured_pipe_peaks.json")

PIPES = (  # (which, name, iters per thread, unit)
    (0, "fp64_fma_flops", 400_000, "flop/s"),
    (1, "fp64_exp_per_s", 20_000, "evaluations/s"),
    (2, "fp32_fma_flops", 400_000, "flop/s"),
    (3, "int32_imad_per_s", 400_000, "operations/s"),
)


def _clock_sampler(device):
    f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
    try:
        p = subprocess.Popen(["nvidia-smi", f"--id={device}", "--query-gpu=clocks.sm,clocks.max.sm",
                              "--format=csv,noheader,nounits", "-lms", "100"], stdout=f, stderr=subprocess.DEVNULL)
    except OSError:
        p = None
    return p, f


def _clock_summary(p, f):
    if p is None:
        return {"sm_mhz_median": None, "sm_max_mhz": None, "samples": 0}
    p.terminate()
    try:
        p.wait(5)
    except Exception:
        p.kill()
    f.flush()
    rows = []
    with open(f.name) as fh:
        for ln in fh:
            a = [x.strip() for x in ln.split(",")]
            if len(a) == 2 and a[0].isdigit() and a[1].isdigit():
                rows.append((float(a[0]), float(a[1])))
    os.unlink(f.name)
    if not rows:
        return {"sm_mhz_median": None, "sm_max_mhz": None, "samples": 0}
    return {"sm_mhz_median": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
            "samples": len(rows)}


def measure(device: int = 0, reps: int = 3) -> dict:
    lib = capi.load()
    out = {}
    p, f = _clock_sampler(device)
    time.sleep(0.3)
    for which, name, iters, unit in PIPES:
        best, best_ms = 0.0, 0.0
        for _ in range(reps):
            v, ms = C.c_double(0.0), C.c_float(0.0)
            rc = lib.slg_pipe_throughput(device, which, iters, C.byref(v), C.byref(ms))
            if rc != 0:
                raise capi.SlgError(rc, f"slg_pipe_throughput({which})")
            if v.value > best:
                best, best_ms = v.value, ms.value
        out[name] = {"value": best, "unit": unit, "ms": best_ms, "iters": iters}
    clocks = _clock_summary(p, f)
    out["warp_inst_issue_per_s"] = {"value": out["fp32_fma_flops"]["value"] / 64.0, "unit": "warp instructions/s",
                                    "basis": "FP32 FMA flop/s / 64 (2 flops x 32 lanes per warp instruction)"}
    out["clocks"] = clocks
    out["how"] = ("slg_pipe_throughput: one launch of 8 x 256-thread blocks per SM, independent chains per "
                  "thread, CUDA events, best of %d after a warm-up launch" % reps)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=DEFAULT_OUT)
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args()
    import torch
    name = torch.cuda.get_device_name(a.device) if torch.cuda.is_available() else None
    r = measure(a.device)
    r["gpu_name"] = name
    with open(a.out, "w") as fh:
        json.dump(r, fh, indent=1)
    print(json.dumps(r))


if __name__ == "__main__":
    main()
