"""Benchmark of SuperLite's per-timestep hot path on B200.

Default workload (--workload batched): one timestep of 128 independent
ejecta models (shells U{50..400}, particle budgets log-uniform in [1e5, 1e7],
snapshot times log-uniform in 1-30 d, 100 groups, analytic grey opacity)
in one context: sources, opacity, means, leakage, emission probabilities and
the source tally, then ONE persistent mixed-precision particle loop over all
models and per-model flux tallies, the timed steps captured in a CUDA graph.
Beside it: the plain FP64 particle loop called once per model, the same step
through the host-pointer C ABI (e2e), the opacity forward/adjoint of
the opacity case (256 shells x 2000 groups x 5e5 lines), and the oracle on the
host cores.

--workload timestep: one full IMC/DDMC timestep on the physical opacities of
256 shells x 2000 groups x 5e5 lines, 5e7 source particles
(--precision fp64|mixed).

metric: particle-steps/s = (IMC + DDMC events, particle_advance.f90:209,219)
        / device time of the step(s).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

N > 1 (torchrun): batched -- every rank runs its own batch of models (no
exchange); timestep -- every rank runs its own particles on the same grid and
the grid/flux tallies are summed with one NCCL all-reduce, as the reference's
reduce_gridtally / reduce_fluxtally do.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-steps/s"
# the reference's atomic data (Verner, Sutherland, data.ion, a subset of its
# line lists), parsed into a committed npz by tests/golden/make_atomic_data.py
ATOMIC_NPZ = os.path.join(ROOT, "tests", "golden", "atomic_data.npz")
T_DAYS = 10.0
SEED_CASE = 2
L_BOL = 1e42
# algorithmic bytes of one particle-step: event-based SoA traffic, 2 x (5 x 8 + 4 x 4 + 8) B
BYTES_PER_STEP = 128.0
# Per particle-loop variant (0..3: particle_advance_mixed_kernel<4..7>): warp
# instructions issued per particle-step and active lanes per warp instruction,
# from one ncu capture of each variant on the batched workload at 0.1x particle
# budgets (--transport-variant V; smsp__inst_executed.sum / particle-steps of
# the launch; smsp__thread_inst_executed.sum / smsp__inst_executed.sum):
# profiles/particle_advance_mixed_batched_128models_npart0.1.md
MIXED_WARP_INST_PER_STEP = {0: 50.2, 1: 52.6, 2: 55.1, 3: 59.6}
MIXED_LANES_PER_INST = {0: 9.99, 1: 9.61, 2: 9.33, 3: 9.03}
# The same for the FP64 particle_advance_kernel<5> (variant 1, the autotuner's
# choice) on the --workload timestep physics (256 shells x 2000 groups, every
# event a DDMC one), from one ncu capture at 2e5 particles
# (profiles/launches_timestep_256x2000_1e6.md): warp instructions, active
# lanes and DRAM bytes (read + write) per particle-step
FP64_TIMESTEP_INST_PER_STEP = 54.9
FP64_TIMESTEP_LANES_PER_INST = 13.3
FP64_TIMESTEP_DRAM_PER_STEP = 2.86e7 / 6.529e8


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed steps (default 1 for the batched workload, whose step runs about a minute; 3 otherwise)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--transport-variant", type=int, choices=(0, 1, 2, 3), default=None,
                    help="batched workload: run this particle-loop variant (no autotuner, no tuning steps)")
    ap.add_argument("--no-tune-steps", dest="tune_steps", action="store_false",
                    help="batched workload: keep the sample autotuner's variant instead of timing each variant on "
                         "one whole untimed step")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--npart", type=float, default=5e7)
    ap.add_argument("--ncell", type=int, default=256)
    ap.add_argument("--ng", type=int, default=2000)
    ap.add_argument("--nline", type=float, default=5e5)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-sample", type=int, default=0, help="particles in the CPU-baseline sample (0: auto)")
    ap.add_argument("--workload", default="batched", choices=["batched", "timestep", "opacity"],
                    help="batched: many models in one persistent launch, graph-captured steps; "
                         "timestep: one 256-shell model on physical opacities")
    ap.add_argument("--nmodel", type=int, default=128)
    ap.add_argument("--opacity-size", type=int, default=4, choices=[1, 4],
                    help="--workload opacity: 4 = 4096 shells x 10000 groups x 2e6 lines (default), "
                         "1 = 256 x 2000 x 5e5")
    ap.add_argument("--no-fp64", action="store_true", help="skip the plain FP64 per-model comparison")
    ap.add_argument("--no-opacity", action="store_true", help="skip the opacity forward/adjoint measurement")
    ap.add_argument("--no-cases", action="store_true",
                    help="skip the lines of the CPU-runnable case and of the full timestep beside the batched one")
    ap.add_argument("--npart-scale", type=float, default=1.0,
                    help="scale the models' particle budgets (small cases for profilers; default 1)")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def make_case(a):
    from superlite_b200 import workloads as W
    return W.opacity_case(ncell=a.ncell, ng=a.ng, nline=int(a.nline), seed=SEED_CASE, t_days=T_DAYS)


def config_dict(a, world):
    return {"workload": "IMC-DDMC timestep on physical LTE opacities (256 shells x 2000 groups x 5e5 lines)",
            "shells": a.ncell, "groups": a.ng, "lines": int(a.nline), "particles_per_gpu": int(a.npart),
            "snapshot_days": T_DAYS, "tauddmc": 5.0, "taulump": 10.0, "transport_precision": a.precision,
            "parallelism": f"particles{world}", "l2": "inputs larger than L2 (particle array 3.2 GB per GPU)"}


# ------------------------------------------------------------------ clocks
class Clocks:
    def __init__(self, index):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={index}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = []
        with open(self.f.name) as fh:
            for ln in fh:
                parts = [x.strip() for x in ln.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


# ------------------------------------------------------------------ our arm
def run_ours(a):
    import torch
    from superlite_b200 import HotPath, workloads as W
    from superlite_b200.timestep import DeviceTimestep
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    case = make_case(a)
    npart = int(a.npart)
    params = W.TransportParams()
    hot = HotPath(local)
    radtemp = case.gas.temp.copy()
    prec = 1 if a.precision == "mixed" else 0
    ts = DeviceTimestep(hot, case, params, npart=npart, precision=prec)
    emit, _ = hot.sourceenergy(radtemp, L_BOL)
    nvol, nnew = hot.sourcenumbers(emit, npart, npart)
    d_radtemp = ts.gas["temp"]
    ts.isv.fill_(1)
    stream = ts.stream
    seed0 = 1000 * (rank + 1)

    def one_step(k):
        hot.interior_source(d_radtemp, emit, nvol, ts.prt, ts.isv, seed=seed0 + 2 * k)
        ts.opacity()
        ts.coefficients()
        ts.transport(seed0 + 2 * k + 1)
        ts.fluxtally()

    # autotune the transport kernel on this workload's particles, then warm up
    hot.interior_source(d_radtemp, emit, nvol, ts.prt, ts.isv, seed=seed0 - 1)
    ts.opacity()
    ts.coefficients()
    variant, tune_ms = ts.autotune(seed=seed0 - 1, nsample=min(npart, 1_000_000))
    ts.transport(seed0 - 1)  # one untimed step with the chosen variant
    ts.fluxtally()           # leaves every slot vacant again
    ts.sync()
    for k in range(a.warmup):
        one_step(k)
        ts.sync()
    # timed region
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ev_op = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(a.steps)]
    ev_tr = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(a.steps)]
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    clk = Clocks(local)
    steps_total = 0
    counters = []
    ev[0].record(stream)
    for k in range(a.steps):
        kk = a.warmup + k
        hot.interior_source(d_radtemp, emit, nvol, ts.prt, ts.isv, seed=seed0 + 2 * kk)
        ev_op[k][0].record(stream)
        ts.opacity()
        ev_op[k][1].record(stream)
        ts.coefficients()
        ev_tr[k][0].record(stream)
        ts.transport(seed0 + 2 * kk + 1)
        ev_tr[k][1].record(stream)
        ts.fluxtally()
        c = ts.sync()
        counters.append(c)
        steps_total += c["nstepimc"] + c["nstepddmc"]
    ev[1].record(stream)
    torch.cuda.synchronize()
    clocks = clk.stop()
    ms = ev[0].elapsed_time(ev[1])
    t_op = [s.elapsed_time(e) for s, e in ev_op]
    t_tr = [s.elapsed_time(e) for s, e in ev_tr]
    ms_max = ms
    steps_all = steps_total
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_max = float(t.item())
        s = torch.tensor([steps_total], device="cuda", dtype=torch.float64)
        dist.all_reduce(s)
        steps_all = int(s.item())
        # reduce_gridtally / reduce_fluxtally (mpimod_mpi.f:797-948): one exchange per step
        for buf in (ts.tally, ts.jrad, ts.lum, ts.lumdev):
            dist.all_reduce(buf)
    value = steps_all / (ms_max / 1e3)
    peak, peak_kind = measured_peaks()
    tr_ms = statistics.mean(t_tr)
    steps_per_launch = steps_total / a.steps
    achieved = BYTES_PER_STEP * steps_per_launch / (tr_ms / 1e3) / 1e9
    from superlite_b200 import peaks as PK
    issue_peak = PK.measure(local)["warp_inst_issue_per_s"]["value"]
    issue = FP64_TIMESTEP_INST_PER_STEP * steps_per_launch / (tr_ms / 1e3)
    opac_evals = a.ncell * a.ng / (statistics.mean(t_op) / 1e3)
    res = {
        "metric": METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": ms_max / a.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator, superlite_b200/workloads.py)",
        "config": config_dict(a, world),
        "opacity_cell_group_evals_per_s": opac_evals,
        "transport_particle_steps_per_s": steps_per_launch / (tr_ms / 1e3),
        "phase_ms": {"opacity+means": statistics.mean(t_op), "particle_advance": tr_ms},
        "counters_last_step": {k: counters[-1][k] for k in ("npckt", "nflux", "nstepimc", "nstepddmc", "nstepmax",
                                                            "nmethodswap")},
        # bound by instruction issue and latency like the batched line's loop; the
        # HBM reading on the 128 B per particle-step basis beside it (non-binding)
        "roofline": {"bound": "issue", "achieved": issue, "peak": issue_peak, "unit": "warp-instructions/s",
                     "frac": issue / issue_peak,
                     "traffic": FP64_TIMESTEP_DRAM_PER_STEP * steps_per_launch,
                     "traffic_basis": "ncu dram__bytes_read.sum + dram__bytes_write.sum of particle_advance_kernel<5> "
                                      "at 2e5 particles, per particle-step, times this launch's particle-steps",
                     "kernel": f"particle_advance_kernel (variant {variant})",
                     "basis": f"{FP64_TIMESTEP_INST_PER_STEP} warp instructions per particle-step (ncu, variant 1) x "
                              "particle-steps/s of the particle loop; peak = measured FP32-FMA issue rate of this "
                              "GPU (slg_pipe_throughput)",
                     "simt_lanes_per_warp_instruction": FP64_TIMESTEP_LANES_PER_INST,
                     "hbm": {"achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                             "binding": False,
                             "basis": f"{BYTES_PER_STEP:.0f} B per particle-step (event-based SoA traffic); "
                                      f"peak {peak_kind}"}},
        "clocks": clocks,
        "autotune": {"variant": variant, "sample_ms": tune_ms},
        "gpu_launches": 20 * a.steps,
    }
    if not a.no_e2e:
        res["e2e"] = run_e2e(a, hot, case, emit, nvol, params, seed0)
    if rank == 0 and world == 1 and not a.no_cpu:
        res["cpu_baseline"] = cpu_baseline(a, case, hot, ts, emit, nvol, params)
    hot.close()
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(res))


def pinned_particles(n):
    """Packet and vacancy arrays in pinned (page-locked) host memory, as
    numpy views (the torch tensors that own the memory are returned too and
    must stay alive): the e2e copies run at DMA speed, as a host code that
    pins its particle arrays would see."""
    import torch
    from superlite_b200.api import PACKET_DTYPE
    try:
        raw = torch.zeros(n * PACKET_DTYPE.itemsize, dtype=torch.uint8, pin_memory=True)
        vac = torch.ones(n, dtype=torch.int32, pin_memory=True)
    except RuntimeError:  # the host cannot page-lock this much (several ranks per node): pageable arrays
        raw = torch.zeros(n * PACKET_DTYPE.itemsize, dtype=torch.uint8)
        vac = torch.ones(n, dtype=torch.int32)
    return (raw, vac), raw.numpy().view(PACKET_DTYPE), vac.numpy()


def run_e2e(a, hot, case, emit, nvol, params, seed0):
    """Same timestep through the host-pointer C ABI: every phase takes and returns
    host arrays (module arrays of the Fortran driver), copies included."""
    from superlite_b200.api import PACKET_DTYPE
    g = case.gas
    npart = int(a.npart)
    keep, prt, isv = pinned_particles(npart)
    radtemp = g.temp.copy()
    tinv = 1.0 / g.temp
    times, steps = [], 0
    h2d = d2h = 0
    for k in range(1 + a.steps):
        t0 = time.perf_counter()
        hot.interior_source(radtemp, emit, nvol, prt, isv, seed=seed0 + 7 + k)
        op = hot.physical_opacity(g.temp, g.natom, g.nelec, case.grid.vol, g.mass, g.natomfr, g.oc, g.ginv)
        grey, ross = hot.opacity_means(g.temp, op["sig"], op["cap"])
        ol = hot.leakage_opacity(tinv, op["sig"], op["cap"], tauddmc=params.tauddmc, taulump=params.taulump)
        ep = hot.emission_probability(tinv, op["cap"], grey)
        en, num = hot.sourcetally(prt, isv)
        tables = dict(tempinv=tinv, sig=op["sig"], capgrey=grey, emitprob=ep, opaclump=ol, cap=op["cap"])
        r = hot.particle_advance(tables, prt, isv, params, seed=seed0 + 11 + k)
        lum, dev, n = hot.fluxtally(prt, isv, case.groups.wl)
        t1 = time.perf_counter()
        if k > 0:  # first pass warms the staging buffers
            times.append(t1 - t0)
            steps += r["nstepimc"] + r["nstepddmc"]
    P = npart * 64 + npart * 4
    nc, ng = case.grid.nx, case.groups.ng
    gas_b = (5 * nc + 31 * nc + 2 * g.oc.size) * 8
    h2d = P * 4 + gas_b + 3 * nc * ng * 4 + nc * 8 * 20
    d2h = P * 3 + 2 * nc * ng * 4 + nc * ng * 8 * 2 + nc * 8 * 20
    return {"value": steps / sum(times), "unit": "particle-steps/s", "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(d2h), "steps": a.steps,
            "path": "host-pointer C ABI per phase (slg_interior_source .. slg_fluxtally)"}


def cpu_baseline(a, case, hot, ts, emit, nvol, params, budget_s=20.0):
    """The oracle (C++ restatement of the Fortran) on the host cores, timed on a
    bounded sample: the full opacity build once, transport of a particle sample."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    op = po.physical_opacity(case)
    grey = po.planckmean(case.groups.wlinv, case.gas.temp, op["cap"])
    t_opac = time.perf_counter() - t0
    tinv = 1.0 / case.gas.temp
    t0 = time.perf_counter()
    ol = po.leakage_opacity11(case.grid, case.groups.wlinv, tinv, op["sig"], op["cap"], tauddmc=params.tauddmc,
                              taulump=params.taulump)
    ep = po.emission_probability(case.groups.wlinv, tinv, op["cap"], grey, case.groups.nep, case.groups.nepg)
    t_coef = time.perf_counter() - t0
    tt = po.TransportTables(case.grid, case.groups, tinv, op["sig"], op["cap"], grey, ep, ol, params)
    npart = int(a.npart)
    sample = a.cpu_sample or 20000
    while True:
        prt, isv, _, _, _ = po.make_source_particles(case.grid, case.groups, case.gas.temp, L_BOL, sample)
        st = po.rnd_init(cores, 0)
        t0 = time.perf_counter()
        r = po.particle_advance(tt, prt, isv, rngmode=0, nthreads=cores, rnd_states=st)
        dt = time.perf_counter() - t0
        if dt > 2.0 or a.cpu_sample or sample >= npart:
            break
        sample = min(npart, int(sample * max(2.0, budget_s / max(dt, 1e-3) * 0.5)))
    steps = r["nstepimc"] + r["nstepddmc"]
    scale = npart / sample
    t_step = t_opac + t_coef + dt * scale
    return {"value": steps * scale / t_step, "unit": "particle-steps/s", "cores": cores, "kind": "port",
            "sample": f"{sample} particles of the {npart}-particle timestep (mzran, OpenMP static,1), "
                      f"full opacity build ({t_opac:.2f} s, 1 thread) + coefficients; transport time scaled "
                      f"by {scale:.1f}",
            "transport_particle_steps_per_s": steps / dt}


# ------------------------------------------------------------------ batched workload
SEED_BATCH = 4


def batched_config(a, world, b):
    return {"workload": "batched: independent ejecta models, one persistent mixed-precision launch, "
                        "graph-captured steps (128 models)",
            "models_per_gpu": int(len(b.nx)), "shells_total": int(b.nx.sum()), "shells_range": [50, 400],
            "particles_per_gpu": int(b.npart.sum()), "particles_range": [1e5, 1e7],
            "snapshot_days_range": [1.0, 30.0], "groups": int(b.groups.ng),
            "opacity": "analytic grey kappa = 0.1 (rho/1e-13) (T/1e4)^-1.5 cm^2/g (1 Msun broken power-law ejecta, T ~ U(6000, 14000) K)",
            "tauddmc": 5.0, "taulump": 10.0, "transport_precision": "mixed (FP32 distances, FP64 weights/tallies)",
            "graph_steps": a.steps, "parallelism": f"models{world}",
            "l2": f"inputs larger than L2 (particle array {b.npart.sum() * 64 / 1e9:.1f} GB per GPU)"}


def _events():
    import torch
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def _lum_rows(ts):
    return (ts.lum.cpu().numpy().copy(), ts.lumdev.cpu().numpy().copy(), ts.lumnum.cpu().numpy().copy())


def batched_transport(ts, seed, precision, autotune=False):
    """One step of the batch (sources, opacities, coefficients), then ONE
    particle-loop launch over all models in `precision` (0: FP64, 1: mixed),
    the loop timed with CUDA events on the library's stream, then the flux
    tallies.  The sources depend only on `seed`, so both precisions transport
    the same particles.  Returns a dict (ms, steps, lum rows, counters)."""
    from superlite_b200.api import transport_out_dict
    ts.set_precision(precision)
    ts.prepare(seed)
    variant = None
    if autotune:
        variant, _ = ts.autotune(seed=seed, nsample=1_000_000)
    ts.sync()
    e0, e1 = _events()
    e0.record(ts.stream)
    ts.transport(seed)
    e1.record(ts.stream)
    ts.flux()
    ts.sync()
    c = transport_out_dict(ts._tout)
    lum, dev, num = _lum_rows(ts)
    ts.set_precision(1)
    return {"ms": e0.elapsed_time(e1), "steps": int(c["nstepimc"] + c["nstepddmc"]), "lum": lum, "dev": dev,
            "num": num, "counters": c, "variant": variant}


def fp64_per_model(b, ts, params, local, seed):
    """The plain FP64 form on the same models: one model per call, as the
    single-model C ABI is called by a driver that runs the models one after
    another (each model in its own context; every call completes before the
    next).  Each call's particle loop is timed with CUDA events on its
    context's stream; the sum of those device times is the FP64 form's time
    (the host wall time around the calls is reported beside it).  Returns a
    dict (ms, wall_s, steps, variant, lum rows of the same step)."""
    import torch
    from superlite_b200 import HotPath
    from superlite_b200.capi import ptr
    hots = []
    co = np.concatenate([[0], np.cumsum(b.nx)])
    eo = co + np.arange(len(b.nx) + 1)
    po = np.concatenate([[0], np.cumsum(b.npart)])
    for m in range(len(b.nx)):
        h = HotPath(local)
        h.set_groups(b.groups.wl)
        h.set_grid(b.xarr[eo[m]:eo[m + 1]], b.vxarr[eo[m]:eo[m + 1]], b.vol[co[m]:co[m + 1]],
                   b.divv[co[m]:co[m + 1]])
        hots.append(h)
    ts.set_precision(1)
    ts.prepare(seed)
    ts.sync()
    sl = lambda t, m: t[co[m]:co[m + 1]]
    # the FP64 kernel's variant: autotuned once (largest model, 1e6-particle
    # sample) and used by every model's context
    import ctypes as C
    big = int(np.argmax(b.npart))
    tin = HotPath.transport_in(sl(ts.tempinv, big), sl(ts.sig, big), sl(ts.capgrey, big), sl(ts.emitprob, big),
                               sl(ts.opaclump, big), sl(ts.cap, big), params, 0)
    best, ms = C.c_int32(0), (C.c_float * 4)()
    hb = hots[big]
    hb._check(hb.lib.slg_autotune_transport(hb.h, C.byref(tin), ptr(ts.prt[po[big]:po[big + 1]]),
                                            ptr(ts.isv[po[big]:po[big + 1]]), int(b.npart[big]), seed,
                                            1_000_000, C.byref(best), ms))
    for h in hots:
        h._check(h.lib.slg_set_transport_variant(h.h, int(best.value)))
    hb.sync()
    outs, dev_ms = [], 0.0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for m, h in enumerate(hots):
        tables = dict(tempinv=sl(ts.tempinv, m), sig=sl(ts.sig, m), capgrey=sl(ts.capgrey, m),
                      emitprob=sl(ts.emitprob, m), opaclump=sl(ts.opaclump, m), cap=sl(ts.cap, m))
        stream = torch.cuda.ExternalStream(h.stream(), device=torch.device("cuda", local))
        e0, e1 = _events()
        e0.record(stream)
        outs.append(h.particle_advance_dev(tables, ts.prt[po[m]:po[m + 1]], ts.isv[po[m]:po[m + 1]],
                                           sl(ts.tally, m), sl(ts.jrad, m), sl(ts.eamp, m), params,
                                           seed=seed, precision=0))
        e1.record(stream)
        h.sync()
        dev_ms += e0.elapsed_time(e1)
    wall = time.perf_counter() - t0
    steps = sum(o.nstepimc + o.nstepddmc for o in outs)
    ts.flux()  # tally the escaped particles and free their slots in the batched context
    ts.sync()
    lum, dev, num = _lum_rows(ts)
    for h in hots:
        h.close()
    return {"ms": dev_ms, "wall_s": wall, "steps": int(steps), "variant": int(best.value), "lum": lum, "dev": dev,
            "num": num}


def luminosity_zscores(A, B, t_days, nbin=4):
    """Per model and wavelength bin (nbin contiguous bins of groups), z = (L_A -
    L_B) / sqrt(lumdev_A + lumdev_B), lumdev = sum of e^2 of the escaped
    particles (fluxtally.f:47-49; an upper bound of the variance of L)."""
    la, da, lb, db = A["lum"], A["dev"], B["lum"], B["dev"]
    nm, ng = la.shape
    edges = np.linspace(0, ng, nbin + 1).astype(int)
    zs = []
    for m in range(nm):
        for a, b in zip(edges[:-1], edges[1:]):
            v = da[m, a:b].sum() + db[m, a:b].sum()
            if v > 0:
                zs.append(((la[m, a:b].sum() - lb[m, a:b].sum()) / math.sqrt(v), m))
    z = np.array([q[0] for q in zs])
    worst = sorted(zs, key=lambda q: -abs(q[0]))[:5]
    tot_a, tot_b = la.sum(axis=1), lb.sum(axis=1)
    rel = np.abs(tot_a - tot_b) / np.maximum(np.abs(tot_b), 1e-300)
    return {"comparisons": int(len(z)), "bins_per_model": nbin, "max_abs_z": float(np.abs(z).max()),
            "frac_abs_z_gt_3": float((np.abs(z) > 3).mean()), "expected_frac_gt_3_if_normal": 0.0027,
            "worst": [{"model": int(m), "t_days": round(float(t_days[m]), 3), "z": round(float(v), 3)}
                      for v, m in worst],
            "median_rel_diff_total_luminosity": float(np.median(rel))}


def run_batched(a):
    import torch
    from superlite_b200 import HotPath, workloads as W
    from superlite_b200.timestep import BatchTimestep
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
        # the single-GPU comparisons (FP64 forms, the snapshot series, the full
        # timestep, opacity) would
        # only repeat per rank what the N = 1 line reports; the N-GPU line keeps
        # the timed step, e2e and the clocks, so the GPUs are held briefly
        a.no_fp64 = a.no_cases = a.no_opacity = True
    b = W.analytic_batch(nmodel=a.nmodel, seed=SEED_BATCH + 1000 * rank)
    if a.npart_scale != 1.0:
        b = W.analytic_batch(nmodel=a.nmodel, seed=SEED_BATCH + 1000 * rank,
                             npart=np.maximum(1000, (b.npart * a.npart_scale).astype(np.int64)))
    params = W.TransportParams()
    hot = HotPath(local)
    ts = BatchTimestep(hot, b, params, precision=1)
    stream = ts.stream
    seed0 = 1000 * (rank + 1)
    # warm-up 1: sources and opacities, the autotuner on a sample of this
    # step's particles (the first 1e6 slots), then the particle loop with the
    # chosen variant
    ts.prepare(seed0 - 1)
    if a.transport_variant is None:
        variant, tune_ms = ts.autotune(seed=seed0 - 1, nsample=1_000_000)
    else:
        variant, tune_ms = a.transport_variant, None
        hot._check(hot.lib.slg_set_transport_variant(hot.h, variant))
    ts.finish(seed0 - 1)
    ts.sync()
    # the kernel variants on whole steps (untimed, beside the warm-ups): the
    # sample above comes from the first models' particles only, so each variant
    # runs one full particle loop, timed with CUDA events, and the fastest is
    # kept for the warm-ups and the timed steps
    ev_p = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    full_ms = {}
    if a.tune_steps and a.transport_variant is None:
        for v in range(4):
            hot._check(hot.lib.slg_set_transport_variant(hot.h, v))
            ts.prepare(seed0 - 10 - v)
            ev_p[1].record(stream)
            ts.finish(seed0 - 10 - v)
            ev_p[2].record(stream)
            ts.sync()
            full_ms[v] = ev_p[1].elapsed_time(ev_p[2])
        variant = min(full_ms, key=full_ms.get)
        hot._check(hot.lib.slg_set_transport_variant(hot.h, variant))
    # warm-ups 2..W (uncaptured); the last one also times its phases
    t_prep = t_tr = None
    for k in range(1, a.warmup):
        if k == a.warmup - 1:
            ev_p[0].record(stream)
            ts.prepare(seed0 + k)
            ev_p[1].record(stream)
            ts.finish(seed0 + k)
            ev_p[2].record(stream)
        else:
            ts.step(seed0 + k)
        ts.sync()
        if k == a.warmup - 1:
            t_prep, t_tr = ev_p[0].elapsed_time(ev_p[1]), ev_p[1].elapsed_time(ev_p[2])
    # the timed steps: one CUDA graph of a.steps whole timesteps, replayed once
    ts.capture(a.steps, seed0 + a.warmup)
    hot.transport_totals(reset=True)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    clk = Clocks(local)
    ev[0].record(stream)
    ts.replay(1)
    ev[1].record(stream)
    torch.cuda.synchronize()
    clocks = clk.stop()
    ms = ev[0].elapsed_time(ev[1])
    tot = hot.transport_totals()
    steps_total = tot["nstepimc"] + tot["nstepddmc"]
    ms_max, steps_all = ms, steps_total
    if world > 1:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms_max = float(t.item())
        s = torch.tensor([steps_total], device="cuda", dtype=torch.float64)
        torch.distributed.all_reduce(s)
        steps_all = int(s.item())
    value = steps_all / (ms_max / 1e3)
    if rank == 0:
        print(f"[bench] batched: {value:.4g} particle-steps/s, {ms_max:.0f} ms for {a.steps} step(s)", file=sys.stderr,
              flush=True)
    peak, peak_kind = measured_peaks()
    tr_rate = (steps_total / a.steps) / (t_tr / 1e3) if t_tr else None
    achieved = BYTES_PER_STEP * tr_rate / 1e9 if tr_rate else None
    from superlite_b200 import peaks as PK
    pipes = PK.measure(local)
    issue_peak = pipes["warp_inst_issue_per_s"]["value"]
    issue = MIXED_WARP_INST_PER_STEP[variant] * tr_rate if tr_rate else None
    res = {
        "metric": METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": ms_max / a.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic (seeded generator, superlite_b200/workloads.py)",
        "config": batched_config(a, world, b),
        "phase_ms_last_warmup_step": {"sources+opacity+coefficients": t_prep, "particle_advance": t_tr},
        "counters": {**{k: tot[k] for k in ("npckt", "nflux", "nstepimc", "nstepddmc", "nstepmax", "nmethodswap",
                                            "ierr")},
                     # events by ptcl2%idist (particle_advance.f90:211-212): -3 (both leaks), -2 (DDMC
                     # effective scatter), -1, 0, 1 collision, 2 Thomson, 3 Doppler, 4 boundary, 5..7
                     "ndist": [int(x) for x in tot["ndist"]]},
        # The particle loop is bound by instruction issue and latency (divergent, dependent gathers
        # of L2-resident tables), not by HBM: its roofline is the measured warp-instruction issue
        # rate; the HBM reading on the 128 B per particle-step basis is kept beside it (non-binding).
        "roofline": {"bound": "issue", "achieved": issue, "peak": issue_peak, "unit": "warp-instructions/s",
                     "frac": issue / issue_peak if issue else None,
                     # DRAM bytes of one launch: ncu dram__bytes_read.sum + dram__bytes_write.sum of this
                     # kernel on the same batch with particle budgets x 0.1 (4.11e9-4.20e9 B for 2.944e7
                     # particles over the four variants: the packets read and written once, plus table
                     # and tally traffic), scaled by the particles of this launch
                     "traffic": 4.19e9 * float(b.npart.sum()) / 2.944e7,
                     "traffic_basis": "ncu capture of particle_advance_mixed_kernel<7> at 0.1x particle budgets "
                                      "(4.19 GB), scaled by particles",
                     "kernel": f"particle_advance_mixed_kernel<{variant + 4}>",
                     "basis": f"{MIXED_WARP_INST_PER_STEP[variant]} warp instructions per particle-step of this "
                              "variant (ncu) x particle-steps/s of the last warm-up step's particle loop; peak = "
                              "measured FP32-FMA issue rate of this GPU (slg_pipe_throughput, one warp instruction "
                              "per cycle per scheduler)",
                     "simt_lanes_per_warp_instruction": MIXED_LANES_PER_INST[variant],
                     "hbm": {"achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak if achieved else None, "binding": False,
                             "basis": f"{BYTES_PER_STEP:.0f} B per particle-step (event-based SoA traffic); "
                                      f"peak {peak_kind}"}},
        "pipe_peaks": {k: pipes[k]["value"] for k in ("fp64_fma_flops", "fp64_exp_per_s", "fp32_fma_flops",
                                                      "int32_imad_per_s", "warp_inst_issue_per_s")},
        "clocks": clocks, "autotune": {"variant": variant, "sample_ms": tune_ms,
                                       "particle_loop_ms_by_variant": {str(k): v for k, v in full_ms.items()} or None},
        "gpu_launches": None,
    }
    # kernels of one step: 6 (sources) + 1 (analytic opacity) + 1 (means) + 1 (leakage) + 1 (emitprob)
    # + 1 (sourcetally) + 2 (cell tables, particle loop) + 1 (counter fold) + nmodel (flux tallies);
    # + 1 epoch counter per graph replay
    res["gpu_launches"] = (14 + int(len(b.nx))) * a.steps + 1
    def whole_job(steps, seconds):
        # every rank runs its own models: steps add up, the job takes the slowest rank's time
        if world == 1:
            return steps / seconds, steps, seconds
        import torch.distributed as dist
        t = torch.tensor([float(steps)], dtype=torch.float64, device="cuda")
        dist.all_reduce(t)
        m = torch.tensor([float(seconds)], dtype=torch.float64, device="cuda")
        dist.all_reduce(m, op=dist.ReduceOp.MAX)
        return float(t.item()) / float(m.item()), int(t.item()), float(m.item())

    if not a.no_fp64:
        # the three forms on one comparison step (same sources), each particle loop timed the same way:
        # CUDA events on the launching stream around the loop (cell tables + kernel)
        S = seed0 + 999
        mix = batched_transport(ts, S, 1)
        f64b = batched_transport(ts, S, 0, autotune=True)
        f64p = fp64_per_model(b, ts, params, local, S)
        r_mix = whole_job(mix["steps"], mix["ms"] / 1e3)[0]
        r_f64b = whole_job(f64b["steps"], f64b["ms"] / 1e3)[0]
        r_f64p, st64, dt64 = whole_job(f64p["steps"], f64p["ms"] / 1e3)
        res["comparison_step"] = {
            "timing": "particle loop only, CUDA events on the launching stream, same step (same sources)",
            "mixed_batched": {"value": r_mix, "unit": "particle-steps/s", "steps": mix["steps"], "ms": mix["ms"]},
            "fp64_batched": {"value": r_f64b, "unit": "particle-steps/s", "steps": f64b["steps"], "ms": f64b["ms"],
                             "variant": f64b["variant"],
                             "form": "FP64 particle loop, all models in one persistent launch"},
            "fp64_plain_per_model": {"value": r_f64p, "unit": "particle-steps/s", "steps": st64, "ms": f64p["ms"],
                                     "wall_s": f64p["wall_s"], "variant": f64p["variant"],
                                     "form": "FP64 particle loop, one call per model (own context), each "
                                             "completed before the next; sum of the calls' device times"},
        }
        res["mixed_batched_over_fp64_plain"] = r_mix / r_f64p
        res["fp64_batched_over_fp64_plain"] = r_f64b / r_f64p
        res["mixed_batched_over_fp64_batched"] = r_mix / r_f64b
        res["mixed_vs_fp64_luminosity"] = luminosity_zscores(mix, f64b, b.t_days)
        res["mixed_vs_fp64_luminosity"]["pair"] = "mixed batched vs FP64 batched, same source particles"
    if not a.no_e2e:
        e = batched_e2e(a, b, params, local, seed0)
        e["value"], e["particle_steps"], e["seconds"] = whole_job(e["particle_steps"], e["seconds"])
        res["e2e"] = e
    if not a.no_cases:
        res["snapshot_series"] = snapshot_series_measure(a, local, rank, world)
        res["full_timestep"] = full_timestep_measure(a, local, rank, world)
    if not a.no_opacity:
        res["opacity"] = opacity_measure(local, exp_per_s=pipes["fp64_exp_per_s"]["value"])
        res["opacity_cell_group_evals_per_s"] = res["opacity"]["forward"]["cell_group_evals_per_s"]
    if rank == 0 and world == 1 and not a.no_cpu:
        res["cpu_baseline"] = batched_cpu_baseline(a, b, params)
    hot.close()
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(res))


def batched_e2e(a, b, params, local, seed0):
    """One step of the batch through the host-pointer C ABI (the calls a
    Fortran driver makes, every module array copied in and out)."""
    from superlite_b200 import HotPath
    from superlite_b200.api import PACKET_DTYPE
    hot = HotPath(local)
    hot.set_groups(b.groups.wl)
    hot.set_models(b.nx, b.npart, b.xarr, b.vxarr, b.vol, b.divv)
    n = int(b.npart.sum())
    keep, prt, isv = pinned_particles(n)
    emit, _ = hot.sourceenergy(b.temp, L_BOL)
    nvol, _ = hot.models_sourcenumbers(emit, b.npart)
    tinv = 1.0 / b.temp
    times, steps = [], 0
    for k in range(1):  # one step (a step of this batch runs for about a minute)
        t0 = time.perf_counter()
        hot.interior_source(b.temp, emit, nvol, prt, isv, seed=seed0 + 31 + k)
        sig, cap = hot.analytic_opacity(b.temp, b.rho, kind=1)
        grey, ross = hot.opacity_means(b.temp, sig, cap)
        ol = hot.leakage_opacity(tinv, sig, cap, tauddmc=params.tauddmc, taulump=params.taulump)
        ep = hot.emission_probability(tinv, cap, grey)
        tables = dict(tempinv=tinv, sig=sig, capgrey=grey, emitprob=ep, opaclump=ol, cap=cap)
        r = hot.particle_advance(tables, prt, isv, params, seed=seed0 + 41 + k, precision=1)
        hot.fluxtally(prt, isv, b.groups.wl)
        t1 = time.perf_counter()
        times.append(t1 - t0)
        steps += r["nstepimc"] + r["nstepddmc"]
    hot.close()
    nc, ng = int(b.nx.sum()), b.groups.ng
    P = n * 68
    h2d = 3 * P + nc * 8 * 12 + 3 * nc * ng * 4 + nc * hot.nep * 8
    d2h = 3 * P + nc * 8 * 20 + 2 * nc * ng * 4 + nc * ng * 8 + 3 * len(b.nx) * ng * 8
    return {"value": steps / sum(times), "unit": "particle-steps/s", "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(d2h), "steps": 1, "particle_steps": int(steps), "seconds": sum(times),
            "pinned": bool(keep[0].is_pinned()),
            "path": "host-pointer C ABI per phase (slg_interior_source .. slg_fluxtally), all models; "
                    "particle arrays in pinned host memory; first step of a fresh context (device buffers "
                    "allocated inside the timed step)"}


def stratified_order(t_days):
    """Models in an order whose every prefix spreads over the snapshot times:
    sorted by t, then visited in bit-reversed rank order (0, n/2, n/4, 3n/4 ...)."""
    n = len(t_days)
    srt = np.argsort(t_days, kind="stable")
    bits = max(1, (n - 1).bit_length())
    ranks = [int(format(i, f"0{bits}b")[::-1], 2) for i in range(1 << bits)]
    return [int(srt[r]) for r in ranks if r < n]


def batched_cpu_baseline(a, b, params, budget_s=20.0):
    """The oracle (C++ restatement of the Fortran, FP64, mzran, OpenMP over
    particles) on a bounded sample: models taken in a stratified order over
    their snapshot times (every prefix spans early and late models), a
    particle sample each, until the time budget is spent."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po
    from superlite_b200 import workloads as W
    cores = os.cpu_count() or 1
    co = np.concatenate([[0], np.cumsum(b.nx)])
    eo = co + np.arange(len(b.nx) + 1)
    steps = 0
    dt = 0.0
    used = []
    for m in stratified_order(b.t_days):
        g = W.Grid(int(b.nx[m]), 0.0, b.xarr[eo[m]:eo[m + 1]], b.vxarr[eo[m]:eo[m + 1]],
                   b.vol[co[m]:co[m + 1]], b.divv[co[m]:co[m + 1]])
        T, rho = b.temp[co[m]:co[m + 1]], b.rho[co[m]:co[m + 1]]
        sig, cap = po.analytic_opacity(b.groups.wlinv, T, rho, kind=1)
        tinv = 1.0 / T
        grey = po.planckmean(b.groups.wlinv, T, cap)
        ol = po.leakage_opacity11(g, b.groups.wlinv, tinv, sig, cap, tauddmc=params.tauddmc, taulump=params.taulump)
        ep = po.emission_probability(b.groups.wlinv, tinv, cap, grey, b.groups.nep, b.groups.nepg)
        tt = po.TransportTables(g, b.groups, tinv, sig, cap, grey, ep, ol, params)
        sample = int(min(b.npart[m], a.cpu_sample or 4000))
        prt, isv, _, _, _ = po.make_source_particles(g, b.groups, T, L_BOL, sample)
        st = po.rnd_init(cores, m)
        t0 = time.perf_counter()
        r = po.particle_advance(tt, prt, isv, rngmode=0, nthreads=cores, rnd_states=st)
        dt += time.perf_counter() - t0
        steps += r["nstepimc"] + r["nstepddmc"]
        used.append((m, sample))
        if dt > budget_s:
            break
    td = np.array([b.t_days[m] for m, _ in used])
    return {"value": steps / dt, "unit": "particle-steps/s", "cores": cores, "kind": "port",
            "sample": f"{len(used)} of {len(b.nx)} models in a stratified order over snapshot time "
                      f"(t = {td.min():.2f}-{td.max():.2f} d, median {np.median(td):.2f} d), {used[0][1]} particles "
                      f"each (mzran, OpenMP static,1, FP64 oracle), transport only",
            "models": [m for m, _ in used]}


# ------------------------------------------------------------------ the other two transport configurations
SNAPSHOT_SERIES = dict(nx=64, ng=100, npart=1_000_000, nsnap=20, t0=1.0, t1=30.0, seed=21)


def snapshot_series_measure(a, local, rank, world):
    """The CPU-runnable case: 64 shells (v 0-1.5e9 cm/s, 1 Msun broken power law,
    T ~ U(6000, 14000) K per shell, seeded), analytic grey opacity, 100 groups,
    1e6 particles per snapshot, 20 snapshots log-spaced in t = 1-30 d, the
    plain FP64 particle loop (one model per context, as the reference runs it).
    Every snapshot: sources, opacity, means, leakage, emission probabilities,
    source tally, particle loop and flux tally on the device; the particle
    loops and the whole snapshots timed with CUDA events.  Beside it the
    oracle (mzran, all host cores) on a bounded particle sample of every
    snapshot."""
    import torch
    from superlite_b200 import HotPath, workloads as W
    from superlite_b200.timestep import BatchTimestep
    C0 = SNAPSHOT_SERIES
    ts_days = np.geomspace(C0["t0"], C0["t1"], C0["nsnap"])
    params = W.TransportParams()
    steps = 0
    ms_tr = ms_all = 0.0
    models = []
    for k, td in enumerate(ts_days):
        b = W.analytic_batch(nmodel=1, seed=C0["seed"] + 1000 * rank, nx=[C0["nx"]], npart=[C0["npart"]],
                             t_range_days=(td, td))
        models.append(b)
        hot = HotPath(local)
        ts = BatchTimestep(hot, b, params, precision=0)
        seed = 100 + k
        if k == 0:  # warm-up snapshot: the FP64 kernel variant picked on this workload
            ts.prepare(seed)
            ts.autotune(seed=seed, nsample=C0["npart"])
            ts.finish(seed)
            ts.sync()
        e0, e1 = _events()
        e2, e3 = _events()
        e0.record(ts.stream)
        ts.prepare(seed)
        e2.record(ts.stream)
        ts.transport(seed)
        e3.record(ts.stream)
        ts.flux()
        e1.record(ts.stream)
        ts.sync()
        c = ts._tout
        steps += int(c.nstepimc + c.nstepddmc)
        ms_tr += e2.elapsed_time(e3)
        ms_all += e0.elapsed_time(e1)
        hot.close()
    res = {"workload": "CPU-runnable case: 64 shells, analytic grey opacity, 100 groups, 1e6 particles, 20 "
                       "snapshots t = 1-30 d, plain FP64 particle loop",
           "metric": METRIC, "value": steps / (ms_all / 1e3), "unit": "particle-steps/s",
           "particle_loop_value": steps / (ms_tr / 1e3), "particle_steps": steps, "ms_all_snapshots": ms_all,
           "ms_particle_loops": ms_tr, "timing": "CUDA events on the library stream, every phase of every snapshot"}
    if rank == 0 and world == 1 and not a.no_cpu:
        res["cpu_baseline"] = snapshot_series_cpu(models, params)
    return res


def snapshot_series_cpu(models, params, sample=40_000):
    """The oracle on every snapshot of the CPU-runnable case, a particle sample each."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po
    from superlite_b200 import workloads as W
    cores = os.cpu_count() or 1
    steps, dt, npart = 0, 0.0, 0
    for k, b in enumerate(models):
        g = W.Grid(int(b.nx[0]), 0.0, b.xarr, b.vxarr, b.vol, b.divv)
        T, rho = b.temp, b.rho
        sig, cap = po.analytic_opacity(b.groups.wlinv, T, rho, kind=1)
        tinv = 1.0 / T
        grey = po.planckmean(b.groups.wlinv, T, cap)
        ol = po.leakage_opacity11(g, b.groups.wlinv, tinv, sig, cap, tauddmc=params.tauddmc, taulump=params.taulump)
        ep = po.emission_probability(b.groups.wlinv, tinv, cap, grey, b.groups.nep, b.groups.nepg)
        tt = po.TransportTables(g, b.groups, tinv, sig, cap, grey, ep, ol, params)
        prt, isv, _, _, _ = po.make_source_particles(g, b.groups, T, L_BOL, sample)
        st = po.rnd_init(cores, k)
        t0 = time.perf_counter()
        r = po.particle_advance(tt, prt, isv, rngmode=0, nthreads=cores, rnd_states=st)
        dt += time.perf_counter() - t0
        steps += r["nstepimc"] + r["nstepddmc"]
        npart = int(b.npart[0])
    return {"value": steps / dt, "unit": "particle-steps/s", "cores": cores, "kind": "port",
            "sample": f"{sample} of {npart} particles in each of the {len(models)} snapshots (mzran, OpenMP "
                      f"static,1, FP64 oracle), particle loop only, {dt:.1f} s"}


def full_timestep_measure(a, local, rank, world, npart=50_000_000):
    """The full timestep: 256 shells x 2000 groups, physical LTE opacity from
    5e5 synthetic lines on the reference's Verner, Sutherland and data.ion
    tables (Saha populations from the device equation of state), 5e7 source
    particles, DDMC where a shell is optically thick; one step with the FP64
    particle loop and one with the mixed-precision loop (each after one
    untimed step), every phase on the device, CUDA events."""
    import dataclasses
    import torch
    from superlite_b200 import HotPath, workloads as W
    from superlite_b200.timestep import DeviceTimestep
    A = W.load_atomic_data(ATOMIC_NPZ)
    case = W.opacity_case(ncell=256, ng=2000, nline=500_000, seed=SEED_CASE, t_days=T_DAYS, tables=A.tables)
    params = W.TransportParams()
    out = {"workload": "full timestep: 256 shells x 2000 groups, physical opacity (5e5 synthetic lines, the "
                       "reference's Verner/Sutherland/data.ion tables), 5e7 particles",
           "metric": METRIC, "unit": "particle-steps/s", "particles": npart}
    for name, prec in (("fp64", 0), ("mixed", 1)):
        hot = HotPath(local)
        hot.set_groups(case.groups.wl)
        hot.set_grid(case.grid.xarr, case.grid.vxarr, case.grid.vol, case.grid.divv)
        hot.set_ions(A.ion, float(case.gas.temp[0]))
        g = case.gas
        nel, oc, ginv, _ = hot.saha_eos(g.temp, g.natom, case.grid.vol, g.natomfr, np.ones(case.grid.nx), acc=1e-10,
                                        noc=A.ion.nstage - 1)
        cz = dataclasses.replace(case, gas=dataclasses.replace(g, nelec=nel, oc=oc, ginv=ginv,
                                                               ion_ni=np.ascontiguousarray(A.ion.ni, np.int32)))
        ts = DeviceTimestep(hot, cz, params, npart=npart, precision=prec)
        emit, _ = hot.sourceenergy(g.temp, L_BOL)
        nvol, _ = hot.sourcenumbers(emit, npart, npart)
        seed0 = 7000 + 1000 * rank
        for k in range(2):  # untimed step (and the autotuner), then the timed one
            hot.interior_source(ts.gas["temp"], emit, nvol, ts.prt, ts.isv, seed=seed0 + 2 * k)
            e0, e1 = _events()
            e2, e3 = _events()
            e0.record(ts.stream)
            ts.opacity()
            ts.coefficients()
            if k == 0:
                ts.autotune(seed=seed0, nsample=1_000_000)
            e2.record(ts.stream)
            ts.transport(seed0 + 2 * k + 1)
            e3.record(ts.stream)
            ts.fluxtally()
            e1.record(ts.stream)
            c = ts.sync()
        st = int(c["nstepimc"] + c["nstepddmc"])
        out[name] = {"value": st / (e2.elapsed_time(e3) / 1e3), "particle_steps": st,
                     "ms_particle_loop": e2.elapsed_time(e3),
                     "ms_step_after_sources": e0.elapsed_time(e1),
                     "steps_per_particle": st / max(int(c["npckt"]), 1)}
        hot.close()
        del ts
        torch.cuda.empty_cache()
    out["mixed_over_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
    return out


# ------------------------------------------------------------------ opacity forward / adjoint
OPACITY_SIZES = {1: (256, 2000, 500_000), 4: (4096, 10000, 2_000_000)}


def opacity_measure(local, reps=5, which=1, exp_per_s=None):
    """Opacity build of the opacity case (which=1: 256 shells x 2000 groups x
    5e5 lines) or the opacity case at scale (which=4: 4096 x 10000 x 2e6) on the
    reference's Verner, Sutherland and data.ion tables (Saha populations of
    every bound stage), FP64, forward and reverse through the device C ABI
    (slg_dev_opacity_grad_forward / _backward): cell-group evaluations per
    second of each, timed with CUDA events on the library's stream.
    exp_per_s: the measured FP64 exp rate (one exp per line-shell term is the
    kernels' binding work)."""
    import numpy as np
    import torch
    from superlite_b200 import HotPath, workloads as W
    from superlite_b200.capi import ptr
    ncell, ngroup, nline = OPACITY_SIZES[which]
    A = W.load_atomic_data(ATOMIC_NPZ)
    case = W.opacity_case(ncell=ncell, ng=ngroup, nline=nline, seed=SEED_CASE, t_days=T_DAYS, tables=A.tables)
    hot = HotPath(local)
    hot.set_groups(case.groups.wl)
    hot.set_grid(case.grid.xarr, case.grid.vxarr, case.grid.vol, case.grid.divv)
    g = case.gas
    hot.set_atomic_data(np.ascontiguousarray(A.ion.ni, dtype=np.int32), A.ion.nstage - 1, case.lines, case.bf_ph1,
                        case.bf_ph2, case.ff_gff)
    hot.set_ions(A.ion, float(g.temp[0]))
    m = np.ascontiguousarray([W.ELEM_MASS.get(z, 2.0 * z) for z in range(1, W.NELEM + 1)], dtype=np.float64)
    hot._check(hot.lib.slg_set_element_masses(hot.h, len(m), ptr(m)))
    dev = torch.device("cuda", local)
    nc, ng = hot.nx, hot.ng
    f64 = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=dev)
    T, R, X = f64(g.temp), f64(g.rho), f64(g.massfr)
    e = lambda *sh: torch.empty(sh, dtype=torch.float64, device=dev)
    nelec = torch.ones(nc, dtype=torch.float64, device=dev)
    cap, sig, grey, ross, ol = e(nc, ng), e(nc), e(nc), e(nc), e(nc, 11)
    gen = torch.Generator(device=dev).manual_seed(5)
    gcap = torch.randn((nc, ng), generator=gen, device=dev, dtype=torch.float64)
    gsig, ggrey, gross = (torch.randn(nc, generator=gen, device=dev, dtype=torch.float64) for _ in range(3))
    gol = torch.randn((nc, 11), generator=gen, device=dev, dtype=torch.float64)
    gT, gR, gX = e(nc), e(nc), torch.empty_like(X)
    torch.cuda.synchronize()
    L, h = hot.lib, hot.h
    acc, taud, taul = 1e-14, 5.0, 10.0

    def fwd():
        nelec.fill_(1.0)
        hot._check(L.slg_dev_opacity_grad_forward(h, ptr(T), ptr(R), ptr(X), acc, taud, taul, ptr(nelec), ptr(cap),
                                                  ptr(sig), ptr(grey), ptr(ross), ptr(ol)))

    def bwd():
        hot._check(L.slg_dev_opacity_grad_backward(h, ptr(T), ptr(R), ptr(X), acc, taud, taul, ptr(nelec), ptr(cap),
                                                   ptr(sig), ptr(grey), ptr(ross), ptr(ol), ptr(gcap), ptr(gsig),
                                                   ptr(ggrey), ptr(gross), ptr(gol), ptr(gT), ptr(gR), ptr(gX)))
    stream = torch.cuda.ExternalStream(hot.stream(), device=dev)
    out = {}
    for name, f in (("forward", fwd), ("backward", bwd)):
        for _ in range(3):
            f()
        hot.sync()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        ev[0].record(stream)
        for _ in range(reps):
            f()
        ev[1].record(stream)
        hot.sync()
        ms = ev[0].elapsed_time(ev[1]) / reps
        out[name] = {"ms": ms, "cell_group_evals_per_s": nc * ng / (ms / 1e3)}
    hot.close()
    lines_bytes = 16 * len(case.lines)
    out["workload"] = f"opacity: {ncell} shells x {ngroup} groups x {nline:.0e} synthetic lines, the reference's " \
                      "Verner, Sutherland and data.ion tables, Saha populations, FP64 (forward: EOS + bb/bf/ff + " \
                      "means + leakage; backward: adjoint of all of it)"
    out["line_shell_terms_per_s"] = {k: nline * ncell / (out[k]["ms"] / 1e3) for k in ("forward", "backward")}
    if exp_per_s:
        out["fp64_exp_roof"] = {
            "peak_exp_per_s": exp_per_s,
            "frac": {k: out["line_shell_terms_per_s"][k] / exp_per_s for k in ("forward", "backward")},
            "basis": "line-shell terms/s (one FP64 exp each, the dominant work) / measured FP64 exp rate "
                     "(slg_pipe_throughput); the whole build's time in the denominator"}
    out["bound"] = "FP64 issue (one exp per line-shell term), not HBM: the algorithmic bytes " \
                   f"({(lines_bytes + 8 * nc * ng * 3) / 1e6:.0f} MB: lines, cap64, dL/dcap) take " \
                   f"{(lines_bytes + 8 * nc * ng * 3) / (measured_peaks()[0] * 1e9) * 1e3:.4f} ms at the measured " \
                   "HBM copy bandwidth"
    return out


# ------------------------------------------------------------------ reference arm
def run_reference_batched(a):
    """The reference's CPU path (the oracle restatement, FP64, one model at a
    time as the reference runs) on the batched workload: per step a bounded
    sample of models and particles on the host cores."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    from superlite_b200 import workloads as W
    b = W.analytic_batch(nmodel=a.nmodel, seed=SEED_BATCH)
    params = W.TransportParams()
    rates, tsteps = [], []
    for k in range(a.warmup + a.steps):
        t0 = time.perf_counter()
        r = batched_cpu_baseline(a, b, params, budget_s=6.0)
        if k >= a.warmup:
            rates.append(r["value"])
            tsteps.append(time.perf_counter() - t0)
    value = statistics.mean(rates)
    res = {"metric": METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": world, "steps": a.steps,
           "warmup": a.warmup, "ms_per_step": 1e3 * statistics.mean(tsteps), "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic (seeded generator, superlite_b200/workloads.py)", "config": batched_config(a, world, b),
           "impl": "reference",
           "cpu_baseline": {"value": value, "unit": "particle-steps/s", "cores": r["cores"], "kind": "port",
                            "sample": "per step: " + r["sample"]},
           "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(res))


def run_reference(a):
    """The reference's CPU path as restated by the oracle (the Fortran itself has
    no compiler here), on the host cores, same workload, bounded sample per step."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po
    from superlite_b200 import workloads as W
    case = make_case(a)
    params = W.TransportParams()
    cores = os.cpu_count() or 1
    npart = int(a.npart)
    sample = a.cpu_sample or 40000
    tinv = 1.0 / case.gas.temp
    rates, tsteps = [], []
    for k in range(a.warmup + a.steps):
        t0 = time.perf_counter()
        op = po.physical_opacity(case)
        grey = po.planckmean(case.groups.wlinv, case.gas.temp, op["cap"])
        po.rossmean(case.groups.wlinv, case.gas.temp, op["sig"], op["cap"])
        ol = po.leakage_opacity11(case.grid, case.groups.wlinv, tinv, op["sig"], op["cap"],
                                  tauddmc=params.tauddmc, taulump=params.taulump)
        ep = po.emission_probability(case.groups.wlinv, tinv, op["cap"], grey, case.groups.nep, case.groups.nepg)
        t_fixed = time.perf_counter() - t0
        prt, isv, _, _, _ = po.make_source_particles(case.grid, case.groups, case.gas.temp, L_BOL, sample,
                                                     ioffset=k)
        tt = po.TransportTables(case.grid, case.groups, tinv, op["sig"], op["cap"], grey, ep, ol, params)
        st = po.rnd_init(cores, k)
        t0 = time.perf_counter()
        po.sourcetally(prt, isv, case.grid, case.groups)
        r = po.particle_advance(tt, prt, isv, rngmode=0, nthreads=cores, rnd_states=st)
        po.fluxtally(prt, isv, case.groups.wl)
        dt = time.perf_counter() - t0
        scale = npart / sample
        t_step = t_fixed + dt * scale
        if k >= a.warmup:
            rates.append((r["nstepimc"] + r["nstepddmc"]) * scale / t_step)
            tsteps.append(t_step)
    value = statistics.mean(rates)
    res = {"metric": METRIC, "value": value, "unit": "particle-steps/s", "n_gpus": world, "steps": a.steps,
           "warmup": a.warmup, "ms_per_step": 1e3 * statistics.mean(tsteps), "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic (seeded generator, superlite_b200/workloads.py)", "config": config_dict(a, world),
           "impl": "reference",
           "cpu_baseline": {"value": value, "unit": "particle-steps/s", "cores": cores, "kind": "port",
                            "sample": f"per step: full opacity build + coefficients, transport of {sample} of "
                                      f"{npart} particles (mzran, OpenMP static,1), transport time scaled"},
           "e2e": {"value": value, "unit": "particle-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(res))


def run_opacity(a):
    """--workload opacity: the differentiable opacity build at the large
    scale (4096 shells x 10000 groups x 2e6 lines), forward and adjoint."""
    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    from superlite_b200 import peaks as PK
    pipes = PK.measure(local)
    r = opacity_measure(local, reps=a.steps, which=a.opacity_size, exp_per_s=pipes["fp64_exp_per_s"]["value"])
    res = {"metric": "opacity cell-group evals/s", "value": r["backward"]["cell_group_evals_per_s"],
           "unit": "cell-group evals/s", "n_gpus": 1, "steps": a.steps, "warmup": 3,
           "ms_per_step": r["forward"]["ms"] + r["backward"]["ms"], "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator, superlite_b200/workloads.py)",
           "config": {"workload": r["workload"]}, "opacity": r, "gpu_launches": None}
    if rank == 0:
        print(json.dumps(res))


def main():
    a = parse()
    if a.steps is None:
        a.steps = 1 if a.workload == "batched" else 3
    if a.impl == "reference":
        if a.workload == "batched":
            run_reference_batched(a)
        else:
            run_reference(a)
    elif a.workload == "batched":
        run_batched(a)
    elif a.workload == "opacity":
        run_opacity(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
