"""Benchmark of the B200 hourly land-surface step (IBIS 3.0 timestep_body).

Workload (one "step"): one day -- 24 hourly steps of timestep_body plus the
day-loop accumulators and hourly wetland CH4 -- on 95,333 independent columns
(the 0.5-degree land-cell count), FP32 structure-of-arrays state, seeded
synthetic forcing and columns (ibis_b200.synth).  Multi-GPU runs are weak
scaling: every rank advances its own 95,333 columns with no data-path
communication (a max-reduce of the timings is the only collective).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Rank 0 prints one JSON line.  ``--impl reference`` times the CPU oracle (the
reference's algorithm restated in NumPy, float64) on all host cores, because
the reference's own JAX step cannot run here (no jax/jaxlib/equinox).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import time
import warnings

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "cell-steps/s at 95,333 cells, ≤1e-4 rel err vs FP64; serve p50/p99 latency"
# What every CPU number of this file is
CPU_CAVEAT = ("the only CPU implementation of the step available here is the float64 NumPy restatement of the "
              "reference (the oracle): the reference's own JAX CPU path cannot be installed on this image (no jax, "
              "jaxlib or equinox), and no compiled CPU port was built, so GPU-to-CPU ratios against it overstate "
              "the speed-up over a compiled (XLA or C++) CPU path")
NCELL = 95333
HOURS = 24


def _peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _algorithmic_bytes(nhours):
    """Bytes one cell needs moved per launch of the hourly-step kernel (FP32):
    prognostic planes read and written, the static planes the step reads, the
    hourly forcing, and the enabled accumulators with their Kahan terms read
    and written."""
    from ibis_b200 import layout as L
    prog = 2 * L.N_PROG * 4
    # static planes the step reads: 10 soil fields x 6 layers, albedos/z0, canopy structure (8),
    # fu/fl, frac, exist/sapfrac/CH4 inputs, cbiow (10 used), cbior, root weights
    stat_planes = (10 * 6) + 3 + 8 + 2 + 12 + 3 + 10 + 12 + 3
    acc_planes = 24 + 1                                          # FLAG_ACC planes + CH4 value plane
    acc = 2 * 2 * acc_planes * 4
    return prog + stat_planes * 4 + acc + nhours * L.N_FORC * 4


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons sampled during a timed
    region: NVML read every 2 ms from a thread (reads only), with the
    nvidia-smi query as the fallback where NVML cannot be loaded."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.rows = []
        self.thread = None

    def _poll(self, nv, h, bits):
        while not self.stop.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.rows.append((float(sm), float(mx), [n for n, bit in zip(self.NAMES, bits) if r & bit]))
            except Exception:
                return
            self.stop.wait(0.002)

    def __enter__(self):
        import threading
        self.stop = threading.Event()
        try:
            import pynvml as nv
            nv.nvmlInit()
            h = nv.nvmlDeviceGetHandleByIndex(int(self.gpu))
            bits = (nv.nvmlClocksEventReasonHwSlowdown, nv.nvmlClocksEventReasonHwThermalSlowdown,
                    nv.nvmlClocksEventReasonSwThermalSlowdown, nv.nvmlClocksEventReasonSwPowerCap)
            self.thread = threading.Thread(target=self._poll, args=(nv, h, bits), daemon=True)
            self.thread.start()
            return self
        except Exception:
            self.thread = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.thread is not None:
            self.stop.set()
            self.thread.join(timeout=5)
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = list(self.rows)
        for line in (self.out or "").strip().splitlines():
            p = [x.strip() for x in line.split(",")]
            if len(p) >= 9 and p[1].replace(".", "").isdigit() and p[2].replace(".", "").isdigit():
                rows.append((float(p[1]), float(p[2]),
                             [n for i, n in enumerate(self.NAMES) if p[5 + i].lower().startswith("active")]))
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        return {"sm_mhz": float(np.median([r[0] for r in rows])), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": sorted({n for r in rows for n in r[2]}), "samples": len(rows),
                "source": "nvml" if self.rows else "nvidia-smi"}


def cpu_baseline_sample(ncell=16384, hours=HOURS, seed=123):
    """The float64 oracle on one host core over a bounded sample of the workload."""
    import oracle
    from ibis_b200 import synth
    wl = synth.make_workload(ncell, hours, seed=seed)
    prog = wl.prog
    acc = oracle.new_acc(ncell)
    t0 = time.perf_counter()
    with np.errstate(all="ignore"):
        for h in range(hours):
            prog, _, acc = oracle.step(prog, wl.stat, wl.forcing_at(h), wl.params, acc)
    dt = time.perf_counter() - t0
    return {"value": ncell * hours / dt, "unit": "cell-steps/s", "cores": 1, "kind": "port",
            "sample": f"{ncell} cells x {hours} hourly steps of the bench's seeded column generator, float64 NumPy "
                      f"oracle, "
                      f"{dt:.1f} s",
            "note": CPU_CAVEAT}


# ---------------------------------------------------------------------------- reference arm
def _oracle_chunk(args):
    prog, stat, forc, params, hours = args
    import oracle
    acc = oracle.new_acc(prog["tg"].shape[0])
    with np.errstate(all="ignore"):
        for h in range(hours):
            prog, _, acc = oracle.step(prog, stat, {k: v[h] for k, v in forc.items()}, params, acc)
    return prog["tg"].shape[0]


def run_reference(args):
    """The CPU oracle on all host cores (spawned process pool), same metric and config."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import multiprocessing as mp
    from ibis_b200 import synth
    warnings.filterwarnings("ignore")
    cores = os.cpu_count() or 1
    ncell = min(NCELL, 4000 * cores)
    wl = synth.make_workload(ncell, HOURS, seed=0)
    chunks = np.array_split(np.arange(ncell), cores)
    tasks = []
    for idx in chunks:
        if idx.size == 0:
            continue
        sl = lambda d: {k: v[idx] for k, v in d.items()}
        tasks.append((sl(wl.prog), sl(wl.stat), {k: v[:, idx] for k, v in wl.forc.items()}, wl.params, HOURS))
    ctx = mp.get_context("spawn")
    with ctx.Pool(processes=len(tasks)) as pool:
        for _ in range(args.warmup):
            pool.map(_oracle_chunk, [(t[0], t[1], {k: v[:1] for k, v in t[2].items()}, t[3], 1) for t in tasks])
        times = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            pool.map(_oracle_chunk, tasks)
            times.append(time.perf_counter() - t0)
    ms = 1e3 * float(np.mean(times))
    v = ncell * HOURS / (ms / 1e3)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "cell-steps/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"{ncell} of 95,333 cells x 24 hourly steps per step (bounded sample), "
                                   "float64 NumPy restatement of the reference step", "ncell": ncell,
                       "hours_per_step": HOURS},
            "cpu_baseline": {"value": v, "unit": "cell-steps/s", "cores": len(tasks), "kind": "port",
                             "sample": f"{ncell} cells x {HOURS} h per step over {len(tasks)} spawned processes"},
            "e2e": {"value": v, "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": CPU_CAVEAT}
    print(json.dumps(line), flush=True)



# ---------------------------------------------------------------------------- sub-workloads of the default line
def _release_params():
    """The step's parameter record under the reference's release parameter file
    (python-port/configs/params/params_31s_ch4h.yaml: sunlit/shaded canopies,
    vmax and slope mixing, the NPP split by capacity, temperature acclimation
    with per-PFT constants, consistent soil-water weights, its respiration and
    methane values), as the release fixture holds it (tests/golden/release.npz,
    made by the reference's own loaders)."""
    from ibis_b200.params import PARAM_FIELDS, StepParams
    z = np.load(os.path.join(REPO, "tests", "golden", "release.npz"))
    P = StepParams()
    for name, _, _ in PARAM_FIELDS:
        if "in.param." + name in z.files:
            setattr(P, name, z["in.param." + name])
    P.flags = int(z["in.param.flags"])
    return P


def release_day(wl, dev, stream, flush, steps):
    """The day workload (95,333 columns x 24 h, accumulators + hourly CH4) under
    the release parameter file's switches: the IBIS 3.0 kernels, long fused
    configuration."""
    import torch
    from ibis_b200.columns import Columns
    P = _release_params()
    rng = np.random.Generator(np.random.PCG64(41))
    stat = dict(wl.stat, acclim_x=rng.uniform(-12.0, 28.0, wl.ncell))
    cols = Columns.from_host(wl.prog, stat, dtype=torch.float32, device=dev, acc=True)
    cols.set_mode(6)
    forc = cols.forcing(wl.forc)
    prog0, acc0 = cols.prog.clone(), cols.acc.clone()
    for _ in range(3):
        cols.run(forc, P, stream=stream)
    out = []
    for _ in range(steps):
        cols.prog.copy_(prog0)
        cols.acc.copy_(acc0)
        flush.fill_(1.0)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        cols.run(forc, P, stream=stream)
        b.record(stream)
        out.append((a, b))
    torch.cuda.synchronize(dev)
    ms = float(np.mean([a.elapsed_time(b) for a, b in out]))
    from ibis_b200.params import X3_FLAGS
    names = {1 << 2: "sunshade_u", 1 << 3: "sunshade_l", 1 << 1: "h2o_consistent_weights", 1 << 12: "vmax_mix",
             1 << 13: "coefm_mix", 1 << 14: "gpp_split_by_capacity", 1 << 15: "acclim_on (per-PFT constants)",
             1 << 10: "ET parts"}
    return {"value": wl.ncell * HOURS / (ms / 1e3), "unit": "cell-steps/s", "ms_per_step": ms,
            "switches": [v for k, v in names.items() if P.flags & k], "x3_kernels": bool(P.flags & X3_FLAGS),
            "nonfinite_columns": cols.nonfinite()[0],
            "note": "the same day under the reference's release parameter file "
                    "(configs/params/params_31s_ch4h.yaml, as captured by tests/golden/release.npz); per-cell "
                    "acclimation states seeded U(-12, 28) C"}


def ensemble_bounded(stream, hours=48):
    """The 356-site x 64-vector calibration ensemble (22,784 runs) over the first
    ``hours`` hours of every record: the persistent launch, the batched hourly
    form (one launch per hour for all runs, replayed from a CUDA graph) and the
    per-vector plain form (one single-parameter launch per hour per vector); and
    the full records' makespan estimated from the persistent hour."""
    import torch
    from ibis_b200 import ensemble as E
    spec = E.make_ensemble(356, 64, years=(1, 15), seed=7, site_hours=np.full(356, hours))
    ens = E.Ensemble(spec)

    def timed(fn, k):
        out = []
        for _ in range(k):
            ens.reset()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            b.synchronize()
            out.append(a.elapsed_time(b))
        return out

    timed(ens.run, 2)
    ms_p = float(np.median(timed(ens.run, 3)))
    timed(lambda: ens.run_hourly(chunk=24, graph=True), 1)
    ms_g = float(np.median(timed(lambda: ens.run_hourly(chunk=24, graph=True), 3)))
    plain = _plain_per_vector(spec, None, stream, hours=hours)
    cs = ens.cell_steps()
    longest = 15 * 8760
    return {"hours": hours, "runs": ens.nrun, "cell_steps": cs,
            "persistent": {"value": cs / (ms_p / 1e3), "ms": ms_p, "launches": 1},
            "hourly_graph": {"value": cs / (ms_g / 1e3), "ms": ms_g, "launches": hours},
            "plain_per_vector": {"value": plain["value"], "ms": plain["ms"], "launches": plain["launches"]},
            "persistent_vs_hourly_graph": ms_g / ms_p, "persistent_vs_plain_per_vector": plain["ms"] / ms_p,
            "full_record_makespan_estimate_s": ms_p / hours * longest / 1e3,
            "note": f"first {hours} h of every run; the full records (1-15 years) take about the persistent "
                    "hour's time x the longest record (131,400 h): one thread's per-hour latency bounds the "
                    "makespan"}


def serve_bounded(rate=50.0, duration=2.0):
    """The request loop over a library of day records (356 sites, 10 years):
    Poisson arrivals at ``rate``/s for ``duration`` s, 1-64 sites, 1-10 years,
    continuously batched; p50/p99 request latency and throughput."""
    from ibis_b200 import serve as S
    lib = S.SiteLibrary(356, 10, seed=3, daily=True)
    srv = S.Server(lib, budget_bytes=150e9, epoch_hours=168)
    srv.serve(S.poisson_requests(np.random.default_rng(1), rate, 0.2, 356, max_years=1))
    st = srv.serve(S.poisson_requests(np.random.default_rng(5), rate, duration, 356))
    return {"requests": st["requests"], "p50_s": st["p50_s"], "p99_s": st["p99_s"],
            "cell_steps_per_s": st["cell_steps_per_s"], "epochs": st["epochs"], "slots": st["slots"],
            "queue_depth_max": st["queue_depth_max"], "hbm_gb": st["hbm_gb"], "status": st["status"],
            "note": f"Poisson {rate}/s for {duration} s, day-record library (hours generated in the kernel); "
                    "latency from arrival to the result in host memory, GPU clock"}


def day_loop_bounded(dev, stream, ncell=95333, nday=3, reps=3):
    """The day loop over ``nday`` days of the day workload's size: per day the
    daily cadence, 24 hours of forcing generated on the GPU from the day's
    weather and 24 hourly steps with accumulators and hourly CH4, then the
    wetland methane of the period (DayLoop.run_month); the daily weather
    resident on the device, the state reset before each timed period."""
    import torch
    from ibis_b200 import forcing as _forcing
    from ibis_b200 import synth
    from ibis_b200.columns import Columns
    from ibis_b200.daily import DayLoop
    from ibis_b200.params import FLAG_CH4, DayParams
    wl = synth.make_workload(ncell, 1, seed=11)
    rng = np.random.Generator(np.random.PCG64(12))
    dayst = synth.make_dayst(rng, wl.stat, wl.latitude)
    cols = Columns.from_host(wl.prog, wl.stat, dtype=torch.float32, device=dev, acc=True)
    P = wl.params.copy()
    P.flags |= FLAG_CH4
    loop = DayLoop(cols, P, DayParams(), dayst, lat=wl.latitude, seed=5, jday=152, day=0)
    d_daily = torch.from_numpy(_forcing.daily_planes(synth.make_daily_weather(rng, wl.latitude, nday),
                                                     cols.ld)).to(dev)
    prog0, stat0, acc0, dayst0 = cols.prog.clone(), cols.stat.clone(), cols.acc.clone(), loop.dayst.clone()
    out = []
    for r in range(reps + 1):
        cols.prog.copy_(prog0); cols.stat.copy_(stat0); cols.acc.copy_(acc0); loop.dayst.copy_(dayst0)
        loop.wet.zero_()
        loop.jday, loop.day = 152, 0
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        loop.run_month(d_daily, from_mean=True, new_year=False, stream=stream)
        b.record(stream)
        b.synchronize()
        if r:                                   # the first period warms up
            out.append(a.elapsed_time(b))
    ms = float(np.median(out))
    return {"value": ncell * 24 * nday / (ms / 1e3), "unit": "cell-steps/s", "ms_per_period": ms,
            "ms_per_day": ms / nday, "days": nday, "cells": ncell, "nonfinite_columns": cols.nonfinite()[0],
            "note": f"the day loop over {nday} days (--workload month runs 30): per day the daily cadence, the "
                    "day's hourly forcing generated on the GPU and 24 hourly steps, then the period's wetland "
                    "methane; median of {reps} after one warm-up".replace("{reps}", str(reps))}


def single_cell(dev, stream, cpu_hours=480):
    """configs[0]'s shape: one column x 8,760 hourly steps, the whole year in one
    fused launch on the GPU (FP32 and FP64), beside the float64 oracle on one
    host core over a bounded sample of the same year."""
    import torch
    import oracle
    from ibis_b200 import synth
    from ibis_b200.columns import Columns
    wl = synth.make_workload(1, 8760, seed=17)
    out = {}
    for name, dt in (("f32", torch.float32), ("f64", torch.float64)):
        cols = Columns.from_host(wl.prog, wl.stat, dtype=dt, device=dev, acc=True)
        forc = cols.forcing(wl.forc)
        P = wl.params.copy()
        if dt == torch.float64:
            P.flags &= ~(1 << 8)
        cols.run(forc[:24], P, stream=stream)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        cols.run(forc, P, stream=stream)
        b.record(stream)
        b.synchronize()
        ms = a.elapsed_time(b)
        out["gpu_" + name] = {"ms_per_year": ms, "value": 8760 / (ms / 1e3), "unit": "cell-steps/s"}
    prog, acc = wl.prog, oracle.new_acc(1)
    t0 = time.perf_counter()
    with np.errstate(all="ignore"):
        for h in range(cpu_hours):
            prog, _, acc = oracle.step(prog, wl.stat, wl.forcing_at(h), wl.params, acc)
    dt = time.perf_counter() - t0
    out["cpu_f64_oracle"] = {"value": cpu_hours / dt, "unit": "cell-steps/s", "cores": 1,
                             "year_estimate_s": dt / cpu_hours * 8760,
                             "sample": f"first {cpu_hours} hours of the year, float64 NumPy oracle",
                             "note": CPU_CAVEAT}
    out["note"] = ("1 column x 8,760 h: the GPU runs one thread through the year (latency bound); the reference's "
                   "JAX CPU path is not installable here, so the CPU leg is the float64 NumPy port on one core")
    return out

# ---------------------------------------------------------------------------- our arm
def run_ours(args):
    import torch
    import torch.distributed as dist
    from ibis_b200 import synth
    from ibis_b200.columns import Columns

    from ibis_b200 import replicas
    W = replicas.world_from_env()
    world, rank, local = W.size, W.rank, W.local
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    replicas.init(W, "nccl", device=dev)

    def barrier():
        replicas.barrier(W)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_sample()

    wl = synth.make_workload(args.ncell, HOURS, seed=replicas.replica_seed(1000, rank))
    P = wl.params
    cols = Columns.from_host(wl.prog, wl.stat, dtype=torch.float32, device=dev, acc=True)
    forc = cols.forcing(wl.forc)
    from ibis_b200 import tune as _tune
    tuned = _tune.tune(cols, forc, P, reps=2) if args.config is None else None
    if args.config is not None:
        cols.set_mode(args.config)
    from ibis_b200 import lib as _ilib
    cfg_desc = next(c for c in _ilib.configs() if c["id"] == cols.config)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)

    def day():
        cols.run(forc, P, stream=stream)

    plain = Columns.from_host(wl.prog, wl.stat, dtype=torch.float32, device=dev, acc=True)

    def day_plain():
        # the plain per-step launch: one default fused launch per hour
        for h in range(HOURS):
            plain.run(forc[h:h + 1], P, stream=stream)

    def timed(fn, k):
        evs = []
        for _ in range(k):
            flush.fill_(1.0)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            evs.append((a, b))
        torch.cuda.synchronize(dev)
        return [a.elapsed_time(b) for a, b in evs]

    with ClockSampler(local) as clk:
        for _ in range(args.warmup):
            day()
            day_plain()
        torch.cuda.synchronize(dev)
        barrier()
        torch.cuda.synchronize(dev)
        ms = timed(day, args.steps)
        barrier()
        torch.cuda.synchronize(dev)
    ms_step = float(np.sum(ms)) / args.steps
    ms_plain = float(np.sum(timed(day_plain, args.steps))) / args.steps

    # end to end through the public API: pinned host forcing in, host state out, copies timed
    h_forc = torch.from_numpy(synth.forcing_planes(wl.forc, cols.ld)).pin_memory()
    h_prog = torch.empty_like(cols.prog, device="cpu").pin_memory()

    def e2e_day():
        # the public host-buffer entry (ibis_step_host_f32): the columns in
        # groups, each group's forcing copied in, stepped and its state copied
        # out on the library's streams, overlapping the other groups' hours
        cols.run_host(h_forc, P, host_prog=h_prog, group=args.e2e_group, stream=stream)

    def e2e_hour_chunks():
        # the same through run_from_host: forcing copied in chunks of hours on a
        # second stream, overlapping the computation of the previous chunk
        cols.run_from_host(h_forc, P, chunk=args.e2e_chunk if args.e2e_chunk == "auto" else int(args.e2e_chunk),
                           stream=stream)
        h_prog.copy_(cols.prog, non_blocking=True)

    e2e_day()
    ms_e2e = float(np.sum(timed(e2e_day, args.steps))) / args.steps
    e2e_hour_chunks()
    ms_e2e_chunks = float(np.sum(timed(e2e_hour_chunks, args.steps))) / args.steps

    # end to end from daily weather: 32 B per cell-day in, the hourly forcing
    # generated on the GPU (ibis_diurnal_f32, the reference's diurnal algorithm)
    from ibis_b200 import forcing as _forcing
    rng = np.random.default_rng(77)
    n = args.ncell
    tmin = rng.uniform(255.0, 295.0, n)
    daily = {"tmin": tmin[None], "tmax": (tmin + rng.uniform(3.0, 14.0, n))[None],
             "cloud": rng.uniform(0.0, 1.0, n)[None], "precip": np.where(rng.uniform(size=n) < 0.6, 0.0,
                                                                       rng.gamma(0.8, 6.0, n))[None],
             "psurf": np.full((1, n), 101300.0), "qd": rng.uniform(0.002, 0.015, n)[None],
             "ud": rng.uniform(1.0, 6.0, n)[None], "fira": np.zeros((1, n))}
    h_daily = torch.from_numpy(_forcing.daily_planes(daily, cols.ld)).pin_memory()
    d_daily = torch.empty_like(h_daily, device=dev)
    lat_d = torch.zeros(cols.ld, dtype=torch.float32, device=dev)
    lat_d[:n] = torch.from_numpy(wl.latitude.astype(np.float32)).to(dev)
    gen_out = torch.empty_like(forc)

    def e2e_daily_day():
        # ibis_day_host_f32: per group of columns the daily weather in, the
        # hourly forcing generated, the day stepped and the state out
        cols.run_host_daily(h_daily, lat_d, P, 172, seed=5, host_prog=h_prog, stream=stream)

    e2e_daily_day()
    ms_e2e_daily = float(np.sum(timed(e2e_daily_day, args.steps))) / args.steps
    ms_gen = float(np.median(timed(lambda: _forcing.hourly_forcing(d_daily, lat_d, n, jday0=172, seed=5, out=gen_out,
                                                                   stream=stream), 5)))

    nonfinite = cols.nonfinite()
    # the sub-workloads of the default line (one GPU only: the scaling runs time the day alone)
    extras = {}
    if world == 1 and not args.no_extras:
        extras["release_params"] = release_day(wl, dev, stream, flush, args.steps)
        extras["ensemble"] = ensemble_bounded(stream)
        extras["serve"] = serve_bounded()
        extras["day_loop"] = day_loop_bounded(dev, stream)
        extras["single_cell"] = single_cell(dev, stream)
    if world > 1:
        ms_step, ms_plain, ms_e2e, ms_e2e_daily, ms_e2e_chunks = replicas.max_over_ranks(
            W, [ms_step, ms_plain, ms_e2e, ms_e2e_daily, ms_e2e_chunks], device=dev)
    cell_steps = world * args.ncell * HOURS
    value = cell_steps / (ms_step / 1e3)
    peak, peak_kind = _peaks()
    bpl = _algorithmic_bytes(HOURS) * args.ncell
    achieved = bpl / (ms_step / 1e3) / 1e9
    traffic = None
    issue = None
    tpath = os.path.join(REPO, "profiles", "hourly_step_traffic.json")
    clocks = clk.summary()
    if os.path.exists(tpath):
        with open(tpath) as f:
            tj = json.load(f)
        per_cell = tj.get("fused_day_bytes_per_cell")
        if per_cell:
            traffic = float(per_cell) * args.ncell
        ipc = tj.get("fused_day_warp_instructions_per_cell_hour")
        if ipc and clocks.get("sm_mhz"):
            # the bound that applies: warp-instruction issue, 4 schedulers per SM each
            # issuing one warp instruction per cycle at the sampled SM clock
            n_sm = torch.cuda.get_device_properties(dev).multi_processor_count
            winst = float(ipc) * args.ncell * HOURS
            ach = winst / (ms_step / 1e3) / 1e9
            pk = n_sm * 4 * clocks["sm_mhz"] * 1e6 / 1e9
            issue = {"bound": "issue", "achieved": ach, "peak": pk, "unit": "G warp-instructions/s",
                     "frac": ach / pk, "warp_instructions_per_launch": winst,
                     "source": "instructions per cell-hour from profiles/hourly_step_kernel_f32_day_32768cells.md; "
                               f"peak = {n_sm} SMs x 4 schedulers x median sampled SM clock"}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "cell-steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"{args.ncell} cells x 24 hourly steps (one day) per step, FP32 SoA state, "
                                   "accumulators + hourly CH4 on, one fused launch per day",
                       "ncell_per_gpu": args.ncell, "hours_per_step": HOURS,
                       "l2": "flushed between timed steps (256 MiB write, outside the events)",
                       "parallelism": f"replicas x{world} (independent columns, no collectives)",
                       "launch_config": cfg_desc,
                       "tuned_ms": ({str(k): round(v, 4) for k, v in tuned["ms"].items()} if tuned else None)},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "peak_source": peak_kind, "algorithmic_bytes_per_launch": bpl},
            "issue_roofline": issue,
            "per_step_launch": {"value": cell_steps / (ms_plain / 1e3), "ms_per_step": ms_plain,
                                "launches_per_step": HOURS, "launch_config": "fused, block 128, 2 blocks/SM",
                                "achieved_gbs": _algorithmic_bytes(1) * args.ncell * HOURS / (ms_plain / 1e3) / 1e9},
            "e2e": {"value": cell_steps / (ms_e2e / 1e3), "unit": "cell-steps/s", "ms_per_step": ms_e2e,
                    "entry": "Columns.run_host -> ibis_step_host_f32",
                    "group_cells": args.e2e_group or "auto (a sixteenth of the columns in whole blocks; chunks of "
                                                     "hours up to 1.15 waves)",
                    "h2d_bytes_per_step": int(h_forc.numel() * 4), "d2h_bytes_per_step": int(h_prog.numel() * 4)},
            "e2e_hour_chunks": {"value": cell_steps / (ms_e2e_chunks / 1e3), "unit": "cell-steps/s",
                                "ms_per_step": ms_e2e_chunks, "entry": "Columns.run_from_host + a state read-back",
                                "chunk_hours": Columns.chunk_schedule(HOURS, args.e2e_chunk if args.e2e_chunk == "auto"
                                                                      else int(args.e2e_chunk))},
            "e2e_daily_forcing": {"value": cell_steps / (ms_e2e_daily / 1e3), "unit": "cell-steps/s",
                                  "h2d_bytes_per_step": int(h_daily.numel() * 4),
                                  "d2h_bytes_per_step": int(h_prog.numel() * 4),
                                  "forcing_generation_ms": ms_gen,
                                  "entry": "Columns.run_host_daily -> ibis_day_host_f32",
                                  "note": "daily weather in, hourly forcing generated on the GPU by the reference's "
                                          "diurnal algorithm (not the hourly generator of the workload above)"},
            "gpu_launches": args.steps * (1 if cfg_desc["form"] == "fused" else 2 * HOURS),
            "clocks": clocks,
            "nonfinite_columns": nonfinite[0],
        }
        line.update(extras)
        if cpu is not None:
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)
    replicas.finish(W)


def _plain_per_vector(spec, args, stream, hours=48):
    """The ensemble through the single-parameter step API as a caller without
    the ensemble kernels would drive it: per parameter vector one set of
    columns (the 356 sites), one ``ibis_step`` launch per hour per vector.
    Timed over the first ``hours`` hours of every record, beside the persistent
    launch on the same truncated records (the full records would take minutes
    in this form)."""
    import torch
    from ibis_b200 import ensemble as E
    from ibis_b200 import layout as L
    from ibis_b200 import synth
    from ibis_b200.columns import Columns

    nsite, nvec = spec.nsite, spec.nparam
    short = E.EnsembleSpec(nsite=nsite, nparam=nvec, site_hours=np.minimum(spec.site_hours, hours), stat=spec.stat,
                           prog=spec.prog, forc=spec.forc, site_first=spec.site_first, vectors=spec.vectors,
                           params=spec.params, latitude=spec.latitude)
    ens = E.Ensemble(short)
    cols = [Columns.from_host(spec.prog, spec.stat, dtype=torch.float32, acc=True) for _ in range(nvec)]
    for c in cols:
        c.set_mode(0)
    params = [E.apply_vector(spec.params, v) for v in spec.vectors]
    ld = cols[0].ld
    fp = np.zeros((hours, L.N_FORC, ld), dtype=np.float32)
    for s_ in range(nsite):
        fp[:, :, s_] = spec.forc[spec.site_first[s_]:spec.site_first[s_] + hours]
    forc = torch.from_numpy(fp).cuda()

    def plain_run():
        for h in range(hours):
            for c, P in zip(cols, params):
                c.run(forc[h:h + 1], P, stream=stream)

    def timed(fn, reset):
        reset()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        b.synchronize()
        return a.elapsed_time(b)

    state0 = [c.prog.clone() for c in cols]

    def reset_plain():
        for c, p0 in zip(cols, state0):
            c.prog.copy_(p0)
            c.acc.zero_()

    timed(plain_run, reset_plain)
    ms_plain = min(timed(plain_run, reset_plain) for _ in range(2))
    timed(ens.run, ens.reset)
    ms_pers = min(timed(ens.run, ens.reset) for _ in range(2))
    cs = nsite * nvec * hours
    return {"hours": hours, "launches": hours * nvec, "ms": ms_plain, "value": cs / (ms_plain / 1e3),
            "persistent_ms_same_records": ms_pers, "persistent_value_same_records": cs / (ms_pers / 1e3),
            "persistent_vs_plain": ms_plain / ms_pers,
            "note": "one single-parameter step launch per hour per parameter vector (ibis_step_config_f32, "
                    "config 0), first 48 hours of every record"}


def run_ensemble(args):
    """The calibration ensemble: 356 sites x 64 parameter vectors (22,784 runs),
    records of U{1..15} years, one step = every run over its whole record.  The
    persistent launch is timed; the same runs with one launch per hour (eager and
    replayed from a CUDA graph) are timed beside it."""
    import torch
    from ibis_b200 import ensemble as E
    from ibis_b200 import synth

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    t0 = time.time()
    hours = None if args.record_hours is None else np.full(args.sites, args.record_hours)
    spec = E.make_ensemble(args.sites, args.params_per_site, years=(1, 15), seed=7, site_hours=hours)
    gen_s = time.time() - t0
    ens = E.Ensemble(spec)
    stream = torch.cuda.current_stream()
    tuned = ens.tune(blocks=[96, 128, 160, 192, 256]) if args.tune else None
    block = tuned["best"] if tuned else 0

    def timed(fn, k):
        out = []
        for _ in range(k):
            ens.reset()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            b.synchronize()
            out.append(a.elapsed_time(b))
        return out

    with ClockSampler(local) as clk:
        timed(lambda: ens.run(block=block), args.warmup)
        ms = timed(lambda: ens.run(block=block), args.steps)
    nonfinite = ens.nonfinite()
    ms_graph = timed(lambda: ens.run_hourly(chunk=24, graph=True), 1 + args.steps)[1:]
    ms_eager = timed(lambda: ens.run_hourly(chunk=24, graph=False), args.steps)
    cs = ens.cell_steps()
    m = float(np.mean(ms))
    plain = _plain_per_vector(spec, args, stream)
    # the daily-weather form: the same sites, vectors and record lengths over
    # day records, each run generating its hours in the kernel
    t0 = time.time()
    spec_d = E.make_ensemble(args.sites, args.params_per_site, seed=7, site_hours=spec.site_hours, daily=True)
    gen_d = time.time() - t0
    ens_d = E.Ensemble(spec_d)

    def timed_d(k):
        out = []
        for _ in range(k):
            ens_d.reset()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            ens_d.run(block=block)
            b.record(stream)
            b.synchronize()
            out.append(a.elapsed_time(b))
        return out

    timed_d(1)
    ms_d = float(np.mean(timed_d(args.steps)))
    daily_form = {"value": ens_d.cell_steps() / (ms_d / 1e3), "ms_per_step": ms_d,
                  "forcing_gb": ens_d.day_records.numel() * 4 / 1e9, "generation_s": gen_d,
                  "nonfinite_runs": ens_d.nonfinite()[0],
                  "note": "same sites, vectors and record lengths over 48-byte day records; each run generates its "
                          "hours in the kernel (ibis_ensemble_daily_f32)"}
    del ens_d
    # calibration runs with the daily cadence: 30 days of every run, one
    # persistent launch per day between the day kernels (EnsembleDayLoop)
    from ibis_b200.ensemble_daily import EnsembleDayLoop
    rng_d = np.random.Generator(np.random.PCG64(8))
    ndl = 30
    edl_args = (spec.stat, spec.prog, synth.make_dayst(rng_d, spec.stat, spec.latitude),
                synth.make_daily_weather(rng_d, spec.latitude, ndl), spec.latitude, spec.vectors, spec.params)
    EnsembleDayLoop(*edl_args, seed=5, jday=150).run(3)
    torch.cuda.synchronize()
    edl = EnsembleDayLoop(*edl_args, seed=5, jday=150)
    a_ev, b_ev = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a_ev.record(stream)
    edl.run()
    b_ev.record(stream)
    b_ev.synchronize()
    ms_dl = a_ev.elapsed_time(b_ev)
    day_loop = {"value": edl.cell_steps() / (ms_dl / 1e3), "ms": ms_dl, "days": ndl, "runs": edl.nrun,
                "ms_per_day": ms_dl / ndl, "nonfinite_runs": edl.nonfinite()[0],
                "note": "every run with the daily cadence (per-run canopy structure and carbon pools): per day the "
                        "sites' forcing generated, day_begin, one persistent launch of 24 hours, day_end"}
    del edl
    line = {
        "metric": "cell-steps/s, calibration ensemble (persistent launch)", "value": cs / (m / 1e3),
        "unit": "cell-steps/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": m,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"{args.sites} sites x {args.params_per_site} parameter vectors = {ens.nrun} runs, "
                               + ("records U{1..15} years of hourly forcing" if hours is None
                                  else f"records of {args.record_hours} hours")
                               + ", one step = every run to the end of its record",
                   "cell_steps_per_step": cs, "longest_record_hours": int(ens.run_nstep_host.max()),
                   "block": block or "auto", "tuned_ms": tuned["ms"] if tuned else None,
                   "forcing_gb": ens.forc.numel() * 4 / 1e9, "generation_s": gen_s,
                   "l2": "inputs (1.2 GB of forcing records) larger than L2"},
        "hourly_graph": {"value": cs / (float(np.mean(ms_graph)) / 1e3), "ms_per_step": float(np.mean(ms_graph)),
                         "launches_per_step": int(ens.run_nstep_host.max()),
                         "note": "one launch per hour, 24-hour CUDA graph replayed"},
        "hourly_eager": {"value": cs / (float(np.mean(ms_eager)) / 1e3), "ms_per_step": float(np.mean(ms_eager))},
        "persistent_vs_hourly_graph": float(np.mean(ms_graph)) / m,
        "plain_per_vector": plain,
        "daily_form": daily_form,
        "day_loop": day_loop,
        "gpu_launches": args.steps,
        "clocks": clk.summary(), "nonfinite_runs": nonfinite[0], "bad_descriptors": nonfinite[1],
    }
    print(json.dumps(line), flush=True)


def run_serve(args):
    """The request loop: Poisson arrivals (50/s by default) of requests for
    U{1..64} of 356 resident tower sites, U{1..10} years, one calibration vector
    each, continuously batched into the resident ensemble; p50/p99 latency."""
    import torch
    from ibis_b200 import serve as S

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    t0 = time.time()
    lib = S.SiteLibrary(args.sites, 10, seed=3)
    gen_s = time.time() - t0
    srv = S.Server(lib, budget_bytes=150e9, epoch_hours=args.epoch_hours)
    srv.serve(S.poisson_requests(np.random.default_rng(1), args.rate, 0.2, args.sites, max_years=1))
    reqs = S.poisson_requests(np.random.default_rng(5), args.rate, args.duration, args.sites)
    with ClockSampler(local) as clk:
        st = srv.serve(reqs)
    # the plain per-request form on the first 0.3 s of a Poisson stream, beside
    # the continuous-batching server on the same requests
    few = S.poisson_requests(np.random.default_rng(7), args.rate, 0.3, args.sites)
    st_few = srv.serve(few)
    pl = S.serve_plain(lib, few)
    plain = {"requests": pl["requests"], "p50_s": pl["p50_s"], "p99_s": pl["p99_s"],
             "batched_p50_s": st_few["p50_s"], "batched_p99_s": st_few["p99_s"],
             "note": "the first 0.3 s of a Poisson stream: one persistent launch per request, one request at a "
                     "time (plain) vs the continuous-batching server"}
    # the same requests over a library of day records (hours generated in the kernel)
    t0 = time.time()
    lib_d = S.SiteLibrary(args.sites, 10, seed=3, daily=True)
    gen_d = time.time() - t0
    srv_d = S.Server(lib_d, budget_bytes=150e9, epoch_hours=args.epoch_hours)
    srv_d.serve(S.poisson_requests(np.random.default_rng(1), args.rate, 0.2, args.sites, max_years=1))
    st_d = srv_d.serve(reqs)
    daily_library = {"p50_s": st_d["p50_s"], "p99_s": st_d["p99_s"], "cell_steps_per_s": st_d["cell_steps_per_s"],
                     "library_gb": lib_d.nbytes / 1e9, "library_generation_s": gen_d, "status": st_d["status"],
                     "note": "the same requests over 48-byte day records per site-day (ibis_ensemble_daily_f32)"}
    del srv_d, lib_d
    line = {
        "metric": "serve p50/p99 request latency", "value": st["p50_s"], "unit": "s", "p99_s": st["p99_s"],
        "n_gpus": 1, "steps": st["requests"], "warmup": 1, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "throughput": {"value": st["cell_steps_per_s"], "unit": "cell-steps/s", "cell_steps": st["cell_steps"]},
        "config": {"workload": f"Poisson {args.rate}/s requests for {args.duration} s, 1-64 of {args.sites} sites, "
                               "1-10 years, one 31-value vector each", "epoch_hours": st["epoch_hours"],
                   "slots": st["slots"], "budget_gb": 150, "library_gb": lib.nbytes / 1e9,
                   "library_generation_s": gen_s},
        "epochs": st["epochs"], "gpu_launches": st["epochs"], "clocks": clk.summary(), "status": st["status"],
        "daily_library": daily_library, "plain_per_request": plain,
        "queue_depth": {"max": st["queue_depth_max"], "mean": st["queue_depth_mean"]},
        "hbm_gb": st["hbm_gb"],
    }
    print(json.dumps(line), flush=True)


def run_month(args):
    """The day loop over a month: 95,333 columns x 30 days, each day the
    daily cadence (phenology, daily sums / 10-day means, decomposition, soil
    C/N), 24 hours of forcing generated on the GPU from the day's weather and
    24 hourly steps with accumulators and hourly CH4, then the month's wetland
    methane (DayLoop.run_month).  One step = one month; the daily weather is
    resident on the device.  e2e: the month's daily weather copied in from
    pinned host memory and the prognostic, daily-cadence and wetland state read
    back, inside the timed region."""
    import torch
    from ibis_b200 import forcing as _forcing
    from ibis_b200 import synth
    from ibis_b200.columns import Columns
    from ibis_b200.daily import DayLoop
    from ibis_b200.params import FLAG_CH4, DayParams

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    nday = args.days
    wl = synth.make_workload(args.ncell, 1, seed=11)
    rng = np.random.Generator(np.random.PCG64(12))
    dayst = synth.make_dayst(rng, wl.stat, wl.latitude)
    cols = Columns.from_host(wl.prog, wl.stat, dtype=torch.float32, device=dev, acc=True)
    if args.config is not None:
        cols.set_mode(args.config)
    P = wl.params.copy()
    P.flags |= FLAG_CH4
    loop = DayLoop(cols, P, DayParams(), dayst, lat=wl.latitude, seed=5, jday=152, day=0)
    h_daily = torch.from_numpy(_forcing.daily_planes(synth.make_daily_weather(rng, wl.latitude, nday),
                                                     cols.ld)).pin_memory()
    d_daily = h_daily.to(dev)
    prog0, stat0, acc0, dayst0 = cols.prog.clone(), cols.stat.clone(), cols.acc.clone(), loop.dayst.clone()
    tuned = None
    if args.config is None:
        from ibis_b200 import tune as _tune
        f0 = _forcing.hourly_forcing(d_daily[:1].contiguous(), loop.lat, cols.ncell, jday0=152, seed=5,
                                     observed_fira=True)
        tuned = _tune.tune(cols, f0, P, reps=2)
        del f0
    stream = torch.cuda.current_stream(dev)
    h_prog = torch.empty_like(cols.prog, device="cpu").pin_memory()
    h_dayst = torch.empty_like(loop.dayst, device="cpu").pin_memory()
    h_wet = torch.empty_like(loop.wet, device="cpu").pin_memory()

    def reset():
        cols.prog.copy_(prog0); cols.stat.copy_(stat0); cols.acc.copy_(acc0); loop.dayst.copy_(dayst0)
        loop.wet.zero_()
        loop.jday, loop.day = 152, 0

    def month():
        loop.run_month(d_daily, from_mean=True, new_year=False, stream=stream)

    def month_e2e():
        d_daily.copy_(h_daily, non_blocking=True)
        loop.run_month(d_daily, from_mean=True, new_year=False, stream=stream)
        h_prog.copy_(cols.prog, non_blocking=True)
        h_dayst.copy_(loop.dayst, non_blocking=True)
        h_wet.copy_(loop.wet, non_blocking=True)

    def timed(fn, k):
        out = []
        for _ in range(k):
            reset()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            b.synchronize()
            out.append(a.elapsed_time(b))
        return out

    with ClockSampler(local) as clk:
        timed(month, args.warmup)
        ms = timed(month, args.steps)
    ms_e2e = timed(month_e2e, args.steps)
    nonfinite = cols.nonfinite()

    # where the month's time goes: each launch kind timed on its own over one month
    reset()
    parts = {"hourly_step": [], "forcing": [], "day_begin": [], "day_end": []}
    ev = lambda: torch.cuda.Event(enable_timing=True)
    for d in range(nday):
        daily = d_daily[d]
        marks = [ev() for _ in range(5)]
        marks[0].record(stream)
        loop._td.copy_(daily[0])
        loop.begin(loop._td, stream)
        marks[1].record(stream)
        _forcing.hourly_forcing(daily[None], loop.lat, cols.ncell, jday0=loop.jday, day0=loop.day, seed=loop.seed,
                                observed_fira=True, out=loop._forc if loop._forc is not None else None,
                                stream=stream)
        marks[2].record(stream)
        cols.run(loop._forc, loop.params, stream=stream)
        marks[3].record(stream)
        loop.end(loop._td, stream)
        marks[4].record(stream)
        marks[4].synchronize()
        parts["day_begin"].append(marks[0].elapsed_time(marks[1]))
        parts["forcing"].append(marks[1].elapsed_time(marks[2]))
        parts["hourly_step"].append(marks[2].elapsed_time(marks[3]))
        parts["day_end"].append(marks[3].elapsed_time(marks[4]))
    part_ms = {k: float(np.sum(v)) for k, v in parts.items()}
    m = float(np.mean(ms))
    cs = args.ncell * 24 * nday
    step_ms = part_ms["hourly_step"] / nday
    bpl = _algorithmic_bytes(HOURS) * args.ncell
    peak, peak_kind = _peaks()
    line = {
        "metric": "cell-steps/s, day loop over a month (daily cadence + hourly steps + monthly CH4)",
        "value": cs / (m / 1e3), "unit": "cell-steps/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": m, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": f"{args.ncell} cells x {nday} days (one month) per step: per day the daily cadence, "
                               "24 hours of forcing generated from the day's weather, 24 hourly steps with "
                               "accumulators and hourly CH4; the month's wetland methane at its end",
                   "ncell": args.ncell, "days": nday, "launch_config": cols.config,
                   "tuned_ms": ({str(k): round(v, 4) for k, v in tuned["ms"].items()} if tuned else None),
                   "l2": "state (27 MB) + statics (48 MB) + a day's forcing (110 MB) exceed L2 each day"},
        "launch_ms_per_month": part_ms,
        "roofline": {"bound": "hbm", "kernel": "hourly step (24 h per launch)",
                     "achieved": bpl / (step_ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": bpl / (step_ms / 1e3) / 1e9 / peak, "traffic": None, "peak_source": peak_kind},
        "e2e": {"value": cs / (float(np.mean(ms_e2e)) / 1e3), "unit": "cell-steps/s",
                "h2d_bytes_per_step": int(h_daily.numel() * 4),
                "d2h_bytes_per_step": int((h_prog.numel() + h_dayst.numel() + h_wet.numel()) * 4)},
        "gpu_launches": args.steps * (4 * nday + 2),
        "clocks": clk.summary(), "nonfinite_columns": nonfinite[0],
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="day", choices=["day", "ensemble", "serve", "month"])
    ap.add_argument("--days", type=int, default=30, help="month: days per step")
    ap.add_argument("--sites", type=int, default=356)
    ap.add_argument("--params-per-site", type=int, default=64)
    ap.add_argument("--tune", action="store_true", help="ensemble: autotune the block size first")
    ap.add_argument("--record-hours", type=int, default=None, help="ensemble: every record this long (profiling)")
    ap.add_argument("--rate", type=float, default=50.0)
    ap.add_argument("--duration", type=float, default=10.0)
    ap.add_argument("--epoch-hours", type=int, default=168)
    ap.add_argument("--e2e-group", type=int, default=0,
                    help="columns per group of the host-buffer entry (a multiple of 32; 0: the library's choice)")
    ap.add_argument("--e2e-chunk", default="auto",
                    help="hours per host-to-device forcing chunk in the e2e path ('auto': 4 hours, growing by 1.75)")
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--ncell", type=int, default=NCELL)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="day only: skip the release-parameter, ensemble, serve and single-column sub-workloads")
    ap.add_argument("--config", type=int, default=None, help="launch configuration (default: autotuned)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "ensemble":
        run_ensemble(args)
    elif args.workload == "month":
        run_month(args)
    elif args.workload == "serve":
        run_serve(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
