"""Precision report: the FP32 kernels against float64 over a year.

The production kernels run the step in FP32 with two FP64 islands (the 9x9
canopy energy/vapour system of ``turvap`` and the soil-water tridiagonal solve)
and Kahan-compensated accumulators; the FP64 kernels run every operation in
double and match the float64 CPU restatement of the reference to ~1e-13 per
step.  :func:`report` runs, on the first ``ncell`` columns of the 95,333-cell
population (the columns of the day workload's generator, latitude
U(-60, 80), Dirichlet(0.5) plant types) for a year of seeded hourly forcing:

* ``f32``   -- the production FP32 kernels;
* ``f64``   -- the FP64 kernels (the float64 GPU oracle);
* ``f64_w32`` -- the FP64 kernels with the soil-water state (``wsoi``,
  ``wisoi``, ``wpud``, ``wipud``) rounded to float32 after every hour, as a
  float32 state stores it (the reference's FP32 production run casts its
  state to float32 after each step, ``_cast_tree_f32``, loops_gswp3.py:304):
  the part of the FP32 drift that storing soil water in float32 causes,
  whatever the arithmetic (temperatures are left alone: rounding a
  temperature held at the float64 melting point to float32 moves it off that
  point, which a float32 kernel, whose melting point is the float32 value,
  never does);
* optionally the float64 CPU oracle (the restatement of the reference pinned
  to its outputs) on the first ``oracle_cells`` columns;

and states, per annual flux, the maximum and mean relative error over the
cells and the relative error of the all-cell total, against ``f64``, and
whether the integer-valued counters agree exactly.  :func:`full_size_year`
runs the FP32 kernels on all 95,333 columns for a year with the hourly forcing
generated on the device from daily weather.

The reference documents its own float32 run against its float64 run the same
way (docs/technote/17_numerics_verification.md:367-383).

Run ``python -m ibis_b200.precision [ncell] [nhour] [oracle_cells]`` for a JSON
report, ``python -m ibis_b200.precision --full`` for the full-size year.
"""
from __future__ import annotations

import json
import sys
import time

import numpy as np
import torch

from . import layout as L
from . import synth
from .columns import Columns
from .params import FLAG_KAHAN, FLAG_SOIL_MEANS, StepParams

# annual flux -> accumulator plane(s); soil temperature by layer from the
# daily-weighted sums of tsoi (annual mean = sum / days)
FLUXES = {
    "gpp": "aygpptot", "npp": "aynpptot", "et": "adaet", "sensible_heat": "afsena",
    "runoff": "aytrunof", "drainage": "aytdrain", "ch4": "ch4",
}
COUNTERS = ("nytimes", "nfirestep", "nfirestep_vpd")
POPULATION = 95333


def _rel(a32, a64, floor):
    return np.abs(a32 - a64) / np.maximum(np.abs(a64), floor)


def _stats(a32, a64, floor_frac=1e-3):
    """Max/mean relative error over cells (floor = floor_frac x the largest |FP64|
    value of the field, so cells where it is ~0 do not dominate) and the relative
    error of the all-cell sum."""
    a32 = np.asarray(a32, np.float64)
    a64 = np.asarray(a64, np.float64)
    floor = max(floor_frac * float(np.max(np.abs(a64))), 1e-300)
    r = _rel(a32, a64, floor)
    tot64 = float(np.sum(a64))
    return {"max_rel": float(np.max(r)), "mean_rel": float(np.mean(r)),
            "total_rel": abs(float(np.sum(a32)) - tot64) / max(abs(tot64), 1e-300),
            "floor": floor, "fp64_total": tot64}


def population(ncell: int, seed: int = 2024, lat_range=(-60.0, 80.0), alpha: float = 0.5):
    """The first ``ncell`` columns of the 95,333-cell population: static planes,
    latitudes and a generator for their forcing (the columns are drawn for the
    whole population, so the first 1,000 are the same whatever ``ncell``)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    lat = rng.uniform(lat_range[0], lat_range[1], size=POPULATION)[:ncell]
    stat = {k: v[:ncell] for k, v in synth.make_columns(rng, POPULATION, alpha).items()}
    return stat, lat, np.random.Generator(np.random.PCG64(seed + 1))


def _annual(cols, nhour):
    acc, prog = cols.acc_host(), cols.prog_host()
    out = {name: np.asarray(acc[a], np.float64) for name, a in FLUXES.items()}
    days = nhour / 24.0
    out["tsoi_mean"] = np.asarray(acc["tsoi_mean"], np.float64) / days
    out["prog"] = prog
    return out


def _compare(x, ref):
    res = {"fluxes": {}, "soil_t": {}, "counters": {}}
    for name in FLUXES:
        res["fluxes"][name] = _stats(x[name], ref[name])
    for k in range(L.NSOILAY):
        res["soil_t"][f"layer{k}"] = _stats(x["tsoi_mean"][:, k], ref["tsoi_mean"][:, k])
    for name in COUNTERS:
        d = np.abs(np.asarray(x["prog"][name]) - np.asarray(ref["prog"][name]))
        res["counters"][name] = {"equal_frac": float(np.mean(d == 0.0)), "max_abs_diff": float(np.max(d)),
                                 "integer_valued": bool(np.all(x["prog"][name] == np.round(x["prog"][name])))}
    return res


def _oracle_chunk(task):
    import oracle
    prog, stat, forcs, P = task
    n = prog["tg"].shape[0]
    acc = oracle.new_acc(n)
    with np.errstate(all="ignore"):
        for F in forcs:
            for h in range(F["ta"].shape[0]):
                prog, _, acc = oracle.step(prog, stat, {k: v[h] for k, v in F.items()}, P, acc)
    return prog, acc


def report(ncell: int = 1000, nhour: int = 8760, seed: int = 2024, chunk: int = 720, device="cuda",
           oracle_cells: int = 0, legs=("f32", "f64", "f64_w32"), params: StepParams | None = None) -> dict:
    """Run the legs on the first ``ncell`` columns for ``nhour`` hours; return the
    report (every leg against ``f64``; with ``oracle_cells`` also ``f64`` and
    ``f32`` against the float64 oracle on the first ``oracle_cells`` columns).
    ``params``: the step's parameters (default: the defaults at 390 ppm CO2);
    under temperature acclimation the columns get seeded acclimation states."""
    from .params import FLAG_ACCLIM
    stat, lat, rng = population(ncell, seed)
    f0 = synth.make_forcing(rng, lat, min(chunk, nhour), start_doy=1)
    prog = synth.make_initial(rng, stat, {k: v[0] for k, v in f0.items()})
    P = StepParams(co2conc=390.0e-6) if params is None else params.copy()
    if P.flags & FLAG_ACCLIM:
        stat = dict(stat, acclim_x=np.random.default_rng(seed + 1).uniform(-12.0, 28.0, ncell))
    P.flags = P.flags | FLAG_SOIL_MEANS
    P64 = P.copy()
    P64.flags = P64.flags & ~FLAG_KAHAN
    cols = {}
    if "f32" in legs:
        cols["f32"] = Columns.from_host(prog, stat, dtype=torch.float32, acc=True, device=device)
    for leg in ("f64", "f64_w32"):
        if leg in legs or leg == "f64":
            cols[leg] = Columns.from_host(prog, stat, dtype=torch.float64, acc=True, device=device)
    oracle_forc = []
    w32 = torch.tensor([L.OFF["PROG"][k][0] + j for k in ("wsoi", "wisoi", "wpud", "wipud")
                        for j in range(L.OFF["PROG"][k][1])], device=device)
    t0 = time.time()
    h = 0
    fc = f0
    gpu_ms = {k: 0.0 for k in cols}
    while h < nhour:
        n = min(chunk, nhour - h)
        if h > 0:
            fc = synth.make_forcing(rng, lat, n, start_doy=1, start_hour=h)
        if oracle_cells:
            oracle_forc.append({k: v[:n, :oracle_cells].copy() for k, v in fc.items()})
        for leg, c in cols.items():
            planes = synth.forcing_planes(fc, c.ld, 0, n,
                                          dtype=np.float32 if c.dtype == torch.float32 else np.float64)
            f = torch.from_numpy(planes).to(c.device)
            par = P if leg == "f32" else P64
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            if leg == "f64_w32":
                for d in range(n):             # one hour per launch, soil water stored as float32 between hours
                    c.run(f[d:d + 1], par)
                    c.prog[w32] = c.prog[w32].float().double()
            else:
                for d in range(0, n, 24):      # one launch per day, as the day loop runs
                    c.run(f[d:d + 24], par)
            b.record()
            b.synchronize()
            gpu_ms[leg] += a.elapsed_time(b)
        h += n
    torch.cuda.synchronize()
    res = {k: _annual(c, nhour) for k, c in cols.items()}
    out = {"ncell": ncell, "nhour": nhour, "seed": seed, "population": f"first {ncell} of {POPULATION} columns",
           "wall_s": time.time() - t0, "gpu_ms": gpu_ms,
           "nonfinite": {k: c.nonfinite()[0] for k, c in cols.items()}, "legs": {}}
    for leg in cols:
        if leg != "f64":
            out["legs"][leg] = _compare(res[leg], res["f64"])
    # the final state of the FP32 leg against the FP64 leg
    if "f32" in res:
        out["state"] = {name: _stats(res["f32"]["prog"][name], res["f64"]["prog"][name])
                        for name in ("tsoi", "wsoi", "tg", "tu", "tl", "fi", "hsno")}
        out["fluxes"] = out["legs"]["f32"]["fluxes"]
        out["soil_t"] = out["legs"]["f32"]["soil_t"]
        out["counters"] = out["legs"]["f32"]["counters"]
    if oracle_cells:
        import multiprocessing as mp
        import os
        nproc = max(1, min(oracle_cells, (os.cpu_count() or 1)))
        idx = np.array_split(np.arange(oracle_cells), nproc)
        sl = lambda d, ix: {k: np.asarray(v)[ix] for k, v in d.items()}
        tasks = [(sl(prog, ix), sl(stat, ix), [{k: v[:, ix] for k, v in F.items()} for F in oracle_forc], P64)
                 for ix in idx if ix.size]
        t1 = time.time()
        with mp.get_context("spawn").Pool(len(tasks)) as pool:
            parts = pool.map(_oracle_chunk, tasks)
        oprog = {k: np.concatenate([p[0][k] for p in parts]) for k in parts[0][0]}
        oacc = {k: np.concatenate([p[1][k] for p in parts]) for k in parts[0][1]}
        ores = {name: np.asarray(oacc[a], np.float64) for name, a in FLUXES.items()}
        ores["tsoi_mean"] = oacc["tsoi_mean"] / (nhour / 24.0)
        ores["prog"] = oprog
        sub = lambda r: {**{k: v[:oracle_cells] for k, v in r.items() if k != "prog"},
                         "prog": {k: np.asarray(v)[:oracle_cells] for k, v in r["prog"].items()}}
        out["oracle"] = {"cells": oracle_cells, "processes": len(tasks), "wall_s": time.time() - t1,
                         "f64_vs_oracle": _compare(sub(res["f64"]), ores)}
        if "f32" in res:
            out["oracle"]["f32_vs_oracle"] = _compare(sub(res["f32"]), ores)
    return out


def full_size_year(ncell: int = POPULATION, ndays: int = 365, seed: int = 2024, check_cells: int = 1000,
                   device="cuda") -> dict:
    """All ``ncell`` columns of the population in FP32 for ``ndays`` days, the
    hourly forcing generated on the device from seeded daily weather (the
    reference's diurnal algorithm, ``ibis_diurnal_f32``): time, finiteness,
    physical bounds, and whether the first ``check_cells`` columns equal a run of
    those columns alone (columns are independent, so they must, bit for bit)."""
    from . import forcing as _forcing
    stat, lat, rng = population(ncell, seed)
    daily = synth.make_daily_weather(rng, lat, ndays)
    f0 = synth.make_forcing(np.random.Generator(np.random.PCG64(seed + 3)), lat, 1, start_doy=1)
    prog = synth.make_initial(rng, stat, {k: v[0] for k, v in f0.items()})
    P = StepParams(co2conc=390.0e-6)
    P.flags = P.flags | FLAG_SOIL_MEANS
    big = Columns.from_host(prog, stat, dtype=torch.float32, acc=True, device=device)
    small = Columns.from_host({k: v[:check_cells] for k, v in prog.items()},
                              {k: v[:check_cells] for k, v in stat.items()}, dtype=torch.float32, acc=True,
                              device=device)
    big.set_mode(6)
    small.set_mode(6)
    d_daily = torch.from_numpy(_forcing.daily_planes(daily, big.ld)).to(big.device)
    lat_d = torch.zeros(big.ld, dtype=torch.float32, device=big.device)
    lat_d[:ncell] = torch.from_numpy(lat.astype(np.float32)).to(big.device)
    step_ms = 0.0
    t0 = time.time()
    for d in range(ndays):
        f = _forcing.hourly_forcing(d_daily[d:d + 1], lat_d, ncell, jday0=1 + d, day0=d, seed=seed)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        big.run(f, P)
        b.record()
        small.run(f[:, :, :small.ld].contiguous(), P)
        b.synchronize()
        step_ms += a.elapsed_time(b)
    torch.cuda.synchronize()
    pb, ps = big.prog_host(), small.prog_host()
    ab, as_ = big.acc_host(), small.acc_host()
    same = all(np.array_equal(np.asarray(pb[k])[:check_cells], np.asarray(ps[k])) for k in pb) and \
        all(np.array_equal(np.asarray(ab[k])[:check_cells], np.asarray(as_[k])) for k in ab)
    bounds = {"tsoi_K": [float(pb["tsoi"].min()), float(pb["tsoi"].max())],
              "wsoi": [float(pb["wsoi"].min()), float(pb["wsoi"].max())],
              "tu_K": [float(pb["tu"].min()), float(pb["tu"].max())]}
    return {"ncell": ncell, "days": ndays, "step_ms": step_ms, "wall_s": time.time() - t0,
            "cell_steps_per_s": ncell * 24 * ndays / (step_ms / 1e3), "nonfinite": big.nonfinite()[0],
            "first_cells_equal_alone": bool(same), "check_cells": check_cells, "bounds": bounds,
            "annual_gpp_total": float(np.sum(ab["aygpptot"])), "annual_runoff_total": float(np.sum(ab["aytrunof"]))}


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    if argv and argv[0] == "--full":
        print(json.dumps(full_size_year(), indent=1))
        return
    ncell = int(argv[0]) if argv else 1000
    nhour = int(argv[1]) if len(argv) > 1 else 8760
    ocells = int(argv[2]) if len(argv) > 2 else 0
    print(json.dumps(report(ncell, nhour, oracle_cells=ocells), indent=1))


if __name__ == "__main__":
    main()
