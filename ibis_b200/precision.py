"""Precision report: the FP32 kernels against the FP64 kernels over a year.

The production kernels run the step in FP32 with two FP64 islands (the 9x9
canopy energy/vapour system of ``turvap`` and the soil-water tridiagonal solve)
and Kahan-compensated accumulators; the FP64 kernels run every operation in
double and match the float64 CPU restatement of the reference to ~1e-13 per
step.  :func:`report` runs both on the same seeded cells for a year of hourly
forcing and states, per annual flux, the maximum and mean relative error of
the FP32 result over the cells and the relative error of the all-cell total,
and whether the integer-valued counters of the state agree exactly.

The reference documents its own float32 run against its float64 run the same
way (docs/technote/17_numerics_verification.md:367-383).

Run ``python -m ibis_b200.precision [ncell] [nhour]`` for a JSON report.
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


def report(ncell: int = 1000, nhour: int = 8760, seed: int = 2024, chunk: int = 720, device="cuda",
           lat_range=(-60.0, 80.0), alpha: float = 0.5) -> dict:
    """Run ``ncell`` cells for ``nhour`` hours in FP32 and FP64; return the report."""
    rng = np.random.Generator(np.random.PCG64(seed))
    lat = rng.uniform(lat_range[0], lat_range[1], size=ncell)
    stat = synth.make_columns(rng, ncell, alpha)
    f0 = synth.make_forcing(rng, lat, min(chunk, nhour), start_doy=1)
    prog = synth.make_initial(rng, stat, {k: v[0] for k, v in f0.items()})
    P = StepParams(co2conc=390.0e-6)
    P.flags = P.flags | FLAG_SOIL_MEANS
    P64 = P.copy()
    P64.flags = P64.flags & ~FLAG_KAHAN
    c32 = Columns.from_host(prog, stat, dtype=torch.float32, acc=True, device=device)
    c64 = Columns.from_host(prog, stat, dtype=torch.float64, acc=True, device=device)
    t0 = time.time()
    h = 0
    fc = f0
    gpu_ms = {"f32": 0.0, "f64": 0.0}
    while h < nhour:
        n = min(chunk, nhour - h)
        if h > 0:
            fc = synth.make_forcing(rng, lat, n, start_doy=1, start_hour=h)
        for cols, par, key in ((c32, P, "f32"), (c64, P64, "f64")):
            planes = synth.forcing_planes(fc, cols.ld, 0, n,
                                          dtype=np.float32 if cols.dtype == torch.float32 else np.float64)
            f = torch.from_numpy(planes).to(cols.device)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            for d in range(0, n, 24):          # one launch per day, as the day loop runs
                cols.run(f[d:d + 24], par)
            b.record()
            b.synchronize()
            gpu_ms[key] += a.elapsed_time(b)
        h += n
    torch.cuda.synchronize()
    a32, a64 = c32.acc_host(), c64.acc_host()
    p32, p64 = c32.prog_host(), c64.prog_host()
    out = {"ncell": ncell, "nhour": nhour, "seed": seed, "wall_s": time.time() - t0, "gpu_ms": gpu_ms,
           "nonfinite": {"f32": c32.nonfinite()[0], "f64": c64.nonfinite()[0]}, "fluxes": {}, "soil_t": {},
           "state": {}, "counters": {}}
    for name, acc in FLUXES.items():
        out["fluxes"][name] = _stats(a32[acc], a64[acc])
    days = nhour / 24.0
    for k in range(L.NSOILAY):
        out["soil_t"][f"layer{k}"] = _stats(a32["tsoi_mean"][:, k] / days, a64["tsoi_mean"][:, k] / days)
    for name in ("tsoi", "wsoi", "tg", "tu", "tl", "fi", "hsno"):
        out["state"][name] = _stats(p32[name], p64[name])
    for name in COUNTERS:
        d = np.abs(p32[name] - p64[name])
        out["counters"][name] = {"equal_frac": float(np.mean(d == 0.0)), "max_abs_diff": float(np.max(d)),
                                 "integer_valued": bool(np.all(p32[name] == np.round(p32[name])))}
    return out


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    ncell = int(argv[0]) if argv else 1000
    nhour = int(argv[1]) if len(argv) > 1 else 8760
    print(json.dumps(report(ncell, nhour), indent=1))


if __name__ == "__main__":
    main()
