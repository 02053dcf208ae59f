"""Load the golden fixtures (reference outputs) and compare arrays against them."""
from __future__ import annotations

import os

import numpy as np

from ibis_b200 import layout as L
from ibis_b200.params import PARAM_FIELDS, StepParams

GOLDEN_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = ("day_mixed", "nobedrock", "sunshade", "perturbed")


class Case:
    def __init__(self, name):
        self.name = name
        z = np.load(os.path.join(GOLDEN_DIR, f"{name}.npz"))
        self.z = {k: z[k] for k in z.files}
        self.prog = {k[8:]: v for k, v in self.z.items() if k.startswith("in.prog.")}
        self.stat = {k[8:]: v for k, v in self.z.items() if k.startswith("in.stat.")}
        self.forc = {k[8:]: v for k, v in self.z.items() if k.startswith("in.forc.")}
        P = StepParams()
        for name_, n, _ in PARAM_FIELDS:
            setattr(P, name_, self.z["in.param." + name_])
        P.flags = int(self.z["in.param.flags"])
        self.params = P
        self.ncell = self.prog["tg"].shape[0]
        self.nhour = self.forc["ta"].shape[0]
        self.record = [int(x) for x in self.z["meta.record"]]
        self.has_day = any(k.startswith("day.") for k in self.z)

    def forcing_at(self, h):
        return {k: v[h] for k, v in self.forc.items()}

    def out(self, h, group):
        pre = f"out.{h}.{group}."
        return {k[len(pre):]: v for k, v in self.z.items() if k.startswith(pre)}

    def day(self, group):
        pre = f"day.{group}."
        return {k[len(pre):]: v for k, v in self.z.items() if k.startswith(pre)}


def rel_err(a, b, floor):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return np.abs(a - b) / np.maximum(np.abs(b), floor)


# Absolute floors for near-zero quantities, by field (used in the relative errors)
FLOORS = {
    "q12": 1e-6, "q34": 1e-6, "wliqu": 1e-6, "wliqs": 1e-6, "wliql": 1e-6, "wsnou": 1e-6, "wsnos": 1e-6,
    "wsnol": 1e-6, "wpud": 1e-6, "wipud": 1e-6, "hsno": 1e-6, "fi": 1e-6, "wisoi": 1e-6, "wsoi": 1e-6,
    "an_upper": 1e-9, "ag_upper": 1e-9, "an_lower": 1e-9, "ag_lower": 1e-9,
    "ci_upper": 1e-8, "ci_lower": 1e-8, "cs_upper": 1e-8, "cs_lower": 1e-8, "gs_upper": 1e-6, "gs_lower": 1e-6,
    "fvapg": 1e-9, "fvapi": 1e-9, "ginvap": 1e-9, "gsuvap": 1e-9, "gtrans": 1e-9, "gtransu": 1e-9,
    "gtransl": 1e-9, "grunof": 1e-9, "gdrain": 1e-9, "gadjust": 1e-9, "raing": 1e-9, "snowg": 1e-9,
    "rainl": 1e-9, "snowl": 1e-9, "raing_avg": 1e-9, "ch4": 1e-15, "aygpptot": 1e-9, "aynpptot": 1e-9,
    "aynpp": 1e-9, "a10ancub": 1e-9, "a10ancls": 1e-9, "a10ancl3": 1e-9, "a10ancl4": 1e-9,
}
# energy fluxes (W m-2): an absolute floor of 1 W m-2 for near-zero fluxes
for _k in ("hflo", "fsenu", "fsens", "fsenl", "fseng", "fseni", "firu", "firs", "firl", "firg", "firi", "firb",
           "heatg", "heati", "fhtop_soil", "fhtop_snow", "sflo_bot", "solu", "sols", "soll", "solg", "soli"):
    FLOORS[_k] = 1.0


def compare(got: dict, want: dict, rtol: float, default_floor=1e-3, skip=()):
    """Return a list of (field, max_rel_err, cell) exceeding rtol."""
    bad = []
    for k, w in want.items():
        if k in skip or k not in got:
            continue
        g = np.asarray(got[k], dtype=np.float64).reshape(w.shape)
        fl = FLOORS.get(k, default_floor)
        e = rel_err(g, w, fl)
        both_nan = np.isnan(g) & np.isnan(w)
        e = np.where(both_nan, 0.0, e)
        e = np.where(np.isnan(e), np.inf, e)
        m = float(np.max(e)) if e.size else 0.0
        if m > rtol:
            idx = np.unravel_index(int(np.argmax(e)), e.shape)
            bad.append((k, m, idx, float(g[idx]), float(w[idx])))
    return bad
