"""The daily cadence: the oracle (oracle/daily.py + the hourly oracle step +
oracle/weather.py) against the reference's own GSWP3 day loop run for three
days on the 16-cell checkpoint (tests/golden/days_16cells.npz), CPU; the
device daily kernels against the same fixture, GPU.

Tolerance: relative 1e-9 after each day on every state field the day loop
touches (prognostic state, phenology, canopy structure, 10-day means, annual
sums, soil carbon), float64 throughout; 1e-6 for the accumulators the
reference sums in float32 steps.
"""
import os
import warnings

import numpy as np
import pytest

import oracle
from goldens import compare
from ibis_b200 import layout as L
from ibis_b200 import restart
from ibis_b200.params import DAY_PARAM_FIELDS, FLAG_ACC, FLAG_CH4, FLAG_KAHAN, PARAM_FIELDS, DayParams, StepParams
from oracle import daily as OD
from oracle import weather as OW

warnings.filterwarnings("ignore", category=RuntimeWarning)
HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden", "days_16cells.npz")
CKPT = os.path.join(HERE, "golden", "restart_16cells.npz")
ACC_CHECK = ("adrain", "adsnow", "adaet", "aynpp", "aynpptot", "aygpptot", "aytrunof", "aytdrain")
STAT_CHECK = ("frac", "lai", "ztop", "zbot", "tco2mic")


def load_case():
    z = np.load(GOLD)
    z = {k: z[k] for k in z.files}
    leaves, _, _ = restart.load(CKPT)
    n = int(np.asarray(leaves["soil.tg"]).shape[0])
    tree = restart.as_tree(leaves)
    from ibis_b200 import dropin
    prog = dropin._leaf_dict(tree, "PROG", n)
    stat = dropin._leaf_dict(tree, "STAT", n)
    stat["f_inund"] = np.zeros(n)
    day = restart.group_from_leaves(leaves, "DAYST", n)
    acc0 = restart.group_from_leaves(leaves, "ACC", n)
    P = StepParams()
    for name, _, _ in PARAM_FIELDS:
        setattr(P, name, z["in.param." + name])
    P.flags = (int(z["in.param.flags"]) | FLAG_ACC) & ~(FLAG_CH4 | FLAG_KAHAN)
    return z, n, prog, stat, day, acc0, P


def day_params(z):
    DP = DayParams()
    for name, _, _ in DAY_PARAM_FIELDS:
        setattr(DP, name, z["in.dparam." + name])
    return DP


def want(z, d, group, n=16):
    out = {}
    for f in L.GROUPS[group]:
        k = f"out.{d}.{f.leaf}"
        if k in z:
            out[f.name] = np.full(n, float(z[k])) if z[k].ndim == 0 else z[k]
    return out


def test_checkpoint_implies_the_reference_parameters():
    """The record a checkpoint implies equals the one the reference derives from
    the same checkpoint under its default SimParams."""
    z, n, prog, stat, day, acc0, P = load_case()
    leaves, _, _ = restart.load(CKPT)
    Q = restart.params_from_leaves(leaves)
    for name, _, _ in PARAM_FIELDS:
        np.testing.assert_allclose(getattr(Q, name), getattr(P, name), rtol=1e-12, err_msg=name)


def test_oracle_day_loop_matches_reference_days():
    z, n, prog, stat, day, acc0, P = load_case()
    DP = day_params(z)
    acc = oracle.new_acc(n)
    for k in ACC_CHECK + ("stresstu_last", "stresstl_last"):
        if k in acc0:
            acc[k] = acc0[k].copy()
    seed, jday0, cells = int(z["in.seed"]), int(z["in.jday0"]), np.arange(n)
    for d in range(int(z["in.ndays"])):
        dd = {k[len(f"in.daily.{d}."):]: v for k, v in z.items() if k.startswith(f"in.daily.{d}.")}
        day, stat, acc = OD.day_begin(day, stat, acc, dd["td"], P, DP)
        plens, startp, endp = OW.precip_timing(OW.uniform24(seed, cells, d, 0), OW.uniform24(seed, cells, d, 1),
                                               dd["precip"], 3600.0)
        with np.errstate(all="ignore"):
            for h in range(24):
                F = OW.diurnal(h * 3600.0, jday0 + d, dd, z["in.lat"], plens, startp, endp,
                               OW.uniform24(seed, cells, d, 2 + h), 3600.0, fira_obs=dd["fira"])
                prog, D, acc = oracle.step(prog, stat, F, P, acc)
        day, stat = OD.day_end(prog, day, stat, acc, dd["td"], P, DP)
        bad = compare(prog, want(z, d, "PROG"), 1e-9) + compare(day, want(z, d, "DAYST"), 1e-9)
        bad += compare({k: stat[k] for k in STAT_CHECK}, want(z, d, "STAT"), 1e-9)
        bad += compare({k: acc[k] for k in ACC_CHECK}, want(z, d, "ACC"), 1e-6)
        assert not bad, (d, bad[:6])
