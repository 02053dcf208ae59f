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
import types
import warnings

import numpy as np
import pytest

import oracle
from goldens import HAVE_REF, REF_PORT, compare, rel_err
from ibis_b200 import layout as L
from ibis_b200 import restart
from ibis_b200.params import DAY_PARAM_FIELDS, FLAG_ACC, FLAG_CH4, FLAG_KAHAN, PARAM_FIELDS, DayParams, StepParams
from oracle import daily as OD
from oracle import weather as OW

warnings.filterwarnings("ignore", category=RuntimeWarning)
HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden", "days_16cells.npz")
GOLD_MODULES = os.path.join(HERE, "golden", "days_modules_16cells.npz")
# the modules case again under the release parameter file's stomata switches
# (acclimation driven by the seasonal state, vmax and slope mixing, capacity split,
# sunlit/shaded canopies)
GOLD_RELEASE = os.path.join(HERE, "golden", "days_release_16cells.npz")
MODULE_LEAVES = {"acclim_x": "seasonal.acclim_x", "ssen_u": "seasonal.ssen_u", "ssen_l": "seasonal.ssen_l",
                 "aystressu": "stress.aystressu", "aystressl": "stress.aystressl", "stress_nday": "stress.nday"}
PARTS = ("et_trans", "et_interc", "et_soilev", "et_snowsub", "nee_night", "nee_day")
CKPT = os.path.join(HERE, "golden", "restart_16cells.npz")
ACC_CHECK = ("adrain", "adsnow", "adaet", "aynpp", "aynpptot", "aygpptot", "aytrunof", "aytdrain")
STAT_CHECK = ("frac", "lai", "ztop", "zbot", "tco2mic")


def load_case(gold=GOLD):
    z = np.load(gold)
    z = {k: z[k] for k in z.files}
    leaves, _, _ = restart.load(CKPT)
    n = int(np.asarray(leaves["soil.tg"]).shape[0])
    tree = restart.as_tree(leaves)
    from ibis_b200 import dropin
    prog = dropin._leaf_dict(tree, "PROG", n)
    stat = dropin._leaf_dict(tree, "STAT", n)
    stat["f_inund"] = np.zeros(n)
    day = restart.group_from_leaves(leaves, "DAYST", n)
    day["latitude"] = np.deg2rad(z["in.lat"])
    for name, leaf in MODULE_LEAVES.items():
        day[name] = z.get("in." + leaf, np.zeros(n))
    acc0 = restart.group_from_leaves(leaves, "ACC", n)
    P = StepParams()
    for name, _, _ in PARAM_FIELDS:
        if "in.param." + name in z:
            setattr(P, name, z["in.param." + name])
    P.flags = (int(z["in.param.flags"]) | FLAG_ACC) & ~(FLAG_CH4 | FLAG_KAHAN)
    return z, n, prog, stat, day, acc0, P


def day_params(z):
    """The case's day parameters; with the optional modules both switched on."""
    DP = DayParams()
    for name, _, _ in DAY_PARAM_FIELDS:
        if "in.dparam." + name in z:
            setattr(DP, name, z["in.dparam." + name])
    DP.seasonal_on = DP.stress_on = float(z.get("in.modules", 0))
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


def day_weather(z, d):
    return {k[len(f"in.daily.{d}."):]: v for k, v in z.items() if k.startswith(f"in.daily.{d}.")}


def hourly(z, d, n):
    """The day's 24 hourly forcing dicts (oracle/weather.py, observed longwave)."""
    seed, jday0, cells, dd = int(z["in.seed"]), int(z["in.jday0"]), np.arange(n), day_weather(z, d)
    plens, startp, endp = OW.precip_timing(OW.uniform24(seed, cells, d, 0), OW.uniform24(seed, cells, d, 1),
                                           dd["precip"], 3600.0)
    with np.errstate(all="ignore"):
        return [OW.diurnal(h * 3600.0, jday0 + d, dd, z["in.lat"], plens, startp, endp,
                           OW.uniform24(seed, cells, d, 2 + h), 3600.0, fira_obs=dd["fira"]) for h in range(24)]


def oracle_days(ndays=None, perturb=None, f_inund=None, gold=GOLD):
    """The oracle's day loop on a three-day case; yields (day, prog, dayst,
    stat, acc) after each day.  ``perturb`` = (day, hour, eps[, fields])
    scales the temperatures (or ``fields``) of the state by (1 + eps) before
    that hour; ``f_inund`` turns on the hourly wetland CH4 with that
    inundated fraction."""
    z, n, prog, stat, day, acc0, P = load_case(gold)
    if f_inund is not None:
        P.flags |= FLAG_CH4
        stat["f_inund"] = np.asarray(f_inund, np.float64)
    DP = day_params(z)
    acc = oracle.new_acc(n)
    for k in ACC_CHECK + ("stresstu_last", "stresstl_last"):
        if k in acc0:
            acc[k] = acc0[k].copy()
    temps = ("tsoi", "tg", "tl", "tu", "ti", "tsno")
    for d in range(int(z["in.ndays"]) if ndays is None else ndays):
        dd = day_weather(z, d)
        DP.jday = float(int(z["in.jday0"]) + d)
        day, stat, acc = OD.day_begin(day, stat, acc, dd["td"], P, DP)
        with np.errstate(all="ignore"):
            for h, F in enumerate(hourly(z, d, n)):
                if perturb is not None and perturb[:2] == (d, h):
                    fields = perturb[3] if len(perturb) > 3 else temps
                    prog = {k: v * (1.0 + perturb[2]) if k in fields else v for k, v in prog.items()}
                prog, _, acc = oracle.step(prog, stat, F, P, acc)
        day, stat = OD.day_end(prog, day, stat, acc, dd["td"], P, DP)
        yield d, prog, day, stat, acc


# Threshold cells of the modules case (three days from day 250): 1e-15
# relative changes of the temperatures or of the water, ice and snow state before
# hour 0 or hour 12 of the first day move cells 0, 3, 4 and 11 beyond 1e-9
# within the three days (test_threshold_cells_of_the_modules_case); cell 0 by
# 8e-7 on the third day.
MODULE_THRESHOLD_CELLS = (0, 3, 4, 11)


def _cells(x, cells, ref):
    return {k: np.asarray(v)[list(cells)] for k, v in x.items() if k in ref}


def _compare_day(z, d, prog, day, stat, acc, exempt=()):
    """Every state field of day ``d`` against the case: 1e-9 (1e-6 for the
    float32-summed accumulators) outside ``exempt``, 1e-2 on it."""
    n = len(z["in.lat"])
    keep = np.setdiff1d(np.arange(n), exempt)
    wa = want(z, d, "ACC")
    pairs = [(prog, want(z, d, "PROG"), 1e-9), (day, want(z, d, "DAYST"), 1e-9),
             ({k: stat[k] for k in STAT_CHECK}, want(z, d, "STAT"), 1e-9),
             ({k: acc[k] for k in ACC_CHECK + PARTS if k in wa}, wa, 1e-6)]
    bad = []
    for got, ref, tol in pairs:
        bad += compare(_cells(got, keep, ref), _cells(ref, keep, ref), tol)
        if len(exempt):
            bad += compare(_cells(got, exempt, ref), _cells(ref, exempt, ref), 1e-2)
    return bad


@pytest.mark.parametrize("gold", [GOLD, GOLD_MODULES, GOLD_RELEASE], ids=["base", "modules", "release"])
def test_oracle_day_loop_matches_reference_days(gold):
    """The base case on every cell, the case whose state carries the optional
    modules (seasonal states with photoperiod-gated senescence, growing-season
    stress sums, ET and NEE parts) outside its threshold cells, and that case
    under the release parameter file's stomata switches on every cell: every
    state field after each day."""
    z = load_case(gold)[0]
    exempt = MODULE_THRESHOLD_CELLS if gold == GOLD_MODULES else ()
    checked = set()
    for d, prog, day, stat, acc in oracle_days(gold=gold):
        checked |= set(want(z, d, "DAYST"))
        bad = _compare_day(z, d, prog, day, stat, acc, exempt)
        assert not bad, (d, bad[:6])
    assert (set(MODULE_LEAVES) <= checked) == (gold != GOLD)


@pytest.mark.parametrize("gold", [GOLD_MODULES, GOLD_RELEASE], ids=["modules", "release"])
def test_threshold_cells_of_the_modules_case(gold):
    """The exempt cells of the modules case (and of the same case under the
    release parameter file's switches) are threshold cells: over the three
    days, 1e-15 perturbations (either sign) of the oracle's own temperatures or
    of its water, ice and snow state, before hour 0 or hour 12 of the first day,
    move exactly them beyond 1e-9."""
    n = 16
    base = list(oracle_days(gold=gold))
    moved = set()
    cases = [(h, eps, f) for h in (0, 12) for eps in (-1e-15, 1e-15)
             for f in (("tsoi", "tg", "tl", "tu", "ti", "tsno"), ("wsoi", "wisoi", "hsno", "wpud", "wipud", "fi"))]
    for h, eps, fields in cases:
        for (_, bp, bd, _, _), (_, pp, pd, _, _) in zip(base, oracle_days(gold=gold, perturb=(0, h, eps, fields))):
            err = np.zeros(n)
            for got, ref in ((pp, bp), (pd, bd)):
                for k, w in ref.items():
                    e = np.nan_to_num(rel_err(np.asarray(got[k], np.float64), np.asarray(w, np.float64), 1e-3))
                    err = np.maximum(err, e.reshape(n, -1).max(axis=1))
            moved |= set(np.nonzero(err > 1e-9)[0].tolist())
    assert moved == set(MODULE_THRESHOLD_CELLS), sorted(moved)


# Cells of the three-day case whose first day crosses a phase-change
# threshold: cell 0 takes 400 mm of snow onto 289 K soil, cell 2 has a frozen
# top layer under a thin snow cover.  A 1e-15 relative change of their
# temperatures before hour 0 moves their end-of-day state by up to 2e-4
# relative (test_threshold_cells_of_the_day_case), so last-bit differences
# between CUDA's and the host's exp/log/pow do the same.
DAY_THRESHOLD_CELLS = (0, 2)


def test_threshold_cells_of_the_day_case():
    """The exempt cells are threshold cells: the oracle's own day moves them
    beyond 1e-9 under a 1e-15 perturbation and leaves every other cell within it."""
    n = 16
    _, base, bday, _, _ = next(oracle_days(1))
    _, pert, pday, _, _ = next(oracle_days(1, perturb=(0, 0, -1e-15)))
    err = np.zeros(n)
    for got, ref in ((pert, base), (pday, bday)):
        for k, w in ref.items():
            e = np.nan_to_num(rel_err(np.asarray(got[k], np.float64), np.asarray(w, np.float64), 1e-3))
            err = np.maximum(err, e.reshape(n, -1).max(axis=1))
    moved = set(np.nonzero(err > 1e-9)[0].tolist())
    assert moved == set(DAY_THRESHOLD_CELLS), sorted(moved)


def _device_loop(dtype, gold=GOLD):
    import torch
    from ibis_b200.columns import Columns
    from ibis_b200.daily import DayLoop
    z, n, prog, stat, day, acc0, P = load_case(gold)
    cols = Columns.from_host(prog, stat, dtype=dtype, acc=True)
    cols.set_acc({k: acc0[k] for k in ACC_CHECK + ("stresstu_last", "stresstl_last") if k in acc0})
    loop = DayLoop(cols, P, day_params(z), day, lat=z["in.lat"], seed=int(z["in.seed"]), jday=int(z["in.jday0"]),
                   day=0, observed_fira=True)
    return z, n, cols, loop, torch


def _daily_tensor(z, d, ld, torch):
    from ibis_b200.forcing import daily_planes
    dd = {k[len(f"in.daily.{d}."):]: v for k, v in z.items() if k.startswith(f"in.daily.{d}.")}
    return dd, torch.from_numpy(daily_planes({k: v[None] for k, v in dd.items()}, ld)[0]).cuda()


def _device_state(cols, loop):
    from ibis_b200 import synth
    stat = synth.from_planes("STAT", cols.stat.cpu().numpy(), cols.ncell)
    return cols.prog_host(), loop.dayst_host(), stat, cols.acc_host()


@pytest.mark.gpu
@pytest.mark.parametrize("gold", [GOLD, GOLD_MODULES, GOLD_RELEASE], ids=["base", "modules", "release"])
def test_device_day_kernels_match_oracle(cuda_lib, gold):
    """ibis_day_begin_f64 / ibis_day_end_f64 on the oracle's own inputs of
    each day of a three-day case (with the optional modules: seasonal states,
    photoperiod-gated phenology, stress sums): 1e-12 relative on everything
    they write."""
    import torch
    from ibis_b200 import synth
    z, n, cols, loop, torch = _device_loop(torch.float64, gold)
    _, _, prog, stat, day, acc0, P = load_case(gold)
    DP = day_params(z)
    acc = oracle.new_acc(n)
    for k in ACC_CHECK + ("stresstu_last", "stresstl_last"):
        if k in acc0:
            acc[k] = acc0[k].copy()
    pad = lambda a: torch.from_numpy(np.pad(np.asarray(a, np.float64), (0, cols.ld - n))).cuda()

    def load(prog_, stat_, day_, acc_):
        cols.set_prog(prog_)
        cols.set_stat(stat_)
        cols.set_acc(acc_)
        loop.set_dayst(day_)

    def check(day_, stat_, acc_=None):
        gs = synth.from_planes("STAT", cols.stat.cpu().numpy(), n)
        bad = compare(loop.dayst_host(), day_, 1e-12) + compare({k: gs[k] for k in stat_}, stat_, 1e-12)
        if acc_ is not None:
            bad += compare(cols.acc_host(), acc_, 1e-12)
        return bad

    for d in range(int(z["in.ndays"])):
        dd = day_weather(z, d)
        load(prog, stat, day, acc)
        DP.jday = loop.jday = int(z["in.jday0"]) + d
        day, stat, acc = OD.day_begin(day, stat, acc, dd["td"], P, DP)
        loop.begin(pad(dd["td"]))
        torch.cuda.synchronize()
        bad = check(day, stat, acc)
        assert not bad, ("begin", d, bad[:6])
        with np.errstate(all="ignore"):
            for F in hourly(z, d, n):
                prog, _, acc = oracle.step(prog, stat, F, P, acc)
        load(prog, stat, day, acc)
        day, stat = OD.day_end(prog, day, stat, acc, dd["td"], P, DP)
        loop.end(pad(dd["td"]))
        torch.cuda.synchronize()
        bad = check(day, stat)
        assert not bad, ("end", d, bad[:6])


@pytest.mark.gpu
def test_device_day_loop_with_modules_matches_reference_days(cuda_lib):
    """The device day loop in float64 on the case whose state carries the
    optional modules (seasonal states with photoperiod-gated senescence of both
    canopies, growing-season stress sums, ET and NEE parts) against the
    reference's day loop after each of the three days: every state field
    within 1e-9 (1e-6 for the float32-summed accumulators) outside the case's
    threshold cells, which stay within 1e-2."""
    import torch
    from ibis_b200 import synth
    z, n, cols, loop, torch = _device_loop(torch.float64, GOLD_MODULES)
    assert loop.day_params.seasonal_on == 1.0 and loop.params.flags & (3 << 10)
    for d in range(int(z["in.ndays"])):
        dd, daily = _daily_tensor(z, d, cols.ld, torch)
        hours = hourly(z, d, n)
        forc = {k: np.stack([F[k] for F in hours]) for k in hours[0]}
        td = torch.from_numpy(np.pad(dd["td"], (0, cols.ld - n))).cuda()
        loop.run_day(daily, forc=torch.from_numpy(synth.forcing_planes(forc, cols.ld, dtype=np.float64)).cuda(), td=td)
        torch.cuda.synchronize()
        prog, dayst, stat, acc = _device_state(cols, loop)
        bad = _compare_day(z, d, prog, dayst, stat, acc, MODULE_THRESHOLD_CELLS)
        assert not bad, (d, bad[:6])


@pytest.mark.gpu
def test_device_day_loop_with_release_switches_matches_reference_days(cuda_lib):
    """The device day loop in float64 under the release parameter file's
    stomata switches, the acclimation state advanced each day by ibis_day_begin
    and read by that day's hourly steps, against the reference's day loop after
    each of the three days: every state field within 1e-9 (1e-6 for the
    float32-summed accumulators) outside the case's threshold cells -- the same
    four as the modules case, proven by the same perturbations
    (test_threshold_cells_of_the_modules_case) -- which stay within 1e-2."""
    import torch
    from ibis_b200 import synth
    from ibis_b200.params import FLAG_ACCLIM
    z, n, cols, loop, torch = _device_loop(torch.float64, GOLD_RELEASE)
    assert loop.day_params.seasonal_on == 1.0 and loop.params.flags & FLAG_ACCLIM
    for d in range(int(z["in.ndays"])):
        dd, daily = _daily_tensor(z, d, cols.ld, torch)
        hours = hourly(z, d, n)
        forc = {k: np.stack([F[k] for F in hours]) for k in hours[0]}
        td = torch.from_numpy(np.pad(dd["td"], (0, cols.ld - n))).cuda()
        loop.run_day(daily, forc=torch.from_numpy(synth.forcing_planes(forc, cols.ld, dtype=np.float64)).cuda(), td=td)
        torch.cuda.synchronize()
        prog, dayst, stat, acc = _device_state(cols, loop)
        bad = _compare_day(z, d, prog, dayst, stat, acc, MODULE_THRESHOLD_CELLS)
        assert not bad, (d, bad[:6])


@pytest.mark.gpu
def test_device_day_loop_f64_matches_reference_days(cuda_lib):
    """The device day loop (daily kernels + the float64 hourly step), fed each
    day's hourly forcing in float64, against the reference's day loop after
    each of the three days: 1e-9 relative on every cell but the threshold
    cells (DAY_THRESHOLD_CELLS), which stay within 1e-2 (their puddle ice,
    ~8e-5 kg m-2, moves by 0.3 %)."""
    import torch
    from ibis_b200 import synth
    z, n, cols, loop, torch = _device_loop(torch.float64)
    keep = np.setdiff1d(np.arange(n), DAY_THRESHOLD_CELLS)
    for d in range(int(z["in.ndays"])):
        dd, daily = _daily_tensor(z, d, cols.ld, torch)
        hours = hourly(z, d, n)
        forc = {k: np.stack([F[k] for F in hours]) for k in hours[0]}
        td = torch.from_numpy(np.pad(dd["td"], (0, cols.ld - n))).cuda()
        loop.run_day(daily, forc=torch.from_numpy(synth.forcing_planes(forc, cols.ld, dtype=np.float64)).cuda(), td=td)
        torch.cuda.synchronize()
        prog, dayst, stat, acc = _device_state(cols, loop)
        pairs = [(prog, want(z, d, "PROG")), (dayst, want(z, d, "DAYST")),
                 ({k: stat[k] for k in STAT_CHECK}, want(z, d, "STAT"))]
        for got, ref in pairs:
            sub = lambda x, c: {k: np.asarray(v)[c] for k, v in x.items() if k in ref}
            bad = compare(sub(got, keep), sub(ref, keep), 1e-9)
            bad += compare(sub(got, list(DAY_THRESHOLD_CELLS)), sub(ref, list(DAY_THRESHOLD_CELLS)), 1e-2)
            assert not bad, (d, bad[:6])
        bad = compare({k: acc[k][keep] for k in ACC_CHECK}, {k: v[keep] for k, v in want(z, d, "ACC").items()}, 1e-6)
        assert not bad, (d, bad[:6])


@pytest.mark.gpu
def test_device_day_loop_f32_generated_forcing(cuda_lib):
    """The whole day on the device in float32 -- forcing generated from the
    daily weather, hourly step, daily kernels -- against the reference's
    float64 day loop after three days.

    Float32 moves the canopy-air and leaf temperatures of single cells by up to
    ~2 K within a day (the reference's own float32 run departs from its float64
    run by up to 1.6 K in hourly canopy temperature,
    docs/technote/17_numerics_verification.md:367-383), and through them the
    fast litter pools.  So: phenology, 10-day means, canopy structure, slow soil
    pools and leaching within 1e-4 relative on every cell; litter, microbial
    carbon and respiration within 5e-2 on every cell and 5e-3 on all but three;
    temperatures within 3 K on every cell and 0.2 K on all but three; soil
    water within 3e-2 and 2e-3 on all but three."""
    import torch
    z, n, cols, loop, torch = _device_loop(torch.float32)
    for d in range(int(z["in.ndays"])):
        _, daily = _daily_tensor(z, d, cols.ld, torch)
        loop.run_day(daily)
    torch.cuda.synchronize()
    d = int(z["in.ndays"]) - 1
    prog, dayst, stat, acc = _device_state(cols, loop)
    for group in (prog, dayst, stat):
        for k, v in group.items():
            assert np.all(np.isfinite(v)), k

    def per_cell(got, ref, absolute=False):
        a = np.asarray(got, np.float64).reshape(ref.shape)
        e = np.abs(a - ref) if absolute else np.nan_to_num(rel_err(a, ref, 1e-3))
        return np.sort(e.reshape(n, -1).max(axis=1))

    w = want(z, d, "DAYST")
    tight = ("tempu", "templ", "agddu", "agddl", "dropu", "dropls", "dropl3", "dropl4", "a10td", "a10ancub",
             "a10ancls", "a10ancl3", "a10ancl4", "ayprcp", "csoislop", "csoislon", "csoipas", "totcsoi", "storedn",
             "tnmin", "yrleach", "ynleach")
    for k in tight:
        assert per_cell(dayst[k], w[k])[-1] < 1e-4, k
    for k in ("clitlm", "clitls", "clitll", "clitrm", "clitrs", "clitrl", "clitwm", "clitws", "clitwl", "totcmic",
              "totlit", "ayco2mic", "ayaet"):
        e = per_cell(dayst[k], w[k])
        assert e[-1] < 5e-2 and e[-4] < 5e-3, (k, e[-4:])
    w = want(z, d, "STAT")
    for k in ("frac", "lai", "ztop", "zbot"):
        assert per_cell(stat[k], w[k])[-1] < 1e-4, k
    e = per_cell(stat["tco2mic"], w["tco2mic"])
    assert e[-1] < 5e-2 and e[-4] < 5e-3, ("tco2mic", e[-4:])
    w = want(z, d, "PROG")
    for k in ("tsoi", "tg", "tu", "tl", "ts", "ti", "tsno", "t12", "t34"):
        e = per_cell(prog[k], w[k], absolute=True)
        assert e[-1] < 3.0 and e[-4] < 0.2, (k, e[-4:])
    for k in ("wsoi", "wisoi"):
        e = per_cell(prog[k], w[k])
        assert e[-1] < 3e-2 and e[-4] < 2e-3, (k, e[-4:])


@pytest.mark.gpu
def test_day_loop_from_checkpoint_and_back(cuda_lib, tmp_path):
    """DayLoop.from_restart seeds columns, daily-cadence state and running sums
    from the 16-cell checkpoint; one float64 day (forcing as the reference
    made it) and DayLoop.save give a checkpoint whose leaves are the loop's
    state in the file's float32 and agree with the reference's own day loop to
    float32 storage (1e-6 outside the threshold cells)."""
    import torch
    from ibis_b200 import synth
    from ibis_b200.daily import DayLoop
    z, n, prog, stat, day, acc0, P = load_case()
    loop = DayLoop.from_restart(CKPT, dtype=torch.float64, params=P, day_params=day_params(z), lat=z["in.lat"],
                                seed=int(z["in.seed"]), jday=int(z["in.jday0"]), day=0)
    loop.params.flags = P.flags
    cols = loop.cols
    dd, daily = _daily_tensor(z, 0, cols.ld, torch)
    hours = hourly(z, 0, n)
    forc = {k: np.stack([F[k] for F in hours]) for k in hours[0]}
    td = torch.from_numpy(np.pad(dd["td"], (0, cols.ld - n))).cuda()
    loop.run_day(daily, forc=torch.from_numpy(synth.forcing_planes(forc, cols.ld, dtype=np.float64)).cuda(), td=td)
    torch.cuda.synchronize()
    path = tmp_path / "after_day.npz"
    loop.save(str(path))
    back, meta, _ = restart.load(str(path))
    orig, meta0, _ = restart.load(CKPT)
    assert meta == meta0
    keep = np.setdiff1d(np.arange(n), DAY_THRESHOLD_CELLS)
    acc = {k: v for k, v in cols.acc_host().items() if k in ACC_CHECK}
    for group, values in (("PROG", cols.prog_host()), ("DAYST", loop.dayst_host()), ("ACC", acc)):
        ref = want(z, 0, group)
        for f in L.GROUPS[group]:
            if f.leaf not in back or f.name not in ref or f.name not in values:
                continue
            mine = np.asarray(values[f.name]).astype(np.asarray(orig[f.leaf]).dtype).astype(np.float64)
            if np.size(back[f.leaf]) == 1:       # a scalar leaf holds the first cell's value
                mine = np.full(np.shape(ref[f.name]), mine.reshape(-1)[0])
            v = np.broadcast_to(np.asarray(back[f.leaf], np.float64), np.shape(ref[f.name]))
            v = v.reshape(np.shape(ref[f.name]))
            assert np.array_equal(v, mine.reshape(v.shape)), f.name
            assert not compare({f.name: v[keep]}, {f.name: ref[f.name][keep]}, 1e-6), (group, f.name)


@pytest.mark.gpu
def test_day_loop_from_checkpoint_with_modules(cuda_lib, tmp_path):
    """A checkpoint that carries the wetland state and the four calibration
    modules (the reference's own save_state): DayLoop.from_restart switches the
    modules on and loads the wetland planes; after one float64 day DayLoop.save
    writes the modules back advanced as the day loop advances them -- the
    acclimation state relaxed toward the day's temperature, the stress sums and
    day count grown by the last hour's stress and one day (the default
    threshold counts every day), the ET parts grown by the day's AET -- and
    the wetland state and smoothed stress as they were."""
    import torch
    from ibis_b200.daily import DayLoop
    from ibis_b200.params import FLAG_ETPARTS, FLAG_NEEPARTS
    z, n, prog, stat, day, acc0, P = load_case()
    ckpt = os.path.join(HERE, "golden", "restart_modules_16cells.npz")
    leaves0, _, _ = restart.load(ckpt)
    loop = DayLoop.from_restart(ckpt, dtype=torch.float64, params=P, day_params=day_params(z), lat=z["in.lat"],
                                seed=int(z["in.seed"]), jday=int(z["in.jday0"]), day=0)
    assert loop.day_params.seasonal_on == 1.0 and loop.day_params.stress_on == 1.0
    assert loop.params.flags & FLAG_ETPARTS and loop.params.flags & FLAG_NEEPARTS
    np.testing.assert_array_equal(loop.wet_host()["zwt"], leaves0["wetland.zwt"])
    dd, daily = _daily_tensor(z, 0, loop.cols.ld, torch)
    ay0 = loop.dayst_host()["ayaet"].copy()
    loop.run_day(daily)
    torch.cuda.synchronize()
    acc = loop.cols.acc_host()
    loop.save(str(tmp_path / "ck.npz"))
    back, _, extra = restart.load(str(tmp_path / "ck.npz"))
    assert extra == []
    f64 = lambda k: np.asarray(back[k], np.float64)
    x0 = np.asarray(leaves0["seasonal.acclim_x"], np.float64)
    np.testing.assert_allclose(f64("seasonal.acclim_x"), x0 + (dd["td"] - 273.16 - x0) / 10.93, rtol=1e-6)
    np.testing.assert_array_equal(back["stress.nday"], (np.asarray(leaves0["stress.nday"], np.float64) + 1.0)
                                  .astype(np.asarray(leaves0["stress.nday"]).dtype))
    np.testing.assert_allclose(f64("stress.aystressu"), np.asarray(leaves0["stress.aystressu"], np.float64)
                               + acc["stresstu_last"], rtol=1e-6)
    et = sum(f64("etparts." + k) - np.asarray(leaves0["etparts." + k], np.float64)
             for k in ("trans", "interc", "soilev", "snowsub"))
    np.testing.assert_allclose(et, loop.dayst_host()["ayaet"] - ay0, rtol=1e-5, atol=1e-5)
    for k in ("wetland.flux", "wetland.annual", "wetland.zwt", "stress.u_smooth"):
        np.testing.assert_array_equal(back[k], leaves0[k], err_msg=k)


@pytest.mark.gpu
def test_device_month_matches_oracle_month(cuda_lib):
    """Three days as a month with hourly wetland CH4: ibis_month_begin, the
    device day loop in float64, ibis_month_end (mean of the hourly fluxes, the
    carbon partition) against the oracle's day loop and oracle.month on the
    same inputs: 1e-9 outside the threshold cells."""
    import torch
    from ibis_b200 import synth
    from oracle import month as OM
    f_inund = np.random.default_rng(2).uniform(0.0, 1.0, 16)
    z, n, _, _, day0, _, P = load_case()
    *_, (d, prog, day, stat, acc) = list(oracle_days(f_inund=f_inund))
    P.flags |= FLAG_CH4
    nd = int(z["in.ndays"])
    wet0 = dict(flux=np.zeros(n), annual=np.zeros(n), zwt=np.zeros(n))
    ref, ay, take = OM.month_end(wet0, prog, stat, acc["ch4"], day["ayco2mic"], day0["ayco2mic"], nd,
                                 np.asarray(P.hsoi, np.float64), P, from_mean=True, partition=True)
    z, n, cols, loop, torch = _device_loop(torch.float64)
    loop.params.flags |= FLAG_CH4
    cols.stat[L.OFF["STAT"]["f_inund"][0], :n] = torch.from_numpy(f_inund).to(cols.stat)
    loop.begin_month(new_year=True)
    for d in range(nd):
        dd, daily = _daily_tensor(z, d, cols.ld, torch)
        hours = hourly(z, d, n)
        forc = {k: np.stack([F[k] for F in hours]) for k in hours[0]}
        td = torch.from_numpy(np.pad(dd["td"], (0, cols.ld - n))).cuda()
        loop.run_day(daily, forc=torch.from_numpy(synth.forcing_planes(forc, cols.ld, dtype=np.float64)).cuda(),
                     td=td)
    loop.end_month(nd, from_mean=True, partition=True)
    torch.cuda.synchronize()
    keep = np.setdiff1d(np.arange(n), DAY_THRESHOLD_CELLS)
    wet = loop.wet_host()
    got = {"flux": wet["flux"], "annual": wet["annual"], "zwt": wet["zwt"], "ch4c": wet["ch4c"],
           "ayco2mic": loop.dayst_host()["ayco2mic"]}
    want_ = {"flux": ref["flux"], "annual": ref["annual"], "zwt": ref["zwt"], "ch4c": take, "ayco2mic": ay}
    assert np.any(want_["flux"][keep] > 0.0) and np.any(take[keep] > 0.0)
    bad = compare({k: v[keep] for k, v in got.items()}, {k: v[keep] for k, v in want_.items()}, 1e-9)
    assert not bad, bad[:5]


_DAY_MAP_CHECK = r"""
import sys, numpy as np
sys.path.insert(0, "{golden}/jaxshim"); sys.path.insert(0, "{ref}"); sys.path.insert(0, "{golden}"); sys.path.insert(0, "{repo}")
import make_golden as mg
from ibis_b200 import dropin
from ibis_b200.params import DAY_PARAM_FIELDS
from ibis_b200.params import DayParams
z = np.load("{gold}")
sp = mg.loops.default_sim_params(16)
dp, defaults = dropin.day_params(sp), DayParams()
for name, path in dropin.DAY_PARAM_PATHS.items():
    assert dropin._get(dict(params=sp), path) is not None, path
    v = np.asarray(getattr(dp, name), float)
    ref = z["in.dparam." + name] if "in.dparam." + name in z.files else np.asarray(getattr(defaults, name), float)
    assert np.array_equal(v, ref), name
print("day mapping ok")
"""


@pytest.mark.skipif(not HAVE_REF, reason="reference sources not present (IBIS_REFERENCE)")
def test_day_param_paths_against_reference_objects():
    """dropin.DAY_PARAM_PATHS resolves every path on the reference's own
    SimParams, to the values the three-day fixture was run with and, for the
    module parameters, to the defaults DayParams restates."""
    import subprocess
    import sys
    code = _DAY_MAP_CHECK.format(golden=os.path.join(HERE, "golden"), ref=REF_PORT,
                                 repo=os.path.dirname(HERE), gold=GOLD)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and "day mapping ok" in r.stdout, r.stderr[-3000:]


def _param_tree(z, lat_deg):
    """consts/params attribute trees with the reference's paths, from the fixture's records."""
    from ibis_b200 import dropin

    def put(root, path, v):
        obj = root
        *head, last = path.split(".")
        for h in head:
            if not hasattr(obj, h):
                setattr(obj, h, types.SimpleNamespace())
            obj = getattr(obj, h)
        setattr(obj, last, v)

    root = types.SimpleNamespace()
    for name, path in dropin.PARAM_PATHS.items():
        if path.startswith(("params.", "consts.")) and "in.param." + name in z:
            v = z["in.param." + name]
            put(root, path, v if np.size(v) > 1 else float(v))
    for name, path in dropin.DAY_PARAM_PATHS.items():
        if "in.dparam." + name not in z:
            continue
        v = z["in.dparam." + name]
        put(root, path, v if np.size(v) > 1 else float(v))
    put(root, "params.latitude", np.deg2rad(lat_deg))
    put(root, "params.h2o_consistent_weights", bool(int(z["in.param.flags"]) & 2))
    return root.consts, root.params


@pytest.mark.gpu
def test_run_month_scan_dropin_equals_day_loop(cuda_lib):
    """dropin.run_month_scan over the checkpoint's own state tree (float32, as
    the reference's day loop runs) and the fixture's three days of weather:
    the same bits as DayLoop on the same inputs, daily outputs equal to the
    differences of the annual sums, and the state within the float32 day
    loop's bounds of the reference's float64 run."""
    import torch
    from ibis_b200 import dropin
    from ibis_b200.daily import DayLoop
    z = load_case()[0]
    n, nd = 16, int(z["in.ndays"])
    leaves, _, _ = restart.load(CKPT)
    state = restart.as_tree({k: (np.asarray(v).copy() if v is not None else None) for k, v in leaves.items()})
    for k in ("z0sno", "rhos", "consno", "hsnotop", "hsnomin", "fimin", "fimax"):
        setattr(state.snow, k, np.float32(z["in.param." + k]))      # the reference takes these from its template
    consts, params = _param_tree(z, z["in.lat"])
    days = [day_weather(z, d) for d in range(nd)]
    xs = tuple(np.stack([dd[k] for dd in days]) for k in ("td", "tmax", "tmin", "cloud", "precip", "psurf", "qd",
                                                         "ud")) + (np.zeros((nd, n)),
                                                                   np.stack([dd["fira"] for dd in days]),
                                                                   int(z["in.jday0"]) + np.arange(nd))
    seed = int(z["in.seed"])
    new, (gpp, aet, rh) = dropin.run_month_scan(state, consts, params, xs, 1, 365, 3600.0, seed=seed)
    # with the hourly CH4 and the soil means the day outputs gain them, per day
    _, extra = dropin.run_month_scan(state, consts, params, xs, 1, 365, 3600.0, seed=seed, ch4_hourly=True,
                                     ch4_args=(np.full(n, 0.3), types.SimpleNamespace(), None), soil_means=True)
    assert len(extra) == 8 and extra[3].shape == (nd, n) and extra[4].shape == (nd, n, 6)
    assert extra[7].shape == (nd, n) and np.all(extra[3] >= 0) and np.any(extra[3] > 0)
    np.testing.assert_allclose(extra[7], np.broadcast_to(extra[7].mean(axis=0), extra[7].shape), rtol=0.05)
    assert np.all((extra[7] > 200.0) & (extra[7] < 340.0))           # day-mean ground temperature, K
    # the same days through DayLoop directly
    P = dropin.step_params(state, consts, params, 3600.0, 365)
    loop = DayLoop.from_restart(CKPT, dtype=torch.float32, params=P, day_params=dropin.day_params(params),
                                lat=z["in.lat"], seed=seed, jday=int(z["in.jday0"]), day=0)
    loop.params.flags = P.flags | FLAG_ACC
    from ibis_b200 import forcing
    daily = torch.from_numpy(forcing.daily_planes({k: np.stack([dd[k] for dd in days]) for k in days[0]},
                                                  loop.cols.ld)).cuda()
    loop.run(daily)
    torch.cuda.synchronize()
    prog = loop.cols.prog_host()
    for f in L.PROG:
        v = dropin._get({"s": new}, "s." + f.leaf)
        if v is None or f.name not in prog:
            continue
        mine = np.asarray(prog[f.name]).astype(np.float32)
        if np.ndim(v) == 0:
            mine = mine.reshape(-1)[0]
        assert np.array_equal(np.asarray(v), mine.reshape(np.shape(v))), f.name
    dayst = loop.dayst_host()
    for f in L.DAYST:
        v = dropin._get({"s": new}, "s." + f.leaf)
        if v is None:                   # the optional modules, and the latitude (a parameter)
            continue
        v = np.asarray(v, np.float64)
        assert np.array_equal(v.reshape(-1), np.asarray(dayst[f.name], np.float32).astype(np.float64).reshape(-1)), \
            f.name
    ay0 = np.asarray(leaves["summary.ayaet"], np.float64)
    np.testing.assert_allclose(np.cumsum(aet, axis=0)[-1], dayst["ayaet"] - ay0, rtol=1e-5, atol=1e-6)
    assert gpp.shape == (nd, n) and rh.shape == (nd, n) and np.isfinite(gpp).all() and np.isfinite(rh).all()
    w = want(z, nd - 1, "DAYST")
    for k in ("tempu", "templ", "agddu", "agddl", "a10td", "ayprcp", "csoipas", "totcsoi"):
        e = np.abs(np.asarray(dayst[k]) - w[k]) / np.maximum(np.abs(w[k]), 1e-3)
        assert e.max() < 1e-4, (k, float(e.max()))


@pytest.mark.gpu
def test_run_month_scan_dropin_with_state_modules(cuda_lib):
    """dropin.run_month_scan over a float32 state tree that carries the
    reference's optional modules (seasonal, stress, ET parts, NEE parts) and
    parameters with photoperiod-gated senescence: the modules advance and are
    written back.  Against the reference's float64 run of the same three days:
    the seasonal states (functions of the daily mean temperature and the day
    length) within 1e-5, the day counts exact, the stress sums within 1e-3
    (the stress of the float32 step), transpiration and interception loss
    within 1e-3 of their largest magnitude on 90 % of the cells, the net NEE
    within 2e-2 of its largest magnitude, and the four ET parts summing to the
    AET booked over the days.  The float64
    day loop checks every part against the reference to 1e-9
    (test_device_day_loop_with_modules_matches_reference_days)."""
    from ibis_b200 import dropin
    z = load_case(GOLD_MODULES)[0]
    n, nd = 16, int(z["in.ndays"])
    leaves, _, _ = restart.load(CKPT)
    state = restart.as_tree({k: (np.asarray(v).copy() if v is not None else None) for k, v in leaves.items()})
    for k in ("z0sno", "rhos", "consno", "hsnotop", "hsnomin", "fimin", "fimax"):
        setattr(state.snow, k, np.float32(z["in.param." + k]))
    f = lambda leaf: np.asarray(z["in." + leaf], np.float32)
    state.seasonal = types.SimpleNamespace(acclim_x=f("seasonal.acclim_x"), ssen_u=f("seasonal.ssen_u"),
                                           ssen_l=f("seasonal.ssen_l"))
    state.stress = types.SimpleNamespace(aystressu=f("stress.aystressu"), aystressl=f("stress.aystressl"),
                                         nday=f("stress.nday"), u_smooth=np.zeros(n, np.float32))
    zero = np.zeros(n, np.float32)
    state.etparts = types.SimpleNamespace(trans=zero, interc=zero, soilev=zero, snowsub=zero)
    state.neeparts = types.SimpleNamespace(night=zero, day=zero)
    consts, params = _param_tree(z, z["in.lat"])
    assert params.pheno.sen_photoperiod_u == 1.0
    days = [day_weather(z, d) for d in range(nd)]
    xs = tuple(np.stack([dd[k] for dd in days]) for k in ("td", "tmax", "tmin", "cloud", "precip", "psurf", "qd",
                                                         "ud")) + (np.zeros((nd, n)),
                                                                   np.stack([dd["fira"] for dd in days]),
                                                                   int(z["in.jday0"]) + np.arange(nd))
    new, _ = dropin.run_month_scan(state, consts, params, xs, 1, 365, 3600.0, seed=int(z["in.seed"]))
    w = lambda leaf: z[f"out.{nd - 1}.{leaf}"]
    for leaf in ("seasonal.acclim_x", "seasonal.ssen_u", "seasonal.ssen_l"):
        np.testing.assert_allclose(dropin._get({"s": new}, "s." + leaf), w(leaf), rtol=1e-5, atol=1e-4, err_msg=leaf)
    np.testing.assert_array_equal(new.stress.nday, w("stress.nday"))
    for leaf in ("stress.aystressu", "stress.aystressl"):
        np.testing.assert_allclose(dropin._get({"s": new}, "s." + leaf), w(leaf), rtol=0, atol=1e-3, err_msg=leaf)
    assert np.any(new.seasonal.ssen_u >= 25.0) and np.any(new.seasonal.ssen_u == 0.0)
    close = lambda g, ref: np.mean(np.abs(g - ref) <= 1e-3 * max(float(np.abs(ref).max()), 1e-30)) >= 0.9
    for leaf in ("etparts.trans", "etparts.interc"):
        assert close(np.asarray(dropin._get({"s": new}, "s." + leaf), np.float64), w(leaf)), leaf
    # an hour whose float32 sun height sits at the horizon books its NEE to the
    # other side of the night/day split, and the net is a small difference of
    # GPP-sized terms: the sum is compared, within 2e-2 of its largest magnitude
    net = np.asarray(new.neeparts.night, np.float64) + new.neeparts.day
    net_ref = w("neeparts.night") + w("neeparts.day")
    assert np.all(np.abs(net - net_ref) <= 2e-2 * np.abs(net_ref).max()), np.abs(net - net_ref).max()
    # soil evaporation and snow sublimation split on the snow cover, which the
    # float32 day with generated forcing moves in single cells; their sum with
    # the other two parts is the AET the state booked over the days
    et = sum(np.asarray(getattr(new.etparts, k), np.float64) for k in ("trans", "interc", "soilev", "snowsub"))
    np.testing.assert_allclose(et, np.asarray(new.summary.ayaet, np.float64) - leaves["summary.ayaet"],
                               rtol=1e-4, atol=1e-4)
    assert state.seasonal.acclim_x is not new.seasonal.acclim_x
