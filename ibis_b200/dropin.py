"""Drop-in for the reference's step function (and its day loop) over its own state pytrees.

The reference's hot path is one pure function,

    timestep_body(state, consts, params, dtime) -> state

(python-port/ibis/timestepping/loops.py:234-284) over Equinox pytrees:
``IBISState`` (state/model_state.py:28-63), ``PhysicalConstants``
(constants.py:16-80) and ``SimParams`` (loops.py:72-134).  It has no operator,
plugin or FFI layer.  :func:`timestep_body` here has the same signature and
meaning: it reads the leaves the step needs from those objects (by attribute
path, so any object with the same paths works), advances them one hour with
the CUDA kernels, and returns a state of the same structure whose prognostic
leaves are the new values and whose diagnostic leaves are the ones
``timestep_body`` writes (loops.py:1158-1241).  Float64 leaves run the float64
kernels; float32 leaves the production FP32 kernels.

:func:`run_hours` is the multi-hour form with the day loop's accumulators
(``_run_day_inner._step_body``, loops_gswp3.py:115-320): one launch for all
hours, forcing given as arrays instead of the reference's weather generator.
:func:`run_month_scan` runs whole days of the GSWP3 day loop
(``_run_month_scan``, loops_gswp3.py:346-612) from the days' weather.

The leaves are copied to and from the device on every call (the reference's
contract is a host-visible pytree); :class:`ibis_b200.columns.Columns` keeps
state resident for callers that can.
"""
from __future__ import annotations

import copy
import dataclasses
import os

import numpy as np
import torch

from . import layout as L
from .columns import Columns
from .params import (FLAG_ACC, FLAG_ACCLIM, FLAG_ACCLIM_LIGHT, FLAG_BEDROCK, FLAG_CAP_SCALE_L, FLAG_CAP_SCALE_U,
                     FLAG_CH4, FLAG_COEFM_MIX, FLAG_CROP, FLAG_ETPARTS, FLAG_FORGANIC, FLAG_FROST,
                     FLAG_GPP_CAPACITY, FLAG_H2O_CONSISTENT, FLAG_LEAF_ONLY, FLAG_NEEPARTS, FLAG_SOIL_MEANS,
                     FLAG_SUNSHADE_L, FLAG_SUNSHADE_U, FLAG_VMAX_MIX, StepParams)

# Where each parameter of the flat record lives in the reference's objects.
# Roots: consts (PhysicalConstants), params (SimParams), state (IBISState).
PARAM_PATHS = {
    **{k: f"consts.{k}" for k in ("stef", "vonk", "grav", "tmelt", "hvap", "hfus", "hsub", "ch2o", "cice", "cair",
                                  "cvap", "rair", "rvap", "cappa", "rhow", "epsilon")},
    "co2conc": "state.atm.co2conc",
    **{k: f"state.snow.{k}" for k in ("z0sno", "rhos", "consno", "hsnotop", "hsnomin", "fimin", "fimax")},
    **{k: f"params.veg_rad.{k}" for k in ("rhoveg", "tauveg", "oriev", "orieh")},
    **{k: f"params.canopy.{k}" for k in ("cleaf", "cstem", "cgrass", "dleaf", "dstem", "alaiml", "alaimu", "chu",
                                         "chs", "chl", "soil_beta_power")},
    **{k: f"params.interception.{k}" for k in ("wliqumax", "wliqsmax", "wliqlmax", "wsnoumax", "wsnosmax",
                                               "wsnolmax", "tdripu", "tdrips", "tdripl", "tblowu", "tblows",
                                               "tblowl", "fmax")},
    **{k: f"params.stomata_params.{k}" for k in ("tau15", "kc15", "ko15", "cimax", "o2conc", "alpha3", "theta3",
                                                 "beta3", "alpha4", "theta4", "beta4", "gamma", "coefm", "coefb",
                                                 "gsmin", "vmax_pft", "stressfac", "cap_kn", "coefm_pft",
                                                 "frost_t0", "frost_t1")},
    **{f"crop_{k}": f"params.crop.{k}" for k in ("vmax_scale_c3", "vmax_scale_c4", "c4_share")},
    **{k: f"params.{k}" for k in ("wpudmax", "zwpmax", "bperm", "rhosoi_val", "csoi_mineral_val")},
    "hsoi": "state.soil.hsoi",
    "froot": "state.vegetation.froot",
    "hsoi_bed": "params.bedrock.hsoi", "consoi_bed": "params.bedrock.consoi",
    "rhosoi_bed": "params.bedrock.rhosoi", "csoi_bed": "params.bedrock.csoi",
    **{k: f"params.fire.{k}" for k in ("d_crit", "vpd_ref", "d_crit_vpd")},
    **{k: f"params.methane.{k}" for k in ("sat_crit", "z_max", "r_ch4", "q10p", "t_ref", "z_wt_max", "z_wt_ref",
                                          "z_tau", "tau_oxid")},
    **{k: f"params.bgc_params.{k}" for k in ("rwood", "rroot", "rgrowth")},
}
# Not parameters of the reference objects: omegasno is a module constant of the
# radiation code (radiation.py:393, _OMEGASNO); flux_max and t_max_dev are read
# from the environment when the step is traced (loops.py:665, 1143); dtime and
# the year length are arguments.
_ENV = {"flux_max": ("IBIS_FLUX_MAX", 2000.0), "t_max_dev": ("IBIS_T_MAX_DEV", 40.0)}


def _get(roots: dict, path: str):
    root, *rest = path.split(".")
    obj = roots[root]
    for part in rest:
        if obj is None:
            return None
        obj = getattr(obj, part, None)
    return obj


def _replace(obj, name, value):
    """A copy of ``obj`` with attribute ``name`` set (dataclass / eqx.Module,
    NamedTuple, or plain object)."""
    if dataclasses.is_dataclass(obj) and not isinstance(obj, type):
        try:
            return dataclasses.replace(obj, **{name: value})
        except (TypeError, ValueError):
            pass
    if hasattr(obj, "_replace") and hasattr(obj, "_fields"):
        return obj._replace(**{name: value})
    new = copy.copy(obj)
    object.__setattr__(new, name, value)
    return new


def tree_set(root, path: str, value):
    """``root`` with the leaf at dotted ``path`` replaced (like ``eqx.tree_at``)."""
    head, _, tail = path.partition(".")
    if not tail:
        return _replace(root, head, value)
    return _replace(root, head, tree_set(getattr(root, head), tail, value))


# StomataParams switches (stomata.py:98-159) -> the step's variant flags.  Every
# switch of the reference's stomata formulation has one; acclim_on acts only on a
# state that carries the seasonal module (loops.py:294) and frost_on only with it
# (loops.py:305).
SWITCH_FLAGS = {"vmax_mix": FLAG_VMAX_MIX, "coefm_mix": FLAG_COEFM_MIX, "gpp_split_by_capacity": FLAG_GPP_CAPACITY,
                "acclim_light": FLAG_ACCLIM_LIGHT, "cap_scale_u": FLAG_CAP_SCALE_U, "cap_scale_l": FLAG_CAP_SCALE_L,
                "scale_leaf_only": FLAG_LEAF_ONLY, "sunshade_u": FLAG_SUNSHADE_U, "sunshade_l": FLAG_SUNSHADE_L}
# Switches the step does not carry: none.  Per-cell PFT tables (the IBIS 3.0
# zone types, io/pft_types.py) are refused by step_params instead.
UNSUPPORTED_SWITCHES: tuple = ()
# Per-PFT tables that IBIS 3.0 zone types make per-cell (npoi, 12)
_PFT_TABLES = ("params.stomata_params.vmax_pft", "params.stomata_params.coefm_pft",
               "params.stomata_params.acclim_s0_pft", "params.stomata_params.acclim_smax_pft",
               "params.bgc_params.rwood", "params.bgc_params.rroot", "params.bgc_params.rgrowth")


def _stomata_flags(state, params, sp) -> int:
    flags = 0
    for name, flag in SWITCH_FLAGS.items():
        if bool(getattr(sp, name, False)):
            flags |= flag
    if bool(getattr(sp, "acclim_on", False)) and getattr(state, "seasonal", None) is not None:
        flags |= FLAG_ACCLIM
        if bool(getattr(sp, "frost_on", False)):
            flags |= FLAG_FROST
    if getattr(params, "cropfrac", None) is not None:
        flags |= FLAG_CROP
    if getattr(params, "forganic", None) is not None:
        flags |= FLAG_FORGANIC
    return flags


def step_params(state, consts, params, dtime: float, ndaypy: float = 365.0) -> StepParams:
    """The flat parameter record (and variant flags) equivalent to the reference
    objects.  Raises NotImplementedError for per-cell PFT tables (IBIS 3.0
    zone types), which the step does not carry."""
    sp = getattr(params, "stomata_params", None)
    roots = {"state": state, "consts": consts, "params": params}
    for path in _PFT_TABLES:
        v = _get(roots, path)
        if v is not None and np.ndim(v) == 2:
            raise NotImplementedError(f"per-cell PFT table {path} (IBIS 3.0 zone types) is not implemented")
    P = StepParams()
    for name, path in PARAM_PATHS.items():
        v = _get(roots, path)
        if v is None or name in _METHANE_FIELDS:
            continue
        n = np.size(getattr(P, name))
        arr = np.asarray(v, dtype=np.float64).reshape(-1)
        if name == "hsoi":
            arr = arr[:L.NSOILAY]
        if n > 1 and arr.size == 1:
            arr = np.full(n, arr[0])
        setattr(P, name, arr if n > 1 else float(arr[0]))
    mp = getattr(params, "methane", None)
    if mp is not None:
        ncell = int(np.size(np.asarray(state.soil.tg)))
        apply_methane(P, {}, mp, ncell)
    for name, (env, default) in _ENV.items():
        setattr(P, name, float(os.environ.get(env, default)))
    P.dtime = float(dtime)
    P.ndaypy = float(ndaypy)
    # the acclimated PFTs as a mask, and the acclimation constants per PFT (the
    # scalars repeated when acclim_per_pft is off: the same arithmetic, loops.py:295-303)
    if sp is not None:
        mask = np.zeros(12)
        for k in tuple(getattr(sp, "acclim_pfts", (3, 5, 8))):
            mask[int(k)] = 1.0
        P.acclim_mask = mask
        if bool(getattr(sp, "acclim_per_pft", False)):
            P.acclim_s0_pft = np.asarray(sp.acclim_s0_pft, dtype=np.float64).reshape(12)
            P.acclim_smax_pft = np.asarray(sp.acclim_smax_pft, dtype=np.float64).reshape(12)
        else:
            P.acclim_s0_pft = np.full(12, float(getattr(sp, "acclim_s0", -3.063)))
            P.acclim_smax_pft = np.full(12, float(getattr(sp, "acclim_smax", 17.72)))
    flags = _stomata_flags(state, params, sp)
    if getattr(state.soil, "tsoi_deep", None) is not None:
        flags |= FLAG_BEDROCK
    if bool(getattr(params, "h2o_consistent_weights", False)):
        flags |= FLAG_H2O_CONSISTENT
    P.flags = flags
    return P


def methane_sets(mp, ncell):
    """A reference ``MethaneParams`` as the step takes it: ``(values, None)``
    when every field is one value, or ``(tables, band)`` when fields are
    per-cell arrays (``biome_methane_params``, methane.py:521-563): the cells'
    distinct parameter sets -- at most three, one per wetland band -- as the
    ``ch4b_*`` tables and each cell's set as its ch4_band value."""
    fields = [k for k in _METHANE_FIELDS if getattr(mp, k, None) is not None]
    if not any(np.size(getattr(mp, k)) > 1 for k in fields):
        return {k: float(np.asarray(getattr(mp, k)).reshape(-1)[0]) for k in fields}, None
    rows = np.stack([np.broadcast_to(np.asarray(getattr(mp, k), np.float64).reshape(-1) if np.size(getattr(mp, k)) > 1
                                     else np.asarray(getattr(mp, k), np.float64), (ncell,)) for k in fields], axis=1)
    sets, band = np.unique(rows, axis=0, return_inverse=True)
    if len(sets) > 3:
        raise NotImplementedError(f"per-cell methane parameters in {len(sets)} distinct sets (the step takes up to "
                                  "three bands, as biome_methane_params forms them)")
    tables = {k: [float(sets[min(b, len(sets) - 1), j]) for b in range(3)] for j, k in enumerate(fields)}
    if "z_wt_ref" in tables and len(set(tables["z_wt_ref"])) > 1:
        raise NotImplementedError("per-cell z_wt_ref (the reference's water table takes one)")
    return tables, np.asarray(band, np.float64).reshape(ncell)


def apply_methane(P, stat, mp, ncell):
    """Put ``methane_sets(mp)`` into the step's record ``P`` (scalars, or the
    per-band tables with FLAG_CH4_BANDS and the first set as the scalars) and
    the STAT dict ``stat`` (the ch4_band plane)."""
    from .params import FLAG_CH4_BANDS
    vals, band = methane_sets(mp, ncell)
    if band is None:
        for k, v in vals.items():
            setattr(P, k, v)
        P.flags &= ~FLAG_CH4_BANDS
        return
    for k, t in vals.items():
        setattr(P, "ch4b_" + k, np.asarray(t, np.float64))
        setattr(P, k, t[0])
    P.flags |= FLAG_CH4_BANDS
    stat["ch4_band"] = band


def _stat_dict(state, params, ncell):
    """STAT planes of ``state`` plus the per-cell SimParams arrays the step reads
    (``cropfrac``, ``forganic``: the layout's ``sim.`` leaves) and, where the
    methane parameters are per cell, their band plane."""
    stat = _leaf_dict(state, "STAT", ncell)
    for f in L.STAT:
        if f.leaf.startswith("sim."):
            v = getattr(params, f.leaf[4:], None)
            if v is not None:
                stat[f.name] = np.asarray(v, dtype=np.float64).reshape((ncell,) + ((f.k,) if f.k > 1 else ()))
    mp = getattr(params, "methane", None)
    if mp is not None:
        _, band = methane_sets(mp, ncell)
        if band is not None:
            stat["ch4_band"] = band
    return stat


def _leaf_dict(state, group, ncell):
    out = {}
    for f in L.GROUPS[group]:
        v = _get({"state": state}, "state." + f.leaf)
        if v is None:
            continue
        a = np.asarray(v, dtype=np.float64)
        if a.ndim == 0:
            a = np.full(ncell, float(a))
        out[f.name] = a
    return out


def _dtype_of(state):
    return torch.float32 if np.asarray(state.soil.tg).dtype == np.float32 else torch.float64


def _write_back(state, values: dict, group: str, dtype):
    np_dtype = np.float32 if dtype == torch.float32 else np.float64
    for f in L.GROUPS[group]:
        if f.name not in values:
            continue
        old = _get({"state": state}, "state." + f.leaf)
        if old is None:          # a leaf this state does not carry (no bedrock, extra diagnostics)
            continue
        v = np.asarray(values[f.name]).astype(np_dtype)
        if old is not None and np.ndim(old) == 0:
            v = np_dtype(v.reshape(-1)[0])
        state = tree_set(state, f.leaf, v)
    return state


def timestep_body(state, consts, params, dtime: float, device="cuda"):
    """One hourly step of ``state`` (same contract as the reference's ``timestep_body``)."""
    P = step_params(state, consts, params, dtime)
    ncell = int(np.asarray(state.soil.tg).shape[0])
    dtype = _dtype_of(state)
    prog = _leaf_dict(state, "PROG", ncell)
    stat = _stat_dict(state, params, ncell)
    forc = {k: v[None] for k, v in _leaf_dict(state, "FORC", ncell).items()}
    cols = Columns.from_host(prog, stat, dtype=dtype, device=device, diag=True, acc=False)
    cols.run(cols.forcing(forc), P)
    torch.cuda.synchronize(cols.device)
    status = cols.nonfinite()
    state = _write_back(state, cols.prog_host(), "PROG", dtype)
    state = _write_back(state, cols.diag_host(), "DIAG", dtype)
    if status[0]:
        import warnings
        warnings.warn(f"non-finite state after the step (first cell {status[1]})", RuntimeWarning)
    return state


_PARTS = ("et_trans", "et_interc", "et_soilev", "et_snowsub", "nee_night", "nee_day")


def parts_flags(state) -> int:
    """FLAG_ETPARTS / FLAG_NEEPARTS for the optional modules ``state`` carries:
    the reference sums the ET components and the day/night NEE only when
    ``state.etparts`` / ``state.neeparts`` is attached (loops_gswp3.py:265, 276)."""
    return (FLAG_ETPARTS if getattr(state, "etparts", None) is not None else 0) | \
        (FLAG_NEEPARTS if getattr(state, "neeparts", None) is not None else 0)


def run_hours(state, consts, params, forcing: dict, dtime: float, ch4_inund=None, soil_means: bool = False,
              ndaypy: float = 365.0, acc=None, device="cuda"):
    """``nhour`` hourly steps with the day loop's accumulators, in one launch.

    ``forcing`` maps the ``atm`` leaf names of ``layout.FORC`` to (nhour, ncell[, k])
    arrays.  ``ch4_inund`` (per-cell inundated fraction) turns on the hourly
    wetland CH4 accumulator.  ``acc`` is a previous return value to continue
    from.  Returns ``(state, acc)`` with ``acc`` a dict of the ``layout.ACC``
    accumulators (value and Kahan planes kept for continuation).  The ET and
    NEE components of a state that carries ``etparts`` / ``neeparts`` are
    summed on top of the state's values and written back into it, as the
    reference's step body does."""
    P = step_params(state, consts, params, dtime, ndaypy)
    P.flags = P.flags | FLAG_ACC | (FLAG_CH4 if ch4_inund is not None else 0) | (FLAG_SOIL_MEANS if soil_means else 0)
    P.flags |= parts_flags(state)
    ncell = int(np.asarray(state.soil.tg).shape[0])
    dtype = _dtype_of(state)
    if dtype == torch.float64:
        P.flags = P.flags & ~(1 << 8)        # plain sums in float64
    prog = _leaf_dict(state, "PROG", ncell)
    stat = _stat_dict(state, params, ncell)
    if ch4_inund is not None:
        stat["f_inund"] = np.asarray(ch4_inund, dtype=np.float64)
    cols = Columns.from_host(prog, stat, dtype=dtype, device=device, acc=True)
    parts = {k: v for k, v in _leaf_dict(state, "ACC", ncell).items() if k in _PARTS}
    if acc is not None:
        cols.acc.copy_(torch.as_tensor(acc["_planes"], dtype=dtype))
    elif parts:
        cols.set_acc(parts)
    cols.run(cols.forcing(forcing), P)
    torch.cuda.synchronize(cols.device)
    state = _write_back(state, cols.prog_host(), "PROG", dtype)
    out = cols.acc_host(compensated=True)
    state = _write_back(state, {k: out[k] for k in parts}, "ACC", dtype)
    out["_planes"] = cols.acc.cpu().numpy().copy()
    return state, out


# Where each daily-cadence parameter lives in the reference's SimParams:
# phenology (physics/phenology.py:20, PhenoParams) and soil biogeochemistry
# (io/parameters.py:176, BGCParams; ``bgc_fmax`` is its ``fmax``).
def _day_param_paths():
    from .params import DAY_LOOP_FIELDS, DAY_PARAM_FIELDS
    names = [n for n, _, _ in DAY_PARAM_FIELDS if n not in DAY_LOOP_FIELDS]
    pheno = names[:names.index("lig_frac")]
    out = {n: (f"params.pheno.{n}" if n in pheno else f"params.bgc_params.{'fmax' if n == 'bgc_fmax' else n}")
           for n in names}
    out["acclim_tau"] = "params.stomata_params.acclim_tau"
    return out


DAY_PARAM_PATHS = _day_param_paths()
_METHANE_FIELDS = ("sat_crit", "z_max", "r_ch4", "q10p", "t_ref", "z_wt_max", "z_wt_ref", "z_tau", "tau_oxid")


def day_params(params):
    """The daily-cadence parameter record equivalent to a reference ``SimParams``."""
    from .params import DayParams
    DP = DayParams()
    for name, path in DAY_PARAM_PATHS.items():
        v = _get({"params": params}, path)
        if v is not None:
            setattr(DP, name, np.asarray(v, dtype=np.float64) if np.size(v) > 1 else float(np.asarray(v)))
    return DP


def run_month_scan(state, consts, params, xs, nsoilcall: int, ndaypy: int, dtime: float, nband: int = 2,
                   obs_sw: bool = False, ch4_hourly: bool = False, ch4_args=None, soil_means: bool = False,
                   seed: int = 0, day0: int = 0, device="cuda"):
    """Days of the reference's GSWP3 day loop on the GPU, with the arguments of
    its ``_run_month_scan`` (python-port/ibis/timestepping/loops_gswp3.py:346-612):
    ``xs`` = (td, tmax, tmin, cloud, precip, psurf, qd, ud, iwet, rlds, jdays[,
    sw_h, use_h]) as (ndays, npoi) arrays (sw_h (ndays, 24, npoi)).  Returns
    ``(state, daily)``: ``daily`` is the reference's per-day output -- GPP, AET
    and Rh, then with ``ch4_hourly`` the CH4 day mean and with ``soil_means``
    the day means of tsoi, wsoi, wisoi (ndays, npoi, 6) and tg.  The reference
    also returns its PRNG key, which has no counterpart here: the day's
    variates (event timing, hourly wind) come from the counter-based generator
    keyed by (``seed``, ``day0`` + day, cell) instead of ``jax.random``.

    Supported: one soil-BGC call per day (``nsoilcall`` 1), two radiation
    bands, no per-cell growth habits (``slot_habit``); the optional state
    modules the state carries (stress, ET parts, seasonal states with
    photoperiod-gated senescence, NEE parts) advance as in the reference, and
    the step's acclimation reads the seasonal state each day's start leaves.
    ``iwet`` is not used (the reference's day loop does not read it either)."""
    from . import forcing as _forcing
    from .daily import DayLoop
    if int(nsoilcall) != 1 or int(nband) != 2:
        raise NotImplementedError("one soil-BGC call per day and two radiation bands only")
    if getattr(params, "slot_habit", None) is not None:
        raise NotImplementedError("per-cell growth habits (params.slot_habit) are not implemented")
    xs = [np.asarray(x) for x in xs]
    td, tmax, tmin, cloud, precip, psurf, qd, ud, _iwet, rlds, jdays = xs[:11]
    sw_h = use_h = None
    if obs_sw:
        sw_h, use_h = xs[11], xs[12]
    nday, ncell = td.shape
    P = step_params(state, consts, params, dtime, ndaypy)
    P.flags |= FLAG_ACC | (FLAG_SOIL_MEANS if soil_means else 0) | parts_flags(state)
    dtype = _dtype_of(state)
    prog = _leaf_dict(state, "PROG", ncell)
    stat = _stat_dict(state, params, ncell)
    if ch4_hourly and ch4_args is not None:
        from .params import FLAG_ZWT_OBS
        f_inund, mp, zwt_obs = ch4_args
        P.flags |= FLAG_CH4
        stat["f_inund"] = np.asarray(f_inund, dtype=np.float64)
        stat.pop("ch4_band", None)
        apply_methane(P, stat, mp, ncell)
        if zwt_obs is not None:
            P.flags |= FLAG_ZWT_OBS
            stat["zwt_obs"] = np.asarray(zwt_obs, dtype=np.float64)
    cols = Columns.from_host(prog, stat, dtype=dtype, device=device, acc=True)
    acc0 = _leaf_dict(state, "ACC", ncell)
    cols.set_acc({k: v for k, v in acc0.items() if not k.startswith("a10anc")})
    lat = np.rad2deg(np.asarray(_get({"params": params}, "params.latitude"), dtype=np.float64)).reshape(ncell)
    DP = day_params(params)
    # the optional modules of the daily cadence advance when the state carries
    # them (loops_gswp3.py:423, 589)
    DP.seasonal_on = float(getattr(state, "seasonal", None) is not None)
    DP.stress_on = float(getattr(state, "stress", None) is not None)
    loop = DayLoop(cols, P, DP, _leaf_dict(state, "DAYST", ncell), lat=lat, seed=seed,
                   jday=int(jdays[0]), day=day0, dtime=dtime, observed_fira=True)
    daily = {"td": td, "tmax": tmax, "tmin": tmin, "cloud": cloud, "precip": precip, "psurf": psurf, "qd": qd,
             "ud": ud, "fira": rlds}
    d_daily = torch.from_numpy(_forcing.daily_planes(daily, cols.ld)).to(cols.device)
    ld = cols.ld
    # running totals read at every day's end; the day's value is the difference
    # (annual GPP, AET and Rh; with the options the CH4 day mean and the soil
    # means, which the step sums across days here and per day in the reference)
    acc_fields = ["aygpptot"] + (["ch4"] if P.flags & FLAG_CH4 else []) + \
        (["tsoi_mean", "wsoi_mean", "wisoi_mean", "tg_mean"] if soil_means else [])
    acc_planes = [p for f in acc_fields for p in range(L.OFF["ACC"][f][0], L.OFF["ACC"][f][0] + L.OFF["ACC"][f][1])]
    day_planes = [L.OFF["DAYST"]["ayaet"][0], L.OFF["DAYST"]["ayco2mic"][0]]
    sums = torch.zeros((nday + 1, len(acc_planes) + 2, ld), dtype=dtype, device=cols.device)
    acc_idx = torch.tensor(acc_planes, device=cols.device)
    day_idx = torch.tensor(day_planes, device=cols.device)

    def snap(i):
        sums[i, :len(acc_planes)] = cols.acc[acc_idx] - cols.acc[acc_idx + L.N_ACC]
        sums[i, len(acc_planes):] = loop.dayst[day_idx]

    snap(0)
    for d in range(nday):
        kw = {}
        if sw_h is not None:
            sw = np.zeros((sw_h.shape[1], ld), np.float32)
            sw[:, :ncell] = sw_h[d]
            use = np.zeros(ld, np.uint8)
            use[:ncell] = np.asarray(use_h[d], dtype=bool)
            kw = dict(sw_obs=torch.from_numpy(sw).to(cols.device), use=torch.from_numpy(use).to(cols.device))
        loop.run_day(d_daily[d], **kw)
        snap(d + 1)
    torch.cuda.synchronize(cols.device)
    s = np.diff(sums.cpu().numpy().astype(np.float64)[:, :, :ncell], axis=0)      # (nday, planes, ncell)
    na = len(acc_planes)
    diag = (s[:, 0], s[:, na], s[:, na + 1])
    j = 1
    for f in acc_fields[1:]:
        k = L.OFF["ACC"][f][1]
        v = s[:, j:j + k]
        diag += (v[:, 0] if k == 1 else np.transpose(v, (0, 2, 1)),)
        j += k
    from . import synth
    st = synth.from_planes("STAT", cols.stat.cpu().numpy(), ncell)
    stat_now = {k: st[k] for k in DayLoop._STAT_WRITTEN}
    acc = {k: v for k, v in cols.acc_host().items() if not k.startswith("a10anc")}
    state = _write_back(state, cols.prog_host(), "PROG", dtype)
    state = _write_back(state, stat_now, "STAT", dtype)
    state = _write_back(state, acc, "ACC", dtype)
    state = _write_back(state, loop.dayst_host(), "DAYST", dtype)
    return state, diag
