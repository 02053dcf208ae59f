"""Scalar and small-table parameters of the hourly step.

One flat, all-``double`` record mirrors every parameter the reference's
``timestep_body`` (``python-port/ibis/timestepping/loops.py:234``) and the
per-step accumulators of ``_run_day_inner._step_body``
(``python-port/ibis/timestepping/loops_gswp3.py:115-320``) read from
``PhysicalConstants``, ``SimParams`` and its sub-modules, plus the static
fields of ``SnowState``.  Defaults are the reference's defaults (the F77
branches of ``configs/params/default.yaml``; ``rhosoi_val``/``csoi_mineral_val``
from ``io/soil_init.py``).

The record is passed by value to the kernels (it lands in the constant bank);
the C declaration ``IbisParams`` in ``include/ibis_layout.h`` is generated from
:data:`PARAM_FIELDS` so host and device agree on the layout.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field, fields
from typing import Sequence

import numpy as np

from . import layout as L

# (name, count, default) -- count > 1 is a fixed-size table
PARAM_FIELDS: list[tuple[str, int, object]] = [
    # --- PhysicalConstants (constants.py:16-80)
    ("stef", 1, 5.67e-8), ("vonk", 1, 0.4), ("grav", 1, 9.80616), ("tmelt", 1, 273.16),
    ("hvap", 1, 2.5104e6), ("hfus", 1, 0.3336e6), ("hsub", 1, 2.5104e6 + 0.3336e6),
    ("ch2o", 1, 4.218e3), ("cice", 1, 2.106e3), ("cair", 1, 1.00464e3), ("cvap", 1, 1.81e3),
    ("rair", 1, 287.04), ("rvap", 1, 461.0), ("cappa", 1, 287.04 / 1.00464e3),
    ("rhow", 1, 1.0e3), ("epsilon", 1, 1.0e-7),
    # --- time step (s) and atmospheric CO2 (mol/mol)
    ("dtime", 1, 3600.0), ("co2conc", 1, 350.0e-6),
    # --- SnowState static fields (state/snow.py:33-39)
    ("z0sno", 1, 0.0005), ("rhos", 1, 250.0), ("consno", 1, 0.20), ("hsnotop", 1, 0.05),
    ("hsnomin", 1, 0.15), ("fimin", 1, 0.00004), ("fimax", 1, 1.00),
    # --- VegRadParams (radiation.py:32-56), [band][story] with story 0 = lower
    ("rhoveg", 4, (0.10, 0.10, 0.60, 0.40)), ("tauveg", 4, (0.07, 0.05, 0.25, 0.20)),
    ("oriev", 2, (0.5, 0.0)), ("orieh", 2, (0.0, 0.0)),
    ("omegasno", 2, (0.9, 0.7)),
    # --- CanopyParams (canopy_exchange.py:68-84)
    ("cleaf", 1, 0.01), ("cstem", 1, 0.01), ("cgrass", 1, 0.01),
    ("dleaf", 2, (0.10, 0.10)), ("dstem", 2, (0.10, 0.10)),
    ("alaiml", 1, 8.0), ("alaimu", 1, 8.0), ("chu", 1, 8436.0), ("chs", 1, 2.109e5),
    ("chl", 1, 8436.0), ("soil_beta_power", 1, 1.0),
    # --- InterceptionParams (interception.py:31-45)
    ("wliqumax", 1, 0.20), ("wliqsmax", 1, 0.40), ("wliqlmax", 1, 0.20),
    ("wsnoumax", 1, 2.00), ("wsnosmax", 1, 4.00), ("wsnolmax", 1, 2.00),
    ("tdripu", 1, 7200.0), ("tdrips", 1, 7200.0), ("tdripl", 1, 7200.0),
    ("tblowu", 1, 43200.0), ("tblows", 1, 43200.0), ("tblowl", 1, 43200.0),
    ("fmax", 1, 0.25),
    # --- StomataParams (stomata.py:33-161); Ball-Berry groups [broadleaf, conifer, shrub, C4, C3]
    ("tau15", 1, 4500.0), ("kc15", 1, 1.5e-4), ("ko15", 1, 0.25), ("cimax", 1, 2000.0e-6),
    ("o2conc", 1, 0.209), ("alpha3", 1, 0.080), ("theta3", 1, 0.950), ("beta3", 1, 0.990),
    ("alpha4", 1, 0.050), ("theta4", 1, 0.970), ("beta4", 1, 0.800),
    ("gamma", 5, (0.015, 0.015, 0.015, 0.030, 0.015)),
    ("coefm", 5, (10.0, 6.0, 9.0, 4.0, 9.0)),
    ("coefb", 5, (0.010, 0.010, 0.010, 0.040, 0.010)),
    ("gsmin", 5, (1e-5, 1e-5, 1e-5, 1e-5, 1e-5)),
    ("vmax_pft", 12, (65e-6, 65e-6, 40e-6, 30e-6, 30e-6, 25e-6,
                      30e-6, 30e-6, 27.5e-6, 27.5e-6, 15e-6, 25e-6)),
    ("stressfac", 1, -5.0), ("cap_kn", 1, 0.15),
    # IBIS 3.0 stomata extensions (stomata.py:98-159; all act only under their IBIS_FLAG_* switches):
    # the per-PFT Ball-Berry slopes of coefm_mix; the acclimated PFTs (acclim_pfts as a 0/1 mask) and the
    # per-PFT acclimation constants (the scalars acclim_s0/acclim_smax repeated when acclim_per_pft is off);
    # the frost ramp on the day's mean air temperature, C
    ("coefm_pft", 12, (10.0, 10.0, 10.0, 6.0, 10.0, 6.0, 10.0, 6.0, 9.0, 9.0, 4.0, 9.0)),
    ("acclim_mask", 12, (0.0, 0.0, 0.0, 1.0, 0.0, 1.0, 0.0, 0.0, 1.0, 0.0, 0.0, 0.0)),
    ("acclim_s0_pft", 12, (-3.063,) * 12), ("acclim_smax_pft", 12, (17.72,) * 12),
    ("frost_t0", 1, -5.0), ("frost_t1", 1, 5.0),
    # --- CropParams of the cropland share's grass capacity (io/parameters.py:262-278; loops.py:218-231)
    ("crop_vmax_scale_c3", 1, 1.0), ("crop_vmax_scale_c4", 1, 1.0), ("crop_c4_share", 1, -1.0),
    # --- soil constants of SimParams (loops.py:92-111)
    ("wpudmax", 1, 10.0), ("zwpmax", 1, 0.5), ("bperm", 1, 0.04),
    ("rhosoi_val", 1, 2650.0 * 0.99 + 1300.0 * 0.01), ("csoi_mineral_val", 1, 870.0 * 0.99 + 1920.0 * 0.01),
    # --- column geometry: soil layer thicknesses (io/soil_init.py:17), root fractions [layer][lower, upper]
    ("hsoi", 6, (0.10, 0.15, 0.25, 0.50, 1.00, 2.00)),
    ("froot", 12, (0.0,) * 12),
    # --- BedrockParams (bedrock.py:35-66)
    ("hsoi_bed", 3, (2.0, 2.0, 4.0)), ("consoi_bed", 1, 3.0), ("rhosoi_bed", 1, 2700.0),
    ("csoi_bed", 1, 740.74074074074076),
    # --- FireParams used per step (fire.py:205-360)
    ("d_crit", 1, 0.5), ("vpd_ref", 1, 3.0), ("d_crit_vpd", 1, 0.33),
    # --- physical clamps read from the environment at trace time (loops.py:665, 1143)
    ("flux_max", 1, 2000.0), ("t_max_dev", 1, 40.0),
    # --- MethaneParams (bgc/methane.py:19-91)
    ("sat_crit", 1, 0.95), ("z_max", 1, 4.0), ("r_ch4", 1, 0.23), ("q10p", 1, 1.60),
    ("t_ref", 1, 295.15), ("z_wt_max", 1, 0.30), ("z_wt_ref", 1, 0.50), ("z_tau", 1, 0.50),
    ("tau_oxid", 1, 0.10),
    # per-band MethaneParams [tropical, temperate, boreal] selected per cell by the STAT ch4_band plane under
    # FLAG_CH4_BANDS: biome_methane_params (methane.py:521-563) with or without a parameter file's methane_bands
    ("ch4b_sat_crit", 3, (0.95,) * 3), ("ch4b_z_max", 3, (4.0,) * 3), ("ch4b_r_ch4", 3, (0.23,) * 3),
    ("ch4b_q10p", 3, (1.60,) * 3), ("ch4b_t_ref", 3, (295.15,) * 3), ("ch4b_z_wt_max", 3, (0.30,) * 3),
    ("ch4b_z_wt_ref", 3, (0.50,) * 3), ("ch4b_z_tau", 3, (0.50,) * 3), ("ch4b_tau_oxid", 3, (0.10,) * 3),
    # --- BGCParams respiration used by the NPP accumulator (io/parameters.py:248-259)
    ("rwood", 12, (0.0125,) * 12), ("rroot", 12, (1.25,) * 12), ("rgrowth", 12, (0.30,) * 12),
    ("ndaypy", 1, 365.0),
]

#: Compile-time switches carried in ``IbisParams.flags``.
FLAG_BEDROCK = 1 << 0          # soil.tsoi_deep present: 9-layer heat solve (bedrock.py:88)
FLAG_H2O_CONSISTENT = 1 << 1   # SimParams.h2o_consistent_weights (soil_physics.py:263)
FLAG_SUNSHADE_U = 1 << 2       # StomataParams.sunshade_u (stomata.py:140)
FLAG_SUNSHADE_L = 1 << 3       # StomataParams.sunshade_l
FLAG_ACC = 1 << 4              # advance the day-loop accumulators (loops_gswp3.py:161-302)
FLAG_CH4 = 1 << 5              # per-step wetland CH4 into the day accumulator (loops_gswp3.py:307-314)
FLAG_SOIL_MEANS = 1 << 6       # per-step day means of tsoi/wsoi/wisoi/tg (loops_gswp3.py:316-318)
FLAG_DIAG = 1 << 7             # write the DIAG buffer
FLAG_KAHAN = 1 << 8            # compensated accumulation (FP32 kernels)
FLAG_ZWT_OBS = 1 << 9          # observed wetland water table (STAT zwt_obs, NaN = the model's; methane.py:366-367)
FLAG_ETPARTS = 1 << 10         # ET components accumulated apart, with FLAG_ACC (loops_gswp3.py:263-272)
FLAG_NEEPARTS = 1 << 11        # day- and night-time NEE accumulated apart, with FLAG_ACC (loops_gswp3.py:274-281)
# IBIS 3.0 extensions of the step (off: the F77 step).  Any of them selects the
# extended kernel instantiations; the F77 kernels never carry their code.
FLAG_VMAX_MIX = 1 << 12        # StomataParams.vmax_mix: big-leaf vmax = displayed-LAI-weighted mean (stomata.py:598-631)
FLAG_COEFM_MIX = 1 << 13       # StomataParams.coefm_mix: big-leaf slope from coefm_pft (stomata.py:646-657)
FLAG_GPP_CAPACITY = 1 << 14    # StomataParams.gpp_split_by_capacity: NPP shares by leaf area x vmax (loops_gswp3.py:197-205)
FLAG_ACCLIM = 1 << 15          # StomataParams.acclim_on with a seasonal state: vmax x f_S(acclim_x) (loops.py:291-303)
FLAG_ACCLIM_LIGHT = 1 << 16    # StomataParams.acclim_light: the big leaf's capacity factor also on the light limit
FLAG_FROST = 1 << 17           # StomataParams.frost_on: frost ramp on atm.td, with FLAG_ACCLIM (loops.py:305-309)
FLAG_CAP_SCALE_U = 1 << 18     # StomataParams.cap_scale_u: canopy-level co-limitation (stomata.py:889-896)
FLAG_CAP_SCALE_L = 1 << 19     # StomataParams.cap_scale_l
FLAG_LEAF_ONLY = 1 << 20       # StomataParams.scale_leaf_only: light scaling over leaves and stems (stomata.py:442-512)
FLAG_CROP = 1 << 21            # SimParams.cropfrac present: grass capacity on the cropland share (loops.py:218-231)
FLAG_FORGANIC = 1 << 22        # SimParams.forganic present: organic dry conductivity (soil_physics.py:74-77)
# per-cell methane parameters by wetland band (biome_methane_params, methane.py:521-563): the ch4b_* tables
# indexed by the STAT ch4_band plane (0 tropical, 1 temperate, 2 boreal) in every CH4 of the step and the month
FLAG_CH4_BANDS = 1 << 23
X3_FLAGS = (FLAG_VMAX_MIX | FLAG_COEFM_MIX | FLAG_GPP_CAPACITY | FLAG_ACCLIM | FLAG_ACCLIM_LIGHT | FLAG_FROST
            | FLAG_CAP_SCALE_U | FLAG_CAP_SCALE_L | FLAG_LEAF_ONLY | FLAG_CROP | FLAG_FORGANIC)

KNOWN_FLAGS = (FLAG_BEDROCK | FLAG_H2O_CONSISTENT | FLAG_SUNSHADE_U | FLAG_SUNSHADE_L | FLAG_ACC
               | FLAG_CH4 | FLAG_SOIL_MEANS | FLAG_DIAG | FLAG_KAHAN | FLAG_ZWT_OBS | FLAG_ETPARTS | FLAG_NEEPARTS
               | X3_FLAGS | FLAG_CH4_BANDS)

# Default root profile (lower, upper) used by the synthetic columns; the reference keeps froot as a
# state leaf vegetation.froot of shape (nsoilay, 2) shared by every cell.
DEFAULT_FROOT = np.array([[0.25, 0.15], [0.25, 0.15], [0.20, 0.20],
                          [0.15, 0.20], [0.10, 0.15], [0.05, 0.15]])


def _ctypes_struct():
    flds = []
    for name, n, _ in PARAM_FIELDS:
        flds.append((name, ctypes.c_double * n if n > 1 else ctypes.c_double))
    flds.append(("flags", ctypes.c_uint32))
    flds.append(("_pad", ctypes.c_uint32))
    return type("IbisParams", (ctypes.Structure,), {"_fields_": flds})


IbisParamsC = _ctypes_struct()


class StepParams:
    """Mutable parameter record with the reference defaults.

    Attribute names follow the reference (``params.stomata_params.coefm`` is
    ``coefm`` here, ``consts.tmelt`` is ``tmelt``).  ``flags`` holds the
    compile-time switches (``FLAG_*``).
    """

    def __init__(self, **overrides):
        for name, n, default in PARAM_FIELDS:
            val = np.array(default, dtype=np.float64) if n > 1 else float(default)
            object.__setattr__(self, name, val)
        self.froot = DEFAULT_FROOT.reshape(-1).copy()
        self.flags = FLAG_BEDROCK | FLAG_ACC | FLAG_CH4 | FLAG_KAHAN
        for k, v in overrides.items():
            setattr(self, k, v)

    def __setattr__(self, key, value):
        spec = {n: c for n, c, _ in PARAM_FIELDS}
        if key == "flags":
            value = int(value)
            if value & ~KNOWN_FLAGS:
                raise ValueError(f"unknown flag bits 0x{value & ~KNOWN_FLAGS:x}")
        elif key in spec:
            if spec[key] > 1:
                arr = np.array(value, dtype=np.float64).reshape(-1)
                if arr.size != spec[key]:
                    raise ValueError(f"{key} needs {spec[key]} values, got {arr.size}")
                value = arr
            else:
                value = float(value)
        else:
            raise AttributeError(f"no parameter named {key!r}")
        object.__setattr__(self, key, value)

    # convenience views
    @property
    def froot2(self) -> np.ndarray:
        """Root fractions as (nsoilay, 2) [lower, upper], like ``vegetation.froot``."""
        return np.asarray(self.froot).reshape(L.NSOILAY, 2)

    def has(self, flag: int) -> bool:
        return bool(self.flags & flag)

    def copy(self) -> "StepParams":
        out = StepParams()
        for name, n, _ in PARAM_FIELDS:
            v = getattr(self, name)
            object.__setattr__(out, name, v.copy() if n > 1 else v)
        out.flags = self.flags
        return out

    def to_c(self):
        s = IbisParamsC()
        for name, n, _ in PARAM_FIELDS:
            v = getattr(self, name)
            if n > 1:
                getattr(s, name)[:] = [float(x) for x in v]
            else:
                setattr(s, name, float(v))
        s.flags = self.flags
        return s


# Parameters of the daily cadence (phenology and soil biogeochemistry), all
# double: PhenoParams (python-port/ibis/physics/phenology.py:30-86, read by
# pheno, phenology.py:89-287) and BGCParams (io/parameters.py, read by soilbgc,
# physics/biogeochem.py:23-243, and the decomposition factors of the day loop,
# timestepping/loops_gswp3.py:494-555), and the acclimation time constant of
# StomataParams (physics/stomata.py:116) the seasonal module advances with.
# The photoperiod switches are 0 or 1.  Defaults are the reference's.
DAY_PARAM_FIELDS: list[tuple[str, int, object]] = [
    ("ddays", 1, 15.0), ("tthresh_u_offset", 1, 5.0), ("tthresh_u_abs", 1, -100.0), ("gthresh_u_c", 1, 0.0),
    ("gdd_thresh_u", 1, 100.0), ("gdd_ramp_u", 1, 50.0), ("tthresh_l_c", 1, 0.0), ("gthresh_l_c", 1, -5.0),
    ("gdd_thresh_l", 1, 150.0), ("gdd_ramp_l", 1, 50.0), ("drop_thresh", 1, 0.0), ("drop_stress_thresh", 1, -1.0),
    ("drop_floor", 1, 0.1), ("stress_accum_tmin", 1, -100.0),
    ("sen_photoperiod_u", 1, 0.0), ("sen_pstart_u", 1, 14.0), ("sen_tb_u", 1, 20.0), ("sen_ycrit_u", 1, 300.0),
    ("sen_photoperiod_l", 1, 0.0), ("sen_pstart_l", 1, 14.0), ("sen_tb_l", 1, 20.0), ("sen_ycrit_l", 1, 300.0),
    ("lig_frac", 1, 0.5), ("fbsom", 1, 0.017), ("effac", 1, 0.4), ("bgc_fmax", 1, 0.45), ("rconst", 1, 1200.0),
    ("cnleaf", 1, 40.0), ("cnroot", 1, 60.0), ("cnwood", 1, 200.0),
    ("cnr", 8, (8.0, 15.0, 10.0, 15.0, 100.0, 150.0, 6.0, 250.0)),
    ("klm", 1, 0.15), ("kls", 1, 0.01), ("kll", 1, 0.01), ("krm", 1, 0.1), ("krs", 1, 0.005), ("krl", 1, 0.005),
    ("kwm", 1, 0.001), ("kws", 1, 0.001), ("kwl", 1, 0.001), ("kbn", 1, 0.045), ("kbp", 1, 0.005),
    ("knb", 1, 0.001), ("kns", 1, 1e-06), ("kpb", 1, 0.0001), ("kps", 1, 1e-06), ("ksb", 1, 8e-07),
    ("ylm", 1, 0.4), ("yls", 1, 0.3), ("yll", 1, 1.0), ("yrm", 1, 0.4), ("yrs", 1, 0.3), ("yrl", 1, 1.0),
    ("ywm", 1, 0.4), ("yws", 1, 0.3), ("ywl", 1, 1.0), ("ybn", 1, 1.0), ("ybp", 1, 1.0), ("yps", 1, 1.0),
    ("yns", 1, 1.0), ("ysb", 1, 0.2), ("ypb", 1, 0.2), ("ynb", 1, 0.25),
    ("lt_e0", 1, 344.0), ("wfps_opt", 1, 60.0), ("k_scale", 1, 1.0),
    ("acclim_tau", 1, 10.93),
    # set by the day loop, not parameters of the reference: the day of year of
    # the day, and whether the state carries the seasonal / stress modules (0 or 1)
    ("jday", 1, 1.0), ("seasonal_on", 1, 0.0), ("stress_on", 1, 0.0),
]
# the day parameters the day loop sets itself
DAY_LOOP_FIELDS = ("jday", "seasonal_on", "stress_on")


class DayParams:
    """Mutable record of :data:`DAY_PARAM_FIELDS` (reference defaults)."""

    def __init__(self, **overrides):
        for name, n, default in DAY_PARAM_FIELDS:
            object.__setattr__(self, name, np.array(default, dtype=np.float64) if n > 1 else float(default))
        for k, v in overrides.items():
            setattr(self, k, v)

    def __setattr__(self, key, value):
        spec = {n: c for n, c, _ in DAY_PARAM_FIELDS}
        if key not in spec:
            raise AttributeError(f"no daily parameter named {key!r}")
        if spec[key] > 1:
            value = np.array(value, dtype=np.float64).reshape(-1)
            if value.size != spec[key]:
                raise ValueError(f"{key} needs {spec[key]} values")
        else:
            value = float(value)
        object.__setattr__(self, key, value)

    def to_c(self):
        s = IbisDayParamsC()
        for name, n, _ in DAY_PARAM_FIELDS:
            v = getattr(self, name)
            if n > 1:
                getattr(s, name)[:] = [float(x) for x in v]
            else:
                setattr(s, name, float(v))
        return s


IbisDayParamsC = type("IbisDayParams", (ctypes.Structure,),
                      {"_fields_": [(n, ctypes.c_double * c if c > 1 else ctypes.c_double)
                                    for n, c, _ in DAY_PARAM_FIELDS]})


#: biome_methane_params' per-biome constants [tropical, temperate, boreal] (methane.py:504, 519)
R_CH4_BIOME = (0.15, 0.32, 0.18)
T_REF_BIOME = (299.6, 283.0, 277.9)
CH4_BAND_FIELDS = ("sat_crit", "z_max", "r_ch4", "q10p", "t_ref", "z_wt_max", "z_wt_ref", "z_tau", "tau_oxid")
CH4_BANDS = ("tropical", "temperate", "boreal")


def methane_band_index(lat_deg, band_index=None) -> np.ndarray:
    """The STAT ch4_band plane (0 tropical, 1 temperate, 2 boreal) the way
    biome_methane_params assigns biomes (methane.py:536-548): tropical for
    -30 < lat < 30, boreal for lat >= 60, temperate otherwise; a Koeppen
    wetland type ``band_index`` >= 0 (0, 1, 2) replaces the latitude rule."""
    lat = np.asarray(lat_deg, np.float64)
    trop = (lat > -30.0) & (lat < 30.0)
    boreal = lat >= 60.0
    if band_index is not None:
        bi = np.asarray(band_index)
        trop = np.where(bi >= 0, bi == 0, trop)
        boreal = np.where(bi >= 0, bi == 2, boreal)
    return np.where(trop, 0.0, np.where(boreal, 2.0, 1.0))


def with_methane_bands(P: "StepParams", bands: dict | None = None) -> "StepParams":
    """A copy of ``P`` with per-band methane parameters (FLAG_CH4_BANDS) as
    biome_methane_params forms them (methane.py:521-563): without ``bands`` the
    per-biome r_ch4 and t_ref constants and ``P``'s other values; with a
    parameter file's ``methane_bands`` section ({tropical|temperate|boreal:
    {field: value}}) each band's given fields, ``P``'s value elsewhere."""
    out = P.copy()
    tables = {f: [float(getattr(P, f))] * 3 for f in CH4_BAND_FIELDS}
    if bands is None:
        tables["r_ch4"] = list(R_CH4_BIOME)
        tables["t_ref"] = list(T_REF_BIOME)
    else:
        given = sorted({k for v in bands.values() for k in v})
        bad = [k for k in given if k not in CH4_BAND_FIELDS]
        if bad:
            raise KeyError(f"unknown methane fields in methane_bands: {bad}")
        if "z_wt_ref" in given:
            # the reference's water table takes one z_wt_ref (its layer weights do not broadcast per cell)
            raise ValueError("methane_bands cannot vary z_wt_ref")
        for f in given:
            tables[f] = [float(bands.get(b, {}).get(f, getattr(P, f))) for b in CH4_BANDS]
    for f, t in tables.items():
        setattr(out, "ch4b_" + f, np.asarray(t, np.float64))
    out.flags |= FLAG_CH4_BANDS
    return out


def header_struct_text() -> str:
    lines = ["/* Parameter record of the hourly step (all double; passed by value). */",
             "typedef struct IbisParams {"]
    for name, n, _ in PARAM_FIELDS:
        lines.append(f"    double {name}[{n}];" if n > 1 else f"    double {name};")
    lines.append("    unsigned int flags;   /* IBIS_FLAG_* */")
    lines.append("    unsigned int _pad;")
    lines.append("} IbisParams;")
    lines.append("")
    lines.append("/* X-macro over the record: S(name) for scalars, A(name, count) for tables. */")
    lines.append("#define IBIS_PARAM_LIST(S, A) \\")
    for name, n, _ in PARAM_FIELDS:
        lines.append(f"    A({name}, {n}) \\" if n > 1 else f"    S({name}) \\")
    lines.append("")
    lines.append("")
    for nm, val in [("BEDROCK", FLAG_BEDROCK), ("H2O_CONSISTENT", FLAG_H2O_CONSISTENT),
                    ("SUNSHADE_U", FLAG_SUNSHADE_U), ("SUNSHADE_L", FLAG_SUNSHADE_L),
                    ("ACC", FLAG_ACC), ("CH4", FLAG_CH4), ("SOIL_MEANS", FLAG_SOIL_MEANS),
                    ("DIAG", FLAG_DIAG), ("KAHAN", FLAG_KAHAN), ("ZWT_OBS", FLAG_ZWT_OBS),
                    ("ETPARTS", FLAG_ETPARTS), ("NEEPARTS", FLAG_NEEPARTS),
                    ("VMAX_MIX", FLAG_VMAX_MIX), ("COEFM_MIX", FLAG_COEFM_MIX), ("GPP_CAPACITY", FLAG_GPP_CAPACITY),
                    ("ACCLIM", FLAG_ACCLIM), ("ACCLIM_LIGHT", FLAG_ACCLIM_LIGHT), ("FROST", FLAG_FROST),
                    ("CAP_SCALE_U", FLAG_CAP_SCALE_U), ("CAP_SCALE_L", FLAG_CAP_SCALE_L),
                    ("LEAF_ONLY", FLAG_LEAF_ONLY), ("CROP", FLAG_CROP), ("FORGANIC", FLAG_FORGANIC),
                    ("CH4_BANDS", FLAG_CH4_BANDS)]:
        lines.append(f"#define IBIS_FLAG_{nm} {val}u")
    lines.append(f"#define IBIS_FLAGS_X3 {X3_FLAGS}u   /* any of these selects the IBIS 3.0 kernels */")
    lines.append("")
    lines.append("/* Parameters of the daily cadence (phenology, soil biogeochemistry), all double. */")
    lines.append("typedef struct IbisDayParams {")
    for name, n, _ in DAY_PARAM_FIELDS:
        lines.append(f"    double {name}[{n}];" if n > 1 else f"    double {name};")
    lines.append("} IbisDayParams;")
    return "\n".join(lines) + "\n"
