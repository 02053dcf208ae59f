"""Structure-of-arrays layout of the hourly-step state on the device.

Every per-cell quantity is stored as one or more *planes*: a plane is a
contiguous run of ``ld`` values (``ld`` >= number of cells, a multiple of 32 so
that each plane starts 128-byte aligned).  A field with a trailing dimension of
``k`` (soil layers, bands, plant-type slots ...) occupies ``k`` consecutive
planes, layer-major, so thread ``i`` of a warp reads element ``i`` of a plane
and every load is coalesced.

The planes are grouped into buffers by how the step uses them:

``PROG``   prognostic state: read at the start of a step, written at its end
``STAT``   per-cell static inputs (soil texture, vegetation structure): read only
``FORC``   hourly forcing (the ``atm`` leaves the step assumes are set)
``DIAG``   diagnostics the step writes but never reads (optional)
``ACC``    per-step accumulators of the day loop (optional; Kahan-compensated
           in the FP32 kernels, so each accumulator plane has a twin holding
           its running compensation)
``RUN``    per-run calibration vector of the ensemble kernels
``YEARLY`` accumulator totals an ensemble run reports at each year end
``DAILY``  daily weather the device forcing generator turns into hours
``DAYST``  state of the daily cadence (phenology, 10-day means, soil carbon)
``WET``    monthly wetland methane state

Each field names the leaf of the reference ``IBISState`` it mirrors
(``python-port/ibis/state/*.py``), so host code can move data between the
reference's pytree and these buffers without a lookup table of its own.  The
C header ``include/ibis_layout.h`` is generated from this table by
:func:`header_text` and checked against it by the test suite.
"""
from __future__ import annotations

from dataclasses import dataclass

NSOILAY = 6
NBEDROCK = 3
NSNOLAY = 3
NPFT = 12
NBAND = 2


@dataclass(frozen=True)
class Field:
    name: str          # C-side name (upper-cased in the header)
    leaf: str          # reference pytree leaf, e.g. "soil.tsoi"
    k: int = 1         # number of planes (trailing dimension)


PROG = (
    Field("tsoi", "soil.tsoi", NSOILAY),
    Field("wsoi", "soil.wsoi", NSOILAY),
    Field("wisoi", "soil.wisoi", NSOILAY),
    Field("tg", "soil.tg"),
    Field("wpud", "soil.wpud"),
    Field("wipud", "soil.wipud"),
    Field("tsoi_deep", "soil.tsoi_deep", NBEDROCK),
    Field("fi", "snow.fi"),
    Field("tsno", "snow.tsno", NSNOLAY),
    Field("hsno", "snow.hsno", NSNOLAY),
    Field("ti", "snow.ti"),
    Field("tlsub", "snow.tlsub"),
    Field("tu", "canopy.tu"),
    Field("ts", "canopy.ts"),
    Field("tl", "canopy.tl"),
    Field("t12", "canopy.t12"),
    Field("t34", "canopy.t34"),
    Field("q12", "canopy.q12"),
    Field("q34", "canopy.q34"),
    Field("wliqu", "canopy.wliqu"),
    Field("wliqs", "canopy.wliqs"),
    Field("wliql", "canopy.wliql"),
    Field("wsnou", "canopy.wsnou"),
    Field("wsnos", "canopy.wsnos"),
    Field("wsnol", "canopy.wsnol"),
    Field("ci_upper", "canopy.ci_upper", 2),
    Field("gs_upper", "canopy.gs_upper", 2),
    Field("cs_upper", "canopy.cs_upper", 2),
    Field("ci_lower", "canopy.ci_lower", 3),
    Field("gs_lower", "canopy.gs_lower", 3),
    Field("cs_lower", "canopy.cs_lower", 3),
    Field("a10scalparamu", "canopy.a10scalparamu"),
    Field("a10daylightu", "canopy.a10daylightu"),
    Field("a10scalparaml", "canopy.a10scalparaml"),
    Field("a10daylightl", "canopy.a10daylightl"),
    Field("firefac", "vegetation.firefac"),
    Field("nytimes", "vegetation.nytimes"),
    Field("nfirestep", "vegetation.nfirestep"),
    Field("sdry", "vegetation.sdry"),
    Field("nfirestep_vpd", "vegetation.nfirestep_vpd"),
    Field("sdry_vpd", "vegetation.sdry_vpd"),
)

STAT = (
    Field("poros", "soil.poros", NSOILAY),
    Field("hydraul", "soil.hydraul", NSOILAY),
    Field("suction", "soil.suction", NSOILAY),
    Field("bex", "soil.bex", NSOILAY),
    Field("sfield", "soil.sfield", NSOILAY),
    Field("swilt", "soil.swilt", NSOILAY),
    Field("sand", "soil.sand", NSOILAY),
    Field("clay", "soil.clay", NSOILAY),
    Field("csoi", "soil.csoi", NSOILAY),
    Field("rhosoi", "soil.rhosoi", NSOILAY),
    Field("albsav", "soil.albsav"),
    Field("albsan", "soil.albsan"),
    Field("z0soi", "soil.z0soi"),
    Field("lai", "vegetation.lai", 2),
    Field("sai", "vegetation.sai", 2),
    Field("ztop", "vegetation.ztop", 2),
    Field("zbot", "vegetation.zbot", 2),
    Field("fu", "vegetation.fu"),
    Field("fl", "vegetation.fl"),
    Field("frac", "vegetation.frac", NPFT),
    Field("exist", "vegetation.exist", NPFT),
    Field("cbiow", "vegetation.cbiow", NPFT),
    Field("cbior", "vegetation.cbior", NPFT),
    Field("sapfrac", "vegetation.sapfrac"),
    Field("tco2mic", "vegetation.tco2mic"),
    Field("f_inund", "methane.f_inund"),
    Field("zwt_obs", "methane.zwt_obs"),   # observed wetland water table, m (NaN: the model's); read under FLAG_ZWT_OBS
    # inputs of the IBIS 3.0 extensions, read only under their flags: the state of
    # temperature acclimation (FLAG_ACCLIM; the day loop refreshes it each day), the
    # day's mean air temperature of the state (FLAG_FROST), and the per-cell arrays
    # of SimParams ("sim." leaves): the cropland share (FLAG_CROP) and the organic
    # fraction of the soil solids per layer (FLAG_FORGANIC)
    Field("acclim_x", "seasonal.acclim_x"),
    Field("td", "atm.td"),
    Field("cropfrac", "sim.cropfrac"),
    Field("forganic", "sim.forganic", NSOILAY),
    # the cell's wetland band for per-band methane parameters (FLAG_CH4_BANDS): 0 tropical, 1 temperate,
    # 2 boreal -- the latitude rule or the Koeppen wetland type of biome_methane_params (methane.py:536-548)
    Field("ch4_band", "sim.ch4_band"),
)

#: Leaf prefixes of fields that are not leaves of the base reference state: the
#: wetland inputs, the optional seasonal module and per-cell SimParams arrays.
OPTIONAL_LEAF_PREFIXES = ("methane.", "seasonal.", "sim.")

FORC = (
    Field("ta", "atm.ta"),
    Field("qa", "atm.qa"),
    Field("ua", "atm.ua"),
    Field("psurf", "atm.psurf"),
    Field("coszen", "atm.coszen"),
    Field("solad", "atm.solad", NBAND),
    Field("solai", "atm.solai", NBAND),
    Field("fira", "atm.fira"),
    Field("raina", "atm.raina"),
    Field("snowa", "atm.snowa"),
)

DIAG = (
    Field("an_upper", "canopy.an_upper", 2),
    Field("ag_upper", "canopy.ag_upper", 2),
    Field("an_lower", "canopy.an_lower", 3),
    Field("ag_lower", "canopy.ag_lower", 3),
    Field("fwetu", "canopy.fwetu"),
    Field("fwets", "canopy.fwets"),
    Field("fwetl", "canopy.fwetl"),
    Field("rliqu", "canopy.rliqu"),
    Field("rliqs", "canopy.rliqs"),
    Field("rliql", "canopy.rliql"),
    Field("solu", "canopy.solu"),
    Field("sols", "canopy.sols"),
    Field("soll", "canopy.soll"),
    Field("solg", "canopy.solg"),
    Field("soli", "canopy.soli"),
    Field("firu", "canopy.firu"),
    Field("firs", "canopy.firs"),
    Field("firl", "canopy.firl"),
    Field("firg", "canopy.firg"),
    Field("firi", "canopy.firi"),
    Field("firb", "canopy.firb"),
    Field("asurd", "canopy.asurd", NBAND),
    Field("asuri", "canopy.asuri", NBAND),
    Field("topparu", "canopy.topparu"),
    Field("topparl", "canopy.topparl"),
    Field("scalcoefu", "canopy.scalcoefu", 4),
    Field("scalcoefl", "canopy.scalcoefl", 4),
    Field("fsenu", "canopy.fsenu"),
    Field("fsens", "canopy.fsens"),
    Field("fsenl", "canopy.fsenl"),
    Field("fseng", "canopy.fseng"),
    Field("fseni", "canopy.fseni"),
    Field("fvapg", "canopy.fvapg"),
    Field("fvapi", "canopy.fvapi"),
    Field("raing", "canopy.raing"),
    Field("snowg", "canopy.snowg"),
    Field("rhoa", "canopy.rhoa"),
    Field("consoi", "soil.consoi", NSOILAY),
    Field("hflo", "soil.hflo", NSOILAY + 1),
    Field("heatg", "soil.heatg"),
    Field("hvasug", "soil.hvasug"),
    Field("qglif", "soil.qglif", 4),
    Field("stresstu", "soil.stresstu"),
    Field("stresstl", "soil.stresstl"),
    Field("stressu", "soil.stressu", NSOILAY),
    Field("stressl", "soil.stressl", NSOILAY),
    Field("porosflo", "soil.porosflo", NSOILAY),
    Field("heati", "snow.heati"),
    Field("hvasui", "snow.hvasui"),
    Field("ginvap", "hydrology.ginvap"),
    Field("gsuvap", "hydrology.gsuvap"),
    Field("gtrans", "hydrology.gtrans"),
    Field("gtransu", "hydrology.gtransu"),
    Field("gtransl", "hydrology.gtransl"),
    Field("grunof", "hydrology.grunof"),
    Field("gdrain", "hydrology.gdrain"),
    Field("gadjust", "hydrology.gadjust"),
    Field("wtot", "hydrology.wtot"),
    Field("raing_avg", "hydrology.raing_avg"),
    Field("traing_avg", "hydrology.traing_avg"),
    Field("fhtop_soil", "hydrology.fhtop_soil"),
    Field("rainl", "hydrology.rainl"),
    Field("snowl", "hydrology.snowl"),
    Field("trainl", "hydrology.trainl"),
    Field("tsnowl", "hydrology.tsnowl"),
    Field("sflo_bot", "hydrology.sflo_bot"),
    Field("fhtop_snow", "hydrology.fhtop_snow"),
    Field("fsena", "canopy.fsena"),
)

ACC = (
    Field("adrain", "summary.adrain"),
    Field("adsnow", "summary.adsnow"),
    Field("adaet", "summary.adaet"),
    Field("a10ancub", "summary.a10ancub"),
    Field("a10ancls", "summary.a10ancls"),
    Field("a10ancl3", "summary.a10ancl3"),
    Field("a10ancl4", "summary.a10ancl4"),
    Field("aynpp", "summary.aynpp", NPFT),
    Field("aynpptot", "summary.aynpptot"),
    Field("aygpptot", "summary.aygpptot"),
    Field("aytrunof", "summary.aytrunof"),
    Field("aytdrain", "summary.aytdrain"),
    Field("ch4", "acc.ch4_day"),
    Field("tsoi_mean", "acc.tsoi_day", NSOILAY),
    Field("wsoi_mean", "acc.wsoi_day", NSOILAY),
    Field("wisoi_mean", "acc.wisoi_day", NSOILAY),
    Field("tg_mean", "acc.tg_day"),
    Field("afsena", "acc.fsena"),
    # last values, not sums: the soil-water stress of the day's last hour, which
    # the next day's phenology reads (loops_gswp3.py:441-442)
    Field("stresstu_last", "soil.stresstu"),
    Field("stresstl_last", "soil.stresstl"),
    # the optional ET and NEE components of the step's sums (state/et_parts.py,
    # state/nee_parts.py; loops_gswp3.py:263-281): under FLAG_ETPARTS / FLAG_NEEPARTS
    Field("et_trans", "etparts.trans"),
    Field("et_interc", "etparts.interc"),
    Field("et_soilev", "etparts.soilev"),
    Field("et_snowsub", "etparts.snowsub"),
    Field("nee_night", "neeparts.night"),
    Field("nee_day", "neeparts.day"),
)

# Per-run calibration vector of the ensemble kernels: the step-relevant
# parameters the reference's tower calibration varies
# (verify/calibration/fit_carbon.py:253-381, setters of SimParams leaves), 31
# values.  rwood/rroot/rgrowth are scalars there and apply to all 12 plant
# types; t_ref of the methane model stays at its SimParams value, as the tower
# fits hold it.
RUN = (
    Field("vmax", "stomata_params.vmax_pft", NPFT),
    Field("coefm", "stomata_params.coefm", 5),
    Field("stressfac", "stomata_params.stressfac"),
    Field("soil_beta_power", "canopy.soil_beta_power"),
    Field("wliqumax", "interception.wliqumax"),
    Field("wliqsmax", "interception.wliqsmax"),
    Field("wliqlmax", "interception.wliqlmax"),
    Field("fmax", "interception.fmax"),
    Field("r_ch4", "methane.r_ch4"),
    Field("q10p", "methane.q10p"),
    Field("z_tau", "methane.z_tau"),
    Field("tau_oxid", "methane.tau_oxid"),
    Field("z_wt_max", "methane.z_wt_max"),
    Field("rwood", "bgc_params.rwood"),
    Field("rroot", "bgc_params.rroot"),
    Field("rgrowth", "bgc_params.rgrowth"),
)

# Accumulators an ensemble run reports at the end of each year of its record
# (running totals; the host differences them into per-year sums).
YEARLY = (
    Field("aygpptot", "summary.aygpptot"),
    Field("aynpptot", "summary.aynpptot"),
    Field("adaet", "summary.adaet"),
    Field("afsena", "acc.fsena"),
    Field("aytrunof", "summary.aytrunof"),
    Field("aytdrain", "summary.aytdrain"),
    Field("ch4", "acc.ch4_day"),
)

# Daily weather the device forcing generator disaggregates to hours
# (DailyWeather, python-port/ibis/physics/weather.py:79-90; fira is the
# observed daily longwave the day loop may use instead of the generator's).
DAILY = (
    Field("td", "daily_weather.td"),
    Field("tmax", "daily_weather.tmax"),
    Field("tmin", "daily_weather.tmin"),
    Field("cloud", "daily_weather.cloud"),
    Field("precip", "daily_weather.precip"),
    Field("psurf", "daily_weather.psurf"),
    Field("qd", "daily_weather.qd"),
    Field("ud", "daily_weather.ud"),
    Field("fira", "gswp3.rlds"),
)

# State of the daily cadence (phenology, 10-day means, annual sums, soil
# carbon), advanced once a day around the day's hourly steps
# (loops_gswp3.py:382-608).  The 10-day means share their reference leaves
# with the daily sums of ACC: before and after a day the reference holds the
# means there, during the day the sums.
DAYST = (
    Field("plai", "vegetation.plai", NPFT),
    Field("tc", "vegetation.tc"),
    Field("tempu", "vegetation.tempu"),
    Field("templ", "vegetation.templ"),
    Field("agddu", "vegetation.agddu"),
    Field("agddl", "vegetation.agddl"),
    Field("dropu", "vegetation.dropu"),
    Field("dropls", "vegetation.dropls"),
    Field("dropl3", "vegetation.dropl3"),
    Field("dropl4", "vegetation.dropl4"),
    Field("tco2root", "vegetation.tco2root"),
    Field("tnmin", "vegetation.tnmin"),
    Field("a10td", "summary.a10td"),
    Field("a10ancub", "summary.a10ancub"),
    Field("a10ancls", "summary.a10ancls"),
    Field("a10ancl3", "summary.a10ancl3"),
    Field("a10ancl4", "summary.a10ancl4"),
    Field("ayprcp", "summary.ayprcp"),
    Field("ayaet", "summary.ayaet"),
    Field("ayco2mic", "summary.ayco2mic"),
    Field("ayco2root", "summary.ayco2root"),
    Field("storedn", "summary.storedn"),
    Field("yrleach", "summary.yrleach"),
    Field("ynleach", "summary.ynleach"),
    Field("clitlm", "carbon.clitlm"),
    Field("clitls", "carbon.clitls"),
    Field("clitll", "carbon.clitll"),
    Field("clitrm", "carbon.clitrm"),
    Field("clitrs", "carbon.clitrs"),
    Field("clitrl", "carbon.clitrl"),
    Field("clitwm", "carbon.clitwm"),
    Field("clitws", "carbon.clitws"),
    Field("clitwl", "carbon.clitwl"),
    Field("csoislop", "carbon.csoislop"),
    Field("csoislon", "carbon.csoislon"),
    Field("csoipas", "carbon.csoipas"),
    Field("totcmic", "carbon.totcmic"),
    Field("decompl", "carbon.decompl"),
    Field("decomps", "carbon.decomps"),
    Field("totlit", "carbon.totlit"),
    Field("totalit", "carbon.totalit"),
    Field("totrlit", "carbon.totrlit"),
    Field("totcsoi", "carbon.totcsoi"),
    Field("totfall", "carbon.totfall"),
    Field("falll", "carbon.falll"),
    Field("fallr", "carbon.fallr"),
    Field("fallw", "carbon.fallw"),
    # the optional modules of the daily cadence (loops_gswp3.py:418-437,
    # 585-596): the seasonal states (temperature acclimation, Delpierre
    # senescence) and the growing-season soil-water stress sums, advanced only
    # when the day parameters switch them on; the latitude (radians) gives the
    # day length the senescence states read
    Field("acclim_x", "seasonal.acclim_x"),
    Field("ssen_u", "seasonal.ssen_u"),
    Field("ssen_l", "seasonal.ssen_l"),
    Field("aystressu", "stress.aystressu"),
    Field("aystressl", "stress.aystressl"),
    Field("stress_nday", "stress.nday"),
    Field("latitude", "params.latitude"),
)

# Monthly wetland methane (MethaneState, python-port/ibis/bgc/methane.py:404-423)
# and what the month's end needs from its start: the heterotrophic respiration
# total then (for the carbon partition) and the year's CH4 carbon taken out of
# Rh so far (scripts/run_global.py:786-839).
WET = (
    Field("flux", "wetland.flux"),
    Field("annual", "wetland.annual"),
    Field("zwt", "wetland.zwt"),
    Field("rh0", "summary.ayco2mic"),      # ayco2mic at the month's start
    Field("ch4c", "summary.ayrh_ch4c"),    # the year's CH4 carbon taken out of Rh
)

GROUPS = {"PROG": PROG, "STAT": STAT, "FORC": FORC, "DIAG": DIAG, "ACC": ACC, "RUN": RUN, "YEARLY": YEARLY,
          "DAILY": DAILY, "DAYST": DAYST, "WET": WET}


def offsets(group):
    """name -> (first plane, number of planes) for one buffer group."""
    out, p = {}, 0
    for f in group:
        out[f.name] = (p, f.k)
        p += f.k
    return out


def nplanes(group):
    return sum(f.k for f in group)


N_PROG = nplanes(PROG)
N_STAT = nplanes(STAT)
N_FORC = nplanes(FORC)
N_DIAG = nplanes(DIAG)
N_ACC = nplanes(ACC)
N_RUN = nplanes(RUN)
N_YEARLY = nplanes(YEARLY)
N_DAILY = nplanes(DAILY)
N_DAYST = nplanes(DAYST)
N_WET = nplanes(WET)

OFF = {g: offsets(v) for g, v in GROUPS.items()}


def leading_dim(ncell: int) -> int:
    """Plane stride for ``ncell`` cells: rounded up to 32 values (128 bytes in FP32)."""
    return max(32, (ncell + 31) // 32 * 32)


def header_text() -> str:
    lines = [
        "/* Generated from ibis_b200/layout.py by header_text(); do not edit by hand.",
        " *",
        " * Plane indices of the structure-of-arrays buffers of the hourly step.",
        " * Element (plane p, cell i) of a buffer with leading dimension ld lives at",
        " * buf[p * ld + i].  Forcing for a run of nstep hours is nstep consecutive",
        " * FORC blocks: step s, plane p, cell i at forc[(s * IBIS_FORC_COUNT + p) * ld + i].",
        " * The ACC buffer holds IBIS_ACC_COUNT value planes followed by the same",
        " * number of Kahan compensation planes.",
        " */",
        "#ifndef IBIS_LAYOUT_H",
        "#define IBIS_LAYOUT_H",
        "",
    ]
    for g, fields in GROUPS.items():
        lines.append(f"/* {g} */")
        lines.append("enum {")
        for f in fields:
            off = OFF[g][f.name][0]
            suffix = f"  /* {f.leaf}, {f.k} planes */" if f.k > 1 else f"  /* {f.leaf} */"
            lines.append(f"    IBIS_{g}_{f.name.upper()} = {off},{suffix}")
        lines.append(f"    IBIS_{g}_COUNT = {nplanes(fields)}")
        lines.append("};")
        lines.append("")
    lines.append("#endif /* IBIS_LAYOUT_H */")
    return "\n".join(lines) + "\n"


if __name__ == "__main__":
    print(header_text(), end="")
