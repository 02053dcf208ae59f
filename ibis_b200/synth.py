"""Seeded synthetic columns and hourly forcing for the hourly step.

No tower, GSWP3 or HWSD data exist in this environment, so every workload is
synthetic, drawn from ``numpy.random.Generator(PCG64(seed))`` with the shapes
and distributions the reference's benchmark configurations describe:

* soil texture: sand and clay fractions U(0.05, 0.6) per cell, the same on all
  six layers, mapped to hydraulic and thermal properties by the USDA texture
  triangle and the Rawls et al. (1992) class table that the reference's
  ``python-port/ibis/io/soil_init.py:17-261`` uses;
* vegetation: per-slot weights ~ Dirichlet(alpha) over the 12 plant-type slots,
  normalised separately within the upper (0-7) and lower (8-11) stories as
  ``python-port/ibis/physics/phenology.py:229-262`` does; a slot exists where
  its weight exceeds 1e-3; leaf/stem area, cover and heights follow the weights;
* forcing: shortwave = max(0, 1000 cos(zenith)) x a daily cloud factor
  U(0.3, 1), split direct/diffuse by Friend's transmissivity relation and into
  VIS/NIR as 0.46/0.54 (``python-port/ibis/physics/weather.py:544-555``); air
  temperature 10 C + 12 C seasonal sine + 5 C diurnal sine + N(0, 2);
  relative humidity U(0.4, 0.95); precipitation zero with p = 0.9, else
  Gamma(k=0.8, theta=2 mm/h), rain above 2.5 C else snow
  (``weather.py:592-596``); wind lognormal with median 3 m/s and sigma 0.5;
  pressure 101.3 kPa; CO2 390 ppm; downward longwave from Brutsaert's
  clear-sky emissivity on temperature and vapour pressure;
* wetland fraction ~ Beta(0.5, 8); heterotrophic respiration a fixed daily
  rate per cell.

Everything here is host-side set-up; none of it is timed.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import layout as L
from .params import StepParams, FLAG_BEDROCK

# --- USDA texture classes and Rawls et al. (1992) properties (reference io/soil_init.py:17-55) ---
_CLASS_TABLE = {  # poros, sfield, swilt, bex, suction (m), hydraul (m/s)
    "sand":            (0.437, 0.091, 0.033, 1.7, 0.07, 5.833e-5),
    "loamy_sand":      (0.437, 0.125, 0.055, 2.1, 0.09, 1.6972e-5),
    "sandy_loam":      (0.453, 0.207, 0.095, 3.1, 0.15, 7.1944e-6),
    "loam":            (0.463, 0.270, 0.117, 4.5, 0.11, 3.6667e-6),
    "silt_loam":       (0.501, 0.330, 0.133, 4.7, 0.21, 1.8889e-6),
    "sandy_clay_loam": (0.398, 0.255, 0.148, 4.0, 0.28, 1.1944e-6),
    "clay_loam":       (0.464, 0.318, 0.197, 5.2, 0.26, 6.3889e-7),
    "silty_clay_loam": (0.471, 0.366, 0.208, 6.6, 0.33, 4.1667e-7),
    "sandy_clay":      (0.430, 0.339, 0.239, 6.0, 0.29, 3.3333e-7),
    "silty_clay":      (0.479, 0.387, 0.250, 7.9, 0.34, 2.5e-7),
    "clay":            (0.475, 0.396, 0.272, 7.6, 0.37, 1.6667e-7),
}
_CLASS_ORDER = list(_CLASS_TABLE)
# polygons in (sand %, clay %) of the USDA triangle, tested in this order
_POLYGONS = [
    [(85, 0), (90, 10), (100, 0)],
    [(70, 0), (85, 15), (90, 10), (85, 0)],
    [(50, 0), (43, 7), (52, 7), (52, 20), (80, 20), (85, 15), (70, 0)],
    [(43, 7), (23, 27), (45, 27), (52, 20), (52, 7)],
    [(0, 0), (0, 27), (23, 27), (50, 0)],
    [(52, 20), (45, 27), (45, 35), (65, 35), (80, 20)],
    [(20, 27), (20, 40), (45, 40), (45, 27)],
    [(0, 27), (0, 40), (20, 40), (20, 27)],
    [(45, 35), (45, 55), (65, 35)],
    [(0, 40), (0, 60), (20, 40)],
    [(20, 40), (0, 60), (0, 100), (45, 55), (45, 40)],
]
FORGANIC = 0.010
RHOSOI_VAL = 2650.0 * (1.0 - FORGANIC) + 1300.0 * FORGANIC
CSOI_VAL = 870.0 * (1.0 - FORGANIC) + 1920.0 * FORGANIC


def _inside(poly, x, y):
    """Even-odd ray test of the point (x, y) against a closed polygon."""
    hit = False
    j = len(poly) - 1
    for i in range(len(poly)):
        xi, yi = poly[i]
        xj, yj = poly[j]
        if (yi > y) != (yj > y) and x < (xj - xi) * (y - yi) / (yj - yi) + xi:
            hit = not hit
        j = i
    return hit


def _texture_table():
    lut = np.full((101, 101), 4, dtype=np.int8)  # silt loam where no polygon claims the point
    for s in range(101):
        for c in range(101 - s):
            if s == 0 and c == 0:
                continue
            for idx, poly in enumerate(_POLYGONS):
                if _inside(poly, float(s), float(c)):
                    lut[s, c] = idx
                    break
    return lut


_LUT = None


def soil_properties(sand_pct, clay_pct):
    """Per-cell hydraulic/thermal properties from sand and clay percent (1-D arrays)."""
    global _LUT
    if _LUT is None:
        _LUT = _texture_table()
    ms = np.clip(np.round(sand_pct).astype(np.int32), 0, 100)
    mc = np.clip(np.round(clay_pct).astype(np.int32), 0, 100)
    cls = _LUT[ms, mc]
    tab = np.array([_CLASS_TABLE[k] for k in _CLASS_ORDER])
    poros, sfield, swilt, bex, suction, hydraul = (tab[cls, i] for i in range(6))
    fs = 0.01 * np.round(sand_pct).astype(int)
    fc = 0.01 * np.round(clay_pct).astype(int)
    albsav = fs * 0.120 + (1.0 - fs - fc) * 0.085 + fc * 0.050
    return dict(poros=poros, sfield=sfield / poros, swilt=swilt / poros, bex=bex, suction=suction,
                hydraul=hydraul, albsav=albsav, albsan=2.0 * albsav)


def _tetens(tk):
    """Saturation vapour pressure (Pa), Tetens, for building synthetic humidity only."""
    tc = tk - 273.15
    return np.where(tc >= 0.0, 610.78 * np.exp(17.27 * tc / (tc + 237.3)),
                    610.78 * np.exp(21.875 * tc / (tc + 265.5)))


@dataclass
class Workload:
    """Host copy (float64) of one synthetic workload in the plane schema of ``layout``."""
    ncell: int
    nhour: int
    prog: dict
    stat: dict
    forc: dict                     # name -> (nhour, ncell[, k])
    params: StepParams
    latitude: np.ndarray
    start_doy: int = 172
    meta: dict = field(default_factory=dict)

    def forcing_at(self, h):
        return {k: v[h] for k, v in self.forc.items()}


def solar_cosz(lat_deg, doy, hour):
    """Cosine of the solar zenith angle (Spencer's declination; local solar time)."""
    g = 2.0 * np.pi * (doy - 1) / 365.0
    dec = (0.006918 - 0.399912 * np.cos(g) + 0.070257 * np.sin(g) - 0.006758 * np.cos(2 * g)
           + 0.000907 * np.sin(2 * g) - 0.002697 * np.cos(3 * g) + 0.00148 * np.sin(3 * g))
    ha = 2.0 * np.pi * (hour + 0.5 - 12.0) / 24.0
    la = np.deg2rad(lat_deg)
    return np.sin(la) * np.sin(dec) + np.cos(la) * np.cos(dec) * np.cos(ha)


def make_forcing(rng, lat, nhour, start_doy=172, start_hour=0):
    """Hourly forcing (nhour, ncell) arrays for cells at latitudes ``lat`` (degrees)."""
    n = lat.size
    hours = start_hour + np.arange(nhour)
    doy = (start_doy - 1 + hours // 24) % 365 + 1
    hod = hours % 24
    ndays = int(hours[-1] // 24 - hours[0] // 24 + 1)
    day_idx = hours // 24 - hours[0] // 24
    cloud = rng.uniform(0.3, 1.0, size=(ndays, n))[day_idx]          # clear-sky fraction of the day
    cosz = solar_cosz(lat[None, :], doy[:, None], hod[:, None])
    sw = np.maximum(0.0, 1000.0 * cosz) * cloud
    trans = 0.251 + 0.509 * cloud
    fdiff = np.where(trans > 0.75, 0.166, 1.0045 + 0.0435 * trans - 3.5227 * trans ** 2 + 2.6313 * trans ** 3)
    fdiff = np.clip(fdiff, 0.0, 1.0)
    bands = np.array([0.46, 0.54])
    solad = sw[..., None] * bands * (1.0 - fdiff[..., None])
    solai = sw[..., None] * bands * fdiff[..., None]
    hemi = np.where(lat >= 0.0, 1.0, -1.0)
    season = np.sin(2.0 * np.pi * (doy[:, None] - 105.0) / 365.0) * hemi[None, :]
    diur = np.sin(2.0 * np.pi * (hod[:, None] - 9.0) / 24.0)
    ta = 283.15 + 12.0 * season + 5.0 * diur + rng.normal(0.0, 2.0, size=(nhour, n))
    rh = rng.uniform(0.4, 0.95, size=(nhour, n))
    psurf = np.full((nhour, n), 101300.0)
    e = rh * _tetens(ta)
    qa = 0.622 * e / (psurf - 0.378 * e)
    wet = rng.uniform(size=(nhour, n)) >= 0.9
    amount = rng.gamma(0.8, 2.0, size=(nhour, n)) / 3600.0           # mm/h -> kg m-2 s-1
    prec = np.where(wet, amount, 0.0)
    warm = (ta - 273.15) > 2.5
    ua = np.exp(np.log(3.0) + 0.5 * rng.normal(size=(nhour, n)))
    ea_hpa = e / 100.0
    emis = np.clip(1.24 * (ea_hpa / ta) ** (1.0 / 7.0), 0.5, 1.0)
    fira = emis * 5.67e-8 * ta ** 4
    return dict(ta=ta, qa=qa, ua=ua, psurf=psurf, coszen=cosz, solad=solad, solai=solai,
                fira=fira, raina=np.where(warm, prec, 0.0), snowa=np.where(warm, 0.0, prec))


def make_columns(rng, n, alpha=0.5):
    """Static inputs (stat) for n cells."""
    sand = rng.uniform(0.05, 0.6, size=n) * 100.0
    clay = rng.uniform(0.05, 0.6, size=n) * 100.0
    over = sand + clay > 95.0                                         # keep inside the texture triangle
    clay = np.where(over, 95.0 - sand, clay)
    sp = soil_properties(sand, clay)
    S = {}
    for k in ("poros", "sfield", "swilt", "bex", "suction", "hydraul"):
        S[k] = np.repeat(sp[k][:, None], L.NSOILAY, axis=1)
    S["sand"] = np.repeat(sand[:, None], L.NSOILAY, axis=1)
    S["clay"] = np.repeat(clay[:, None], L.NSOILAY, axis=1)
    S["csoi"] = np.full((n, L.NSOILAY), CSOI_VAL)
    S["rhosoi"] = np.full((n, L.NSOILAY), RHOSOI_VAL)
    S["albsav"], S["albsan"] = sp["albsav"], sp["albsan"]
    S["z0soi"] = np.full(n, 0.005)
    w = rng.dirichlet(np.full(L.NPFT, alpha), size=n)
    up, lo = w[:, :8].sum(1), w[:, 8:].sum(1)
    frac = np.empty_like(w)
    frac[:, :8] = w[:, :8] / np.maximum(up, 1e-12)[:, None]
    frac[:, 8:] = w[:, 8:] / np.maximum(lo, 1e-12)[:, None]
    S["frac"] = frac
    S["exist"] = (w > 1e-3).astype(np.float64)
    S["lai"] = np.stack([0.3 + 2.5 * lo, 0.5 + 5.0 * up], 1)
    S["sai"] = np.stack([0.1 + 0.4 * lo, 0.2 + 1.0 * up], 1)
    S["fu"] = np.clip(0.25 + 0.7 * up, 0.25, 0.975)
    S["fl"] = np.clip(0.25 + 0.7 * lo, 0.25, 0.975)
    S["ztop"] = np.stack([np.full(n, 1.0), 10.0 + 15.0 * up], 1)
    S["zbot"] = np.stack([np.full(n, 0.05), 2.0 + 3.0 * up], 1)
    S["cbiow"] = np.concatenate([12.0 * w[:, :8], 1.5 * w[:, 8:10], np.zeros((n, 2))], 1)
    S["cbior"] = 0.6 * w
    S["sapfrac"] = np.full(n, 0.1)
    S["tco2mic"] = rng.uniform(0.5, 3.0, size=n) * 1e-3 / 12.0 / 86400.0   # 0.5-3 gC m-2 d-1 in mol CO2 m-2 s-1
    S["f_inund"] = rng.beta(0.5, 8.0, size=n)
    return S


def make_initial(rng, S, F0):
    """Prognostic state at the start of a run, consistent with the first hour's forcing."""
    n = S["poros"].shape[0]
    ta, qa = F0["ta"], F0["qa"]
    P = {}
    tmean = np.full(n, 283.15)
    P["tsoi"] = np.repeat(tmean[:, None], L.NSOILAY, 1) + 0.5 * (ta - tmean)[:, None] * np.exp(-np.arange(L.NSOILAY))[None, :]
    w0 = rng.uniform(0.3, 0.9, size=n)
    P["wsoi"] = np.minimum(w0[:, None] + 0.03 * np.arange(L.NSOILAY)[None, :], 0.98)
    P["wisoi"] = np.zeros((n, L.NSOILAY))
    P["tg"] = ta.copy()
    P["wpud"] = np.zeros(n)
    P["wipud"] = np.zeros(n)
    P["tsoi_deep"] = np.repeat(P["tsoi"][:, -1:], L.NBEDROCK, 1)
    P["fi"] = np.zeros(n)
    P["tsno"] = np.full((n, L.NSNOLAY), 273.16)
    P["hsno"] = np.zeros((n, L.NSNOLAY))
    P["ti"] = np.full(n, 273.16)
    P["tlsub"] = np.full(n, 273.16)
    for k in ("tu", "ts", "tl", "t12", "t34"):
        P[k] = ta.copy()
    P["q12"], P["q34"] = qa.copy(), qa.copy()
    for k in ("wliqu", "wliqs", "wliql", "wsnou", "wsnos", "wsnol"):
        P[k] = np.zeros(n)
    P["ci_upper"] = np.full((n, 2), 350.0e-6)
    P["gs_upper"] = np.full((n, 2), 0.01)
    P["cs_upper"] = np.full((n, 2), 350.0e-6)
    P["ci_lower"] = np.full((n, 3), 350.0e-6)
    P["gs_lower"] = np.full((n, 3), 0.01)
    P["cs_lower"] = np.full((n, 3), 350.0e-6)
    P["a10scalparamu"] = np.full(n, 0.5)
    P["a10daylightu"] = np.full(n, 100.0)
    P["a10scalparaml"] = np.full(n, 0.5)
    P["a10daylightl"] = np.full(n, 100.0)
    for k in ("firefac", "nytimes", "nfirestep", "sdry", "nfirestep_vpd", "sdry_vpd"):
        P[k] = np.zeros(n)
    return P


def apply_edge_cases(prog, stat, forc):
    """Overwrite leading cells with the regimes the reference's tests single out:
    bare ground, a deep cold snowpack, frozen saturated soil, a flooded puddle,
    polar night and a hot dry desert (python-port/tests/test_regression.py:40-114,
    docs/technote/17_numerics_verification.md:678-686)."""
    n = prog["tg"].shape[0]
    cases = []
    if n > 0:   # bare cell: no canopy at all (turvap bare-cell rows, noveg reset)
        stat["lai"][0] = 0.0
        stat["sai"][0] = 0.0
        stat["fu"][0] = 0.0
        stat["fl"][0] = 0.0
        cases.append("bare")
    if n > 1:   # deep, cold snowpack with buried lower canopy
        prog["fi"][1] = 0.9
        prog["hsno"][1] = [0.05, 0.3, 0.3]
        prog["tsno"][1] = [262.0, 265.0, 268.0]
        prog["ti"][1] = 262.0
        prog["tlsub"][1] = 268.0
        forc["ta"][:, 1] = np.minimum(forc["ta"][:, 1], 263.0)
        cases.append("snowpack")
    if n > 2:   # frozen, nearly saturated soil (permafrost-like)
        prog["tsoi"][2] = [265.0, 266.0, 268.0, 270.0, 271.0, 272.0]
        prog["wsoi"][2] = 0.3
        prog["wisoi"][2] = 0.65
        prog["tsoi_deep"][2] = 272.5
        cases.append("frozen")
    if n > 3:   # flooded: saturated column with a puddle, heavy rain
        prog["wsoi"][3] = 0.999
        prog["wpud"][3] = 6.0
        prog["wipud"][3] = 1.0
        forc["raina"][:, 3] = 5.0 / 3600.0
        forc["snowa"][:, 3] = 0.0
        cases.append("flooded")
    if n > 4:   # polar night
        forc["coszen"][:, 4] = -0.3
        forc["solad"][:, 4] = 0.0
        forc["solai"][:, 4] = 0.0
        cases.append("polar_night")
    if n > 5:   # hot dry desert, sparse canopy
        forc["ta"][:, 5] = 318.0
        forc["qa"][:, 5] = 0.002
        prog["wsoi"][5] = 0.05
        stat["lai"][5] = [0.05, 0.01]
        stat["fu"][5] = 0.01
        cases.append("desert")
    return cases


def make_workload(ncell, nhour, seed=0, lat_range=(-60.0, 80.0), lat=None, alpha=0.5,
                  start_doy=172, edge_cases=False, bedrock=True):
    """Build a seeded synthetic workload (host float64 arrays)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    if lat is None:
        lat = rng.uniform(lat_range[0], lat_range[1], size=ncell)
    else:
        lat = np.broadcast_to(np.asarray(lat, dtype=np.float64), (ncell,)).copy()
    stat = make_columns(rng, ncell, alpha)
    forc = make_forcing(rng, lat, nhour, start_doy)
    prog = make_initial(rng, stat, {k: v[0] for k, v in forc.items()})
    cases = apply_edge_cases(prog, stat, forc) if edge_cases else []
    P = StepParams(co2conc=390.0e-6)
    if not bedrock:
        P.flags = P.flags & ~FLAG_BEDROCK
    return Workload(ncell=ncell, nhour=nhour, prog=prog, stat=stat, forc=forc, params=P,
                    latitude=lat, start_doy=start_doy, meta=dict(seed=seed, edge_cases=cases, alpha=alpha))


def make_dayst(rng, stat, lat):
    """Seeded daily-cadence state (``layout.DAYST``) in the ranges of a spun-up
    run: potential LAI from the columns' existence flags, 10-day means near the
    climate of the latitude, annual sums part-way through a year, litter and
    soil carbon pools of a few kgC m-2."""
    n = lat.shape[0]
    u = lambda lo, hi, shape=(n,): rng.uniform(lo, hi, shape)
    tclim = 300.0 - 0.35 * np.abs(lat)
    plai = stat["exist"] * u(0.5, 6.0, (n, L.NPFT))
    d = dict(plai=plai, tc=tclim - 273.16 - u(5.0, 15.0), tempu=u(0.0, 1.0), templ=u(0.5, 1.0),
             agddu=u(0.0, 3e6), agddl=u(0.0, 3e6), dropu=u(0.5, 1.0), dropls=u(0.5, 1.0), dropl3=u(0.5, 1.0),
             dropl4=u(0.5, 1.0), tco2root=np.zeros(n), tnmin=u(0.0, 4e-8), a10td=tclim + u(-3.0, 3.0),
             a10ancub=u(1e-7, 9e-7), a10ancls=u(1e-8, 5e-7), a10ancl3=u(1e-8, 5e-7), a10ancl4=u(1e-7, 9e-7),
             ayprcp=u(100.0, 1800.0), ayaet=u(100.0, 1200.0), ayco2mic=u(0.05, 1.2), ayco2root=np.zeros(n),
             storedn=u(0.01, 0.1), yrleach=u(2.0, 36.0), ynleach=u(0.2, 3.0))
    pools = dict(clitlm=(2e-5, 2e-3), clitls=(4e-3, 0.1), clitll=(1.6e-3, 0.04), clitrm=(3e-5, 7e-4),
                 clitrs=(8e-3, 0.15), clitrl=(5e-3, 0.08), clitwm=(0.0, 0.0), clitws=(4e-3, 1.0),
                 clitwl=(3e-3, 0.8), csoislop=(1.0, 22.0), csoislon=(0.09, 2.3), csoipas=(1.3, 16.0),
                 totcmic=(0.04, 0.55), falll=(0.03, 0.35), fallr=(0.04, 0.24), fallw=(0.005, 0.5))
    for k, (lo, hi) in pools.items():
        d[k] = u(lo, hi)
    d["decompl"], d["decomps"] = u(0.1, 2.5), u(0.2, 2.3)
    d["totfall"] = d["falll"] + d["fallr"] + d["fallw"]
    return d


def make_daily_weather(rng, lat, nday):
    """Seeded daily weather (``layout.DAILY``, (nday, ncell) arrays) for the
    device forcing generator: temperatures about the latitude's climate, cloud,
    gamma-distributed precipitation on 40 % of days, humidity, wind and the
    daily longwave."""
    n = lat.shape[0]
    tclim = 300.0 - 0.35 * np.abs(lat)
    tmin = tclim[None, :] - rng.uniform(2.0, 10.0, (nday, n))
    tmax = tmin + rng.uniform(3.0, 14.0, (nday, n))
    wet = rng.uniform(size=(nday, n)) < 0.4
    return dict(td=0.5 * (tmin + tmax), tmax=tmax, tmin=tmin, cloud=rng.uniform(0.0, 1.0, (nday, n)),
                precip=np.where(wet, rng.gamma(0.8, 6.0, (nday, n)), 0.0), psurf=np.full((nday, n), 101300.0),
                qd=rng.uniform(0.002, 0.015, (nday, n)), ud=rng.uniform(1.0, 6.0, (nday, n)),
                fira=rng.uniform(250.0, 400.0, (nday, n)))


# ----------------------------------------------------------------------------
# plane packing
# ----------------------------------------------------------------------------

def to_planes(group_name, values, ld, dtype=np.float32, out=None):
    """Pack a dict of (n,) / (n, k) arrays into a (nplanes, ld) array."""
    group = L.GROUPS[group_name]
    npl = L.nplanes(group)
    if out is None:
        out = np.zeros((npl, ld), dtype=dtype)
    off = L.OFF[group_name]
    for f in group:
        if f.name not in values:
            continue
        p0, k = off[f.name]
        v = np.asarray(values[f.name])
        n = v.shape[0]
        if k == 1:
            out[p0, :n] = v
        else:
            out[p0:p0 + k, :n] = v.T
    return out


def from_planes(group_name, planes, n):
    """Unpack a (nplanes, ld) array into a dict of float64 (n,) / (n, k) arrays."""
    group = L.GROUPS[group_name]
    off = L.OFF[group_name]
    out = {}
    for f in group:
        p0, k = off[f.name]
        if k == 1:
            out[f.name] = np.asarray(planes[p0, :n], dtype=np.float64).copy()
        else:
            out[f.name] = np.asarray(planes[p0:p0 + k, :n], dtype=np.float64).T.copy()
    return out


def forcing_planes(forc, ld, h0=0, h1=None, dtype=np.float32):
    """(nhour, FORC planes, ld) array for hours [h0, h1)."""
    nh = next(iter(forc.values())).shape[0]
    h1 = nh if h1 is None else h1
    out = np.zeros((h1 - h0, L.N_FORC, ld), dtype=dtype)
    for h in range(h0, h1):
        to_planes("FORC", {k: v[h] for k, v in forc.items()}, ld, dtype, out=out[h - h0])
    return out
