"""Float64 restatement of the reference's daily-to-hourly weather disaggregation.

Test infrastructure: the checker of the device forcing generator
(ibis_b200/csrc/ibis_diurnal.cuh), never a product path.

* :func:`precip_timing` -- ``compute_precip_timing``
  (python-port/ibis/physics/weather.py:395-443): length and start of the day's
  precipitation event from two uniform variates;
* :func:`diurnal` -- ``diurnal`` (weather.py:483-601): solar geometry and the
  direct/diffuse split, the Fourier temperature cycle, humidity capped at 99 %
  saturation, EPIC wind, Idso longwave, and the rain/snow split of the event;
* :func:`uniform24` -- the counter-based variates the device generator draws
  (the SplitMix64 finalizer of Steele, Lea and Flood 2014, applied twice to
  (seed, day, slot) and the cell), as 24-bit fractions k / 2**24.

The reference draws its variates from ``jax.random`` (Threefry); this
restatement takes them as inputs, so fixtures made with any variates pin it.
"""
from __future__ import annotations

import numpy as np

from .physics import esat, qsat

PI = np.float64(np.pi)
STEF = 5.67e-8
BANDS = np.array([0.46, 0.54])


def _mix(z):
    """SplitMix64 finalizer on uint64 arrays (wrapping arithmetic)."""
    z = np.asarray(z, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = z + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def uniform24(seed: int, cell, day: int, slot: int):
    """k / 2**24, k the top 24 bits of mix(mix((seed << 32) | (day << 8) | slot) ^ cell),
    vectorised over cells (slot < 256, day < 2**24)."""
    c = (np.uint64(seed & 0xFFFFFFFF) << np.uint64(32)) | np.uint64(((day & 0xFFFFFF) << 8) | (slot & 0xFF))
    z = _mix(_mix(c) ^ np.asarray(cell, dtype=np.uint64))
    return (z >> np.uint64(40)).astype(np.float64) / float(1 << 24)


def effective_solar_constant(jday):
    orbit = 2.0 * PI * jday / 365.2425
    return 1370.0 * (1.000110 + 0.034221 * np.cos(orbit) + 0.001280 * np.sin(orbit)
                     + 0.000719 * np.cos(2.0 * orbit) + 0.000077 * np.sin(2.0 * orbit))


def precip_timing(u_plen, u_start, precip, dtime):
    """(plens, startp, endp) in seconds (weather.py:395-443)."""
    niter = int(86400.0 / dtime)
    plenmin = 1 + int((4.0 * 3600.0 - 1.0) / dtime)
    plenmax = max(int(24.0 * 3600.0 / dtime), plenmin)
    plen_random = plenmin + np.floor(np.asarray(u_plen) * (plenmax - plenmin + 1)).astype(np.int64)
    plen_random = np.clip(plen_random, plenmin, plenmax)
    plen_needed = np.ceil(np.asarray(precip) / 15.0).astype(np.int64)
    plen = np.clip(np.maximum(plen_random, plen_needed), plenmin, plenmax)
    plens = dtime * plen.astype(np.float64)
    max_start = np.maximum(0, niter - plen)
    start_idx = np.minimum(np.floor(np.asarray(u_start) * (max_start + 1)).astype(np.int64), max_start)
    startp = dtime * start_idx.astype(np.float64)
    return plens, startp, startp + plens


def diurnal(time, jday, daily, lat_deg, plens, startp, endp, u_wind, dtime, fira_obs=None):
    """Hourly forcing dict (atm leaf names) at ``time`` seconds after midnight
    (weather.py:483-601).  ``daily`` maps tmax, tmin, cloud, precip, psurf, qd,
    ud to per-cell arrays.  With ``fira_obs`` the longwave is the observed daily
    value, as the day loop overrides it (loops_gswp3.py:131)."""
    rtime = time / 3600.0
    orbit = 2.0 * PI * jday / 365.2425
    xdecl = (0.006918 - 0.399912 * np.cos(orbit) + 0.070257 * np.sin(orbit) - 0.006758 * np.cos(2.0 * orbit)
             + 0.000907 * np.sin(2.0 * orbit) - 0.002697 * np.cos(3.0 * orbit) + 0.001480 * np.sin(3.0 * orbit))
    angle = 2.0 * PI * (rtime - 12.0) / 24.0
    sw = effective_solar_constant(jday)
    xlat = np.asarray(lat_deg) * PI / 180.0
    coszen = np.maximum(0.0, np.sin(xlat) * np.sin(xdecl) + np.cos(xlat) * np.cos(xdecl) * np.cos(angle))
    cloud = daily["cloud"]
    trans = 0.251 + 0.509 * (1.0 - cloud)
    fdiffuse = np.where(trans > 0.75, 0.166, 1.0045 + 0.0435 * trans - 3.5227 * trans ** 2 + 2.6313 * trans ** 3)
    solad = sw * coszen[:, None] * BANDS[None, :] * trans[:, None] * (1.0 - fdiffuse[:, None])
    solai = sw * coszen[:, None] * BANDS[None, :] * trans[:, None] * fdiffuse[:, None]
    gamma = 0.44 - 0.46 * np.sin(PI / 12.0 * rtime + 0.9) + 0.11 * np.sin(2.0 * PI / 12.0 * rtime + 0.9)
    ta = daily["tmax"] * gamma + daily["tmin"] * (1.0 - gamma)
    psurf = daily["psurf"]
    qmin = np.minimum(daily["qd"], 0.99 * qsat(esat(daily["tmin"]), psurf))
    qmax = (daily["qd"] - 0.56 * qmin) / 0.44
    esat_ta = esat(ta)
    qsa = 0.99 * qsat(esat_ta, psurf)
    qa = np.minimum(qsa, qmax * gamma + qmin * (1.0 - gamma))
    ua = np.clip(1.13989 * daily["ud"] * (-np.log(np.maximum(u_wind, 1e-10))) ** 0.30, 2.5, 10.0)
    if fira_obs is None:
        emb = 0.01 * (psurf * qa / (0.622 + qa))
        ea = 0.70 + 5.95e-5 * emb * np.exp(1500.0 / ta)
        fira = (1.0 - cloud) * ea * STEF * ta ** 4 + cloud * 0.950 * STEF * ta ** 4
    else:
        fira = np.asarray(fira_obs, dtype=np.float64)
    in_event = (time >= startp) & (time < endp)
    warm = (ta - 273.15) > 2.5
    rate = daily["precip"] / np.maximum(plens, dtime)
    return dict(coszen=coszen, ta=ta, qa=qa, ua=ua, psurf=np.asarray(psurf, dtype=np.float64), fira=fira,
                raina=np.where(in_event & warm, rate, 0.0), snowa=np.where(in_event & ~warm, rate, 0.0),
                solad=solad, solai=solai)


def observed_shortwave(sw_obs, use, coszen, jday, solad_gen, solai_gen):
    """observed_shortwave (weather.py:458-481): where ``use`` is set, the observed
    hourly total split into direct and diffuse by the hourly clearness-index
    relation of Spitters et al. (1986), then into the two bands; elsewhere the
    generator's values unchanged."""
    coszen = np.asarray(coszen, dtype=np.float64)
    kt = np.clip(sw_obs / np.maximum(effective_solar_constant(jday) * coszen, 1.0), 0.0, 1.0)
    r = 0.847 - 1.61 * coszen + 1.04 * coszen ** 2
    kk = (1.47 - r) / 1.66
    fd = np.where(kt <= 0.22, 1.0, np.where(kt <= 0.35, 1.0 - 6.4 * (kt - 0.22) ** 2,
                                            np.where(kt <= kk, 1.47 - 1.66 * kt, r)))
    fd = np.where(coszen <= 0.0, 1.0, np.clip(fd, 0.0, 1.0))
    sw = np.maximum(sw_obs, 0.0)
    solad = sw[:, None] * BANDS[None, :] * (1.0 - fd)[:, None]
    solai = sw[:, None] * BANDS[None, :] * fd[:, None]
    use = np.asarray(use, dtype=bool)[:, None]
    return np.where(use, solad, solad_gen), np.where(use, solai, solai_gen)
