"""Float64 restatement of the reference's monthly wetland methane (test infrastructure).

The checker of the device month kernels (ibis_b200/csrc/ibis_month.cuh).
The functions of python-port/ibis/bgc/methane.py:431-496 and the way the
GSWP3 month driver calls them (python-port/ibis/timestepping/loops_gswp3.py:740-760):

* :func:`methane_step` -- the month's flux from the end-of-month state
  (``methane_flux`` with Rh = tco2mic x 12e-3 x 86400), water table, annual sum;
* :func:`methane_step_from_mean` -- the month's flux as the mean of the hourly
  fluxes (the day-mean accumulator of the step), water table, annual sum;
* :func:`scale_month` -- the month scaled to an inundated fraction;
* :func:`ch4_carbon_from_rh` -- the month's CH4 carbon to take out of Rh;
* :func:`reset_annual` -- year-end reset.

The wetland state is a dict with ``flux``, ``annual``, ``zwt`` (MethaneState,
methane.py:404-423).  Values the reference forms in float32 (the scale
factor, the Rh conversion) are rounded to float32 here as well.
"""
from __future__ import annotations

import numpy as np

from .column import methane as methane_flux
from .column import methane_params, wetland_water_table

RH_CONV = np.float64(np.float32(12.0e-3 * 86400.0))


def methane_step(wet: dict, f_inund, rh, tsoi, wsoi, wisoi, hsoi, ndays, P, zwt_obs=None) -> dict:
    """methane.py:431-456."""
    flux = methane_flux(f_inund, rh, tsoi, wsoi, wisoi, hsoi, P, zwt_obs)
    zwt = wetland_water_table(wsoi, wisoi, hsoi, P, zwt_obs)
    return dict(flux=flux, annual=wet["annual"] + flux * ndays, zwt=zwt)


def methane_step_from_mean(wet: dict, flux_month, wsoi, wisoi, hsoi, ndays, P, zwt_obs=None) -> dict:
    """methane.py:459-474."""
    zwt = wetland_water_table(wsoi, wisoi, hsoi, P, zwt_obs)
    return dict(flux=np.asarray(flux_month, np.float64), annual=wet["annual"] + flux_month * ndays, zwt=zwt)


def reset_annual(wet: dict) -> dict:
    """methane.py:477-480."""
    return dict(wet, annual=np.zeros_like(wet["annual"]))


def scale_month(wet: dict, annual_before, f) -> dict:
    """methane.py:483-489: flux and the month's share of the annual total, linear in ``f``."""
    a0 = np.zeros_like(wet["annual"]) if annual_before is None else annual_before
    f = np.asarray(f, np.float32).astype(np.float64)
    return dict(wet, flux=wet["flux"] * f, annual=a0 + (wet["annual"] - a0) * f)


def ch4_carbon_from_rh(annual, annual_before, rh, rh_before):
    """methane.py:492-496."""
    w0 = np.zeros_like(annual) if annual_before is None else annual_before
    return np.minimum(np.maximum(annual - w0, 0.0), np.maximum(rh - rh_before, 0.0))


def month_end(wet: dict, prog: dict, stat: dict, ch4_sum, ayco2mic, rh0, ndays, hsoi, P, from_mean=True, scale=None,
              partition=False, zwt_obs=None):
    """The month's end as the GSWP3 driver and the global driver compose it
    (loops_gswp3.py:740-760; scripts/run_global.py:824-839): the monthly
    methane step (from the mean of the hourly fluxes when ``from_mean``;
    ``ch4_sum`` is the month's sum of the day means), optionally scaled to the
    inundated fraction ``scale``, optionally with the CH4 carbon taken out of
    Rh.  Returns (wet, ayco2mic, take)."""
    a0 = wet["annual"]
    P = methane_params(P, stat)
    if from_mean:
        new = methane_step_from_mean(wet, ch4_sum / ndays, prog["wsoi"], prog["wisoi"], hsoi, ndays, P, zwt_obs)
    else:
        rh = stat["tco2mic"] * RH_CONV
        new = methane_step(wet, stat["f_inund"], rh, prog["tsoi"], prog["wsoi"], prog["wisoi"], hsoi, ndays, P,
                           zwt_obs)
    if scale is not None:
        new = scale_month(new, a0, scale)
    take = np.zeros_like(a0)
    if partition:
        take = ch4_carbon_from_rh(new["annual"], a0, ayco2mic, rh0)
        ayco2mic = ayco2mic - take
    return new, ayco2mic, take
