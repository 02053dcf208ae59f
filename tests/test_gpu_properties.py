"""Size-independent properties of the FP32 step at the full 95,333-cell size.

Column water balance of one hour (the reference's own closure test,
python-port/tests/test_water_balance.py:34-49): the change of soil water plus
puddle equals (rain reaching the soil - soil evaporation - transpiration -
runoff - drainage) x dt within 2 % of the fluxes + 0.05 kg m-2, for a moist, a
near-saturated and a saturated column under rain.  And a day of the workload
stays finite and inside physical bounds, as does a year of the day loop (daily
cadence and monthly methane) on 4,096 cells.
"""
import numpy as np
import pytest
import torch

from ibis_b200 import layout as L
from ibis_b200 import synth
from ibis_b200.columns import Columns

pytestmark = pytest.mark.gpu
N = 95333


@pytest.fixture(scope="module")
def workload():
    return synth.make_workload(N, 24, seed=0)


def _column_water(prog, stat, hsoi):
    w = 1000.0 * stat["poros"] * hsoi[None, :6] * ((1.0 - prog["wisoi"]) * prog["wsoi"] + prog["wisoi"])
    return w.sum(axis=1) + prog["wpud"] + prog["wipud"]


@pytest.mark.parametrize("wsoi,rain", [(0.6, 0.0), (0.98, 2.0e-3), (1.0, 5.0e-3)])
def test_column_water_balance_full_size(cuda_lib, workload, wsoi, rain):
    wl = workload
    prog = {k: v.copy() for k, v in wl.prog.items()}
    prog["wsoi"] = np.full_like(prog["wsoi"], wsoi)
    prog["wisoi"] = np.zeros_like(prog["wisoi"])
    forc = {k: v[:1].copy() for k, v in wl.forc.items()}
    forc["raina"] = np.full_like(forc["raina"], rain)
    forc["snowa"] = np.zeros_like(forc["snowa"])
    forc["ta"] = np.maximum(forc["ta"], 280.0)
    cols = Columns.from_host(prog, wl.stat, dtype=torch.float32, diag=True, acc=False)
    p0 = cols.prog_host()
    cols.run(cols.forcing(forc), wl.params)
    torch.cuda.synchronize()
    p1, D = cols.prog_host(), cols.diag_host()
    hs = np.asarray(wl.params.hsoi)
    w0, w1 = _column_water(p0, wl.stat, hs), _column_water(p1, wl.stat, hs)
    dt = wl.params.dtime
    into = D["raing_avg"]
    out = D["gsuvap"] + D["gtrans"] + D["grunof"] + D["gdrain"]
    resid = (w1 - w0) - (into - out) * dt
    scale = np.maximum(np.abs(into) + np.abs(out), 1e-6) * dt
    bad = np.abs(resid) > 0.02 * scale + 0.05
    assert not bad.any(), (int(bad.sum()), float(np.abs(resid).max()))
    if wsoi == 1.0:
        assert float(D["gdrain"].max()) > 0.0


def test_day_stays_finite_and_physical(cuda_lib, workload):
    wl = workload
    cols = Columns.from_host(wl.prog, wl.stat, dtype=torch.float32, acc=True)
    cols.run(cols.forcing(wl.forc), wl.params)
    torch.cuda.synchronize()
    assert not cols.nonfinite()[0]
    p = cols.prog_host()
    for k in ("tsoi", "tg", "tu", "ts", "tl", "t12", "t34"):
        assert np.all((p[k] > 180.0) & (p[k] < 350.0)), k
    for k in ("wsoi", "wisoi", "fi"):
        assert np.all((p[k] >= 0.0) & (p[k] <= 1.0 + 1e-6)), k
    assert np.all(p["wpud"] >= 0.0) and np.all(p["hsno"] >= 0.0)


def test_a_year_of_the_day_loop_stays_finite_and_physical(cuda_lib):
    """A year of the FP32 day loop -- twelve 30-day months: daily cadence,
    forcing generated from the days' weather, hourly CH4, the month's methane
    at each month's end -- on 4,096 cells of
    the seeded generators: no non-finite column, soil water and ice within
    [0, 1], temperatures within [180, 350] K, carbon pools and annual sums
    non-negative, canopy fractions within [0, 1] and phenology factors within
    their bounds at the end of every month."""
    from ibis_b200.daily import DayLoop
    from ibis_b200.forcing import daily_planes
    from ibis_b200.params import FLAG_CH4, DayParams
    n = 4096
    wl = synth.make_workload(n, 1, seed=3)
    rng = np.random.Generator(np.random.PCG64(4))
    cols = Columns.from_host(wl.prog, wl.stat, dtype=torch.float32, acc=True)
    cols.stat[L.OFF["STAT"]["f_inund"][0], :n] = torch.from_numpy(wl.stat["f_inund"]).to(cols.stat)
    P = wl.params.copy()
    P.flags |= FLAG_CH4
    loop = DayLoop(cols, P, DayParams(), synth.make_dayst(rng, wl.stat, wl.latitude), lat=wl.latitude, seed=2,
                   jday=1)
    daily = torch.from_numpy(daily_planes(synth.make_daily_weather(rng, wl.latitude, 360), cols.ld)).cuda()
    pools = ("clitlm", "clitls", "clitll", "clitrm", "clitrs", "clitrl", "clitwm", "clitws", "clitwl", "csoislop",
             "csoislon", "csoipas", "totcmic", "ayprcp", "storedn")
    for month in range(12):
        loop.run_month(daily[30 * month:30 * (month + 1)], from_mean=True, new_year=month == 0)
        torch.cuda.synchronize()
        assert not cols.nonfinite()[0], month
        p, d = cols.prog_host(), loop.dayst_host()
        for k in ("tsoi", "tg", "tu", "ts", "tl"):
            assert np.all((p[k] > 180.0) & (p[k] < 350.0)), (month, k)
        for k in ("wsoi", "wisoi", "fi"):
            assert np.all((p[k] >= 0.0) & (p[k] <= 1.0 + 1e-6)), (month, k)
        for k in pools:
            assert np.all(np.isfinite(d[k]) & (d[k] >= 0.0)), (month, k)
        for k in ("tempu", "templ", "dropu", "dropls", "dropl3", "dropl4"):
            assert np.all((d[k] >= 0.0) & (d[k] <= 1.0)), (month, k)
        s = synth.from_planes("STAT", cols.stat.cpu().numpy(), n)
        assert np.all((s["frac"] >= 0.0) & (s["frac"] <= 1.0 + 1e-6)), month
        w = loop.wet_host()
        assert np.all(np.isfinite(w["flux"]) & (w["flux"] >= 0.0) & (w["annual"] >= 0.0)), month

