"""Wetland area of the monthly methane on the GPU, against the reference and the oracle.

* Feature builder (``ibis_wetland_features``): the reference's own predictors
  over 9 months on a 12 x 20 grid (``tests/golden/wetland_area.npz``), bit for
  bit; and the oracle's on the global 0.5-degree grid (360 x 720, 60 % land)
  over 5 months, bit for bit (float64 in the reference's operation order, no
  FMA contraction).
* Dynamic area (``ibis_wetland_dynamic_f32``): the oracle on the same state,
  bit for bit after the float32 cast the kernel writes.
* Learned fraction (``ibis_wetland_learned``): the oracle's restatement of the
  file's boosters (random depth-6 forests with thresholds inside the
  predictors' ranges, 3 bands, missing values routed by default direction),
  bit for bit after the float32 cast.
* The learned month on a day loop (``run_month_learned``): its fraction equals
  the oracle's from the same month's means and totals (read from a second,
  identical loop run at unit fraction) within 1e-6 -- the device forms the
  month means in float32 from Kahan-compensated sums, the check in float64 --
  and the month's flux equals the unit-fraction flux times that fraction.
"""
import os

import numpy as np
import pytest
import torch

from oracle import wetland as W
from wetland_models import random_booster
from ibis_b200 import layout as L
from ibis_b200 import wetland as WD

pytestmark = pytest.mark.gpu
GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "wetland_area.npz"))


def test_feature_builder_equals_reference(cuda_lib):
    z = GOLD
    fb = WD.FeatureBuilder(z["in.I"], z["in.J"], z["in.poros"], z["in.hsoi"], int(z["in.nlat"]), int(z["in.nlon"]))
    for t in range(z["in.ws"].shape[0]):
        f = fb.step_host(z["in.ts"][t], z["in.ws"][t], z["in.wi"][t], z["in.tg"][t], z["in.prcp"][t],
                         z["in.aet"][t], z["in.runoff"][t])
        for k, name in enumerate(WD.DYN_FEATS):
            np.testing.assert_array_equal(f[name], z["out.feats"][t, k], err_msg=f"month {t} {name}")


def _global_points(rng, frac=0.6):
    I, J = np.where(rng.random((360, 720)) < frac)
    return I, J


def test_feature_builder_equals_oracle_on_the_global_grid(cuda_lib):
    rng = np.random.default_rng(7)
    I, J = _global_points(rng)
    n = len(I)
    poros = rng.uniform(0.3, 0.6, (n, 6))
    hsoi = np.array([0.10, 0.15, 0.25, 0.50, 1.0, 2.0])
    fb = WD.FeatureBuilder(I, J, poros, hsoi)
    ob = W.FeatureBuilder(I, J, poros, hsoi)
    for t in range(5):
        args = [rng.uniform(250.0, 300.0, (n, 6)), rng.uniform(0.0, 1.0, (n, 6)), rng.uniform(0.0, 0.3, (n, 6)),
                rng.uniform(250.0, 300.0, n), rng.uniform(0.0, 200.0, n), rng.uniform(0.0, 100.0, n),
                rng.uniform(0.0, 80.0, n)]
        args = [np.asarray(a, np.float32) for a in args]
        got, want = fb.step_host(*args), ob.step(*args)
        for name in WD.DYN_FEATS:
            np.testing.assert_array_equal(got[name], want[name], err_msg=f"month {t} {name}")


def test_dynamic_fraction_equals_oracle(cuda_lib):
    from ibis_b200.columns import Columns
    from ibis_b200 import synth
    z = GOLD
    n = len(z["in.I"])
    wl = synth.make_workload(n, 1, seed=3)
    cols = Columns.from_host(wl.prog, wl.stat, dtype=torch.float32, acc=False)
    prog = cols.prog.cpu().numpy()
    stat = cols.stat.cpu().numpy()
    # the golden month's soil state in the columns
    prog[L.OFF["PROG"]["wsoi"][0]:L.OFF["PROG"]["wsoi"][0] + 6, :n] = z["in.ws"][0].T
    prog[L.OFF["PROG"]["tsoi"][0]:L.OFF["PROG"]["tsoi"][0] + 6, :n] = z["in.ts"][0].T
    stat[L.OFF["STAT"]["poros"][0]:L.OFF["STAT"]["poros"][0] + 6, :n] = z["in.poros"].T
    cols.prog.copy_(torch.from_numpy(prog))
    cols.stat.copy_(torch.from_numpy(stat))
    area = np.zeros((6, cols.ld))
    for k, key in enumerate(("in.fclim", "in.mu", "in.sd", "in.beta", "in.fmin", "in.fmax")):
        area[k, :n] = z[key]
    f = WD.dynamic_fraction(cols, torch.from_numpy(area).cuda(), params=wl.params).cpu().numpy()[:n]
    ws = prog[L.OFF["PROG"]["wsoi"][0]:L.OFF["PROG"]["wsoi"][0] + 6, :n].T
    ts = prog[L.OFF["PROG"]["tsoi"][0]:L.OFF["PROG"]["tsoi"][0] + 6, :n].T
    por = stat[L.OFF["STAT"]["poros"][0]:L.OFF["STAT"]["poros"][0] + 6, :n].T
    Wz = W.root_zone_water(ws, por, np.asarray(wl.params.hsoi, np.float64), ts)
    want = W.dynamic_fraction(z["in.fclim"], Wz, z["in.mu"], z["in.sd"], z["in.beta"], z["in.fmin"], z["in.fmax"],
                              frozen=np.asarray(ts[:, 0], np.float64) <= W.T_FREEZE)
    np.testing.assert_array_equal(f, want.astype(np.float32))


def _trained(rng, I, J, ncell_file, nband=3):
    nf = len(W.DYN_FEATS) + len(W.STAT_FEATS)
    lo = np.concatenate([np.zeros(len(W.DYN_FEATS)), np.zeros(len(W.STAT_FEATS))])
    hi = np.concatenate([np.full(len(W.DYN_FEATS), 100.0), np.ones(len(W.STAT_FEATS))])
    pick = rng.choice(len(I), ncell_file, replace=False)
    cI = np.concatenate([I[pick], [359]])            # one cell of the file outside the run's land
    cJ = np.concatenate([J[pick], [719]])
    m = len(cI)
    return dict(dyn_feats=np.array(W.DYN_FEATS), stat_feats=np.array(W.STAT_FEATS), cells_I=cI, cells_J=cJ,
                band=rng.integers(0, nband, m), pbar=rng.uniform(0.0, 1.0, (12, m)),
                fclim=rng.uniform(0.0, 0.5, (12, m)), fmax=rng.uniform(0.05, 1.0, m),
                lam=rng.uniform(0.5, 3.0, nband), stat=rng.random((m, len(W.STAT_FEATS))),
                models=np.array([random_booster(rng, ntree=40, depth=6, nfeat=nf, lo=lo, hi=hi)
                                 for _ in range(nband)]))


def test_learned_fraction_equals_oracle(cuda_lib):
    rng = np.random.default_rng(11)
    I, J = _global_points(rng, 0.05)
    n = len(I)
    tf = _trained(rng, I, J, min(2000, n))
    lw = WD.LearnedWetland(tf, I, J)
    lo = W.LearnedWetland(tf, I, J)
    assert lw.n_dropped == 1 == lo.n_dropped and np.array_equal(lw.pts, lo.pts)
    feats = {k: rng.uniform(0.0, 100.0, n) for k in W.DYN_FEATS}
    feats["W"][:50] = np.nan                           # missing predictors take the default direction
    fd = np.zeros((len(W.DYN_FEATS), lw.ld))
    for k, name in enumerate(W.DYN_FEATS):
        fd[k, :n] = feats[name]
    base = np.zeros(lw.ld, np.float32)
    base[:n] = rng.uniform(-0.1, 1.1, n)
    for imonth in (0, 7):
        got = lw.fraction(imonth, torch.from_numpy(fd).cuda(), torch.from_numpy(base).cuda()).cpu().numpy()[:n]
        want = lo.fraction(imonth, feats, base[:n].astype(np.float64))
        np.testing.assert_array_equal(got, want.astype(np.float32), err_msg=f"month {imonth}")
    # the reference's call form: predictor dict and base fraction on the host
    got = lw.fraction_host(3, feats, base[:n])
    np.testing.assert_array_equal(got, lo.fraction(3, feats, base[:n].astype(np.float64)).astype(np.float32))


def test_learned_month_on_the_day_loop(cuda_lib):
    from ibis_b200 import forcing as _forcing
    from ibis_b200 import synth
    from ibis_b200.columns import Columns
    from ibis_b200.daily import DayLoop
    from ibis_b200.params import FLAG_CH4, FLAG_SOIL_MEANS, DayParams
    rng = np.random.default_rng(5)
    ncell, nday = 512, 4
    I = rng.permutation(360 * 720)[:ncell]
    I, J = I // 720, I % 720
    wl = synth.make_workload(ncell, 1, seed=21)
    drng = np.random.Generator(np.random.PCG64(22))
    dayst = synth.make_dayst(drng, wl.stat, wl.latitude)
    daily = torch.from_numpy(_forcing.daily_planes(synth.make_daily_weather(drng, wl.latitude, nday),
                                                   L.leading_dim(ncell))).cuda()

    def loop():
        cols = Columns.from_host(wl.prog, wl.stat, dtype=torch.float32, acc=True)
        P = wl.params.copy()
        P.flags |= FLAG_CH4 | FLAG_SOIL_MEANS
        return DayLoop(cols, P, DayParams(), dayst, lat=wl.latitude, seed=5, jday=152, day=0)

    poros = np.asarray(wl.stat["poros"], np.float64)
    tf = _trained(rng, I, J, 300)
    base = torch.zeros(L.leading_dim(ncell), dtype=torch.float32, device="cuda")
    base[:ncell] = torch.from_numpy(rng.uniform(0.0, 0.3, ncell).astype(np.float32))

    a = loop()
    fb = WD.FeatureBuilder(I, J, poros, wl.params.hsoi)
    lw = WD.LearnedWetland(tf, I, J)
    f = WD.run_month_learned(a, daily, fb, lw, 5, base).cpu().numpy()[:ncell]
    torch.cuda.synchronize()
    assert not a.cols.nonfinite()[0]

    # the same month at unit fraction, its means and totals read on the host
    b = loop()
    c = b.cols
    planes = list(range(L.OFF["ACC"]["tsoi_mean"][0], L.OFF["ACC"]["tsoi_mean"][0] + 19))
    tr, dr = L.OFF["ACC"]["aytrunof"][0], L.OFF["ACC"]["aytdrain"][0]

    def acc_vals():
        A = c.acc.cpu().numpy().astype(np.float64)
        return A[:L.N_ACC] - A[L.N_ACC:]

    b.begin_month(False)
    c.stat[L.OFF["STAT"]["f_inund"][0]].fill_(1.0)
    a0, d0 = acc_vals(), b.dayst.cpu().numpy().astype(np.float64)
    b.run(daily)
    b.end_month(nday, True, None, False)
    a1, d1 = acc_vals(), b.dayst.cpu().numpy().astype(np.float64)
    m = ((a1 - a0)[planes] / nday)[:, :ncell]
    dp, da = L.OFF["DAYST"]["ayprcp"][0], L.OFF["DAYST"]["ayaet"][0]
    ob = W.FeatureBuilder(I, J, poros, wl.params.hsoi)
    feats = ob.step(m[0:6].T, m[6:12].T, m[12:18].T, m[18], (d1 - d0)[dp, :ncell], (d1 - d0)[da, :ncell],
                    ((a1 - a0)[tr] + (a1 - a0)[dr])[:ncell])
    want = W.LearnedWetland(tf, I, J).fraction(5, feats, base.cpu().numpy()[:ncell].astype(np.float64))
    np.testing.assert_allclose(f, want, rtol=0, atol=1e-6)
    # the month's flux scaled by the fraction (scale_month)
    flux_a = a.wet[L.OFF["WET"]["flux"][0]].cpu().numpy()[:ncell]
    flux_b = b.wet[L.OFF["WET"]["flux"][0]].cpu().numpy()[:ncell]
    np.testing.assert_allclose(flux_a, flux_b * f, rtol=1e-6, atol=1e-12)
