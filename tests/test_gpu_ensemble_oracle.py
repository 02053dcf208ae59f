"""Calibration ensembles and served requests against the float64 oracle.

Each ensemble run is one (site, parameter vector) pair; the oracle runs the
same site columns with ``ensemble.apply_vector`` of the run's vector (the
uniform-parameter equivalent of that run) over the same hourly forcing.  Three
paths are checked against it:

* ``ibis_ensemble_f32`` over hourly records (8 sites x 4 vectors, 48 hours);
* ``ibis_ensemble_daily_f32`` over day records, the hours generated in the
  kernel -- the oracle gets the hours ``ibis_diurnal_f32`` generates from the
  same days with the same variates;
* one request answered by the serving loop (3 sites, 2 model years of 48
  hours): its per-year sums against the oracle's sums over each year;
* every ensemble form under the release parameter file's switches (the kernels
  with the IBIS 3.0 extensions), the oracle under the same switches.

Tolerances (FP32 kernels against float64 after 48 hours): temperatures within
``T_ABS`` K, soil water within ``W_ABS``, and the day-loop sums within
``ACC_REL`` of the largest magnitude of their plane; a served request's per-year
sums within ``SERVE_REL`` (they are differences of running totals at the year
ends), runoff within ``SERVE_RUNOFF_REL`` (surface runoff switches on at
saturation and puddle thresholds, so an hour's FP32 soil water can move its
onset: measured 6.0e-5 with the default parameters and 6.1e-4 under the
release switches, where the other sums stay within 1.4e-5) -- about 10x (runoff
3x) the departures measured on these cases
(``measured_errors``: temperatures 0.26 / 0.55 mK, soil water 1.6e-6, sums
4e-6 / 3.2e-6, served sums 1.4e-5, served runoff 6.1e-4).
"""
import warnings

import numpy as np
import pytest
import torch

import oracle
from ibis_b200 import ensemble as E
from ibis_b200 import layout as L
from ibis_b200 import serve as S
from ibis_b200 import synth

warnings.filterwarnings("ignore", category=RuntimeWarning)
pytestmark = pytest.mark.gpu

T_ABS = 5e-3
W_ABS = 2e-5
ACC_REL = 5e-5
SERVE_REL = 2e-4
SERVE_RUNOFF_REL = 2e-3
TEMPS = ("tsoi", "tg", "tu", "ts", "tl", "t12", "t34", "tsno", "ti", "tsoi_deep")
SUMS = ("aygpptot", "aynpptot", "adaet", "afsena", "aytrunof", "aytdrain", "ch4")


def records_to_forcing(rec):
    """(nsite, N_FORC) forcing records of one hour -> the oracle's forcing dict."""
    out = {}
    for f in L.FORC:
        p0, k = L.OFF["FORC"][f.name]
        out[f.name] = rec[:, p0] if k == 1 else rec[:, p0:p0 + k]
    return out


def oracle_runs(spec, hour_records, vectors, sites, nhour, year_hours=None):
    """The oracle over ``sites`` for ``nhour`` hours under each vector:
    ``hour_records(h)`` gives the (len(sites), N_FORC) records of hour h.
    Returns {vector index: (prog, acc, [acc at each year end])}."""
    out = {}
    stat = {k: np.asarray(v)[sites].astype(np.float64) for k, v in spec.stat.items()}
    for j, v in enumerate(vectors):
        P = E.apply_vector(spec.params, v)
        prog = {k: np.asarray(x)[sites].astype(np.float64) for k, x in spec.prog.items()}
        acc = oracle.new_acc(len(sites))
        snaps = []
        with np.errstate(all="ignore"):
            for h in range(nhour):
                prog, _, acc = oracle.step(prog, stat, records_to_forcing(hour_records(h)), P, acc)
                if year_hours and (h + 1) % year_hours == 0:
                    snaps.append({k: np.array(acc[k]) for k in SUMS})
        out[j] = (prog, acc, snaps)
    return out


def _errors(got_prog, got_acc, want_prog, want_acc):
    e = {"temp": 0.0, "water": 0.0, "acc": 0.0}
    for k in TEMPS:
        e["temp"] = max(e["temp"], float(np.max(np.abs(np.asarray(got_prog[k]) - want_prog[k]))))
    for k in ("wsoi", "wisoi"):
        e["water"] = max(e["water"], float(np.max(np.abs(np.asarray(got_prog[k]) - want_prog[k]))))
    for k in SUMS:
        w = np.asarray(want_acc[k], np.float64)
        scale = max(float(np.max(np.abs(w))), 1e-30)
        e["acc"] = max(e["acc"], float(np.max(np.abs(np.asarray(got_acc[k]) - w))) / scale)
    return e


def release_params():
    """The release parameter file's step parameters (tests/golden/release.npz)
    for an ensemble: its switches and tables, the run accumulators on."""
    from goldens import Case
    from ibis_b200 import params as prm
    P = Case("release").params.copy()
    P.flags |= prm.FLAG_ACC | prm.FLAG_CH4 | prm.FLAG_KAHAN
    return P


def _ensemble_vs_oracle(daily, params=None, hourly=False):
    nsite, nparam, hours = 8, 4, 48
    spec = E.make_ensemble(nsite, nparam, site_hours=np.full(nsite, hours), seed=23, daily=daily, params=params)
    if params is not None:
        # per-site acclimation states for the release file's temperature acclimation
        spec.stat["acclim_x"] = np.random.default_rng(5).uniform(-12.0, 28.0, nsite)
    ens = E.Ensemble(spec, year_steps=24)
    if hourly:
        ens.run_hourly(chunk=24, graph=False)          # one launch per hour
    else:
        ens.run()
    torch.cuda.synchronize()
    assert not ens.nonfinite()[0]
    got_p, got_a = ens.prog_host(), ens.acc_host()
    if daily:
        from ibis_b200 import forcing
        ld = L.leading_dim(nsite)
        lat = torch.zeros(ld, dtype=torch.float32, device="cuda")
        lat[:nsite] = torch.from_numpy(spec.latitude.astype(np.float32)).cuda()
        hourly = np.zeros((hours, nsite, L.N_FORC), np.float32)
        for s in range(nsite):
            d0 = int(spec.site_first[s])
            days = spec.daily[d0:d0 + hours // 24]
            planes = np.zeros((hours // 24, L.N_DAILY, ld), np.float32)
            planes[:, :, s] = days[:, :L.N_DAILY]
            f = forcing.hourly_forcing(torch.from_numpy(planes).cuda(), lat, nsite, jday0=int(days[0, L.N_DAILY]),
                                       day0=d0, seed=spec.weather_seed, observed_fira=True)
            hourly[:, s] = f.cpu().numpy()[:, :, s]
        recs = lambda h: hourly[h].astype(np.float64)
    else:
        recs = lambda h: np.stack([spec.forc[spec.site_first[s] + h] for s in range(nsite)]).astype(np.float64)
    want = oracle_runs(spec, recs, spec.vectors, np.arange(nsite), hours)
    err = {"temp": 0.0, "water": 0.0, "acc": 0.0}
    for j in range(nparam):
        runs = np.arange(nsite) * nparam + j                 # run = site * nparam + vector
        gp = {k: np.asarray(v)[runs] for k, v in got_p.items()}
        ga = {k: np.asarray(v)[runs] for k, v in got_a.items()}
        e = _errors(gp, ga, want[j][0], want[j][1])
        err = {k: max(err[k], e[k]) for k in err}
    return err


def measured_errors():
    """The departures the bounds are set from (run this on a GPU to see them)."""
    return {"ensemble": _ensemble_vs_oracle(False), "ensemble_daily": _ensemble_vs_oracle(True),
            "served": _served_vs_oracle()}


def _served_vs_oracle(params=None):
    year_hours = 48
    lib = S.SiteLibrary(nsite=5, years=2, seed=4, year_hours=year_hours, params=params)
    if params is not None:
        # per-site acclimation states for the release file's temperature acclimation
        lib.spec.stat["acclim_x"] = np.random.default_rng(6).uniform(-12.0, 28.0, 5)
        lib.stat.copy_(torch.from_numpy(synth.to_planes("STAT", lib.spec.stat, lib.ld_site)).to(lib.stat))
    rng = np.random.default_rng(8)
    req = S.Request(rid=0, sites=np.array([0, 2, 4]), years=2, vector=E.draw_vectors(rng, 1)[0], arrival=0.0)
    srv = S.Server(lib, budget_bytes=lib.nbytes + 64 * S.slot_bytes(2), epoch_hours=24)
    srv.serve([req], realtime=False, epoch_seconds=1.0)
    got = srv.results[0].yearly                               # (3, years, N_YEARLY)
    spec = lib.spec
    recs = lambda h: np.stack([spec.forc[spec.site_first[s] + h] for s in req.sites]).astype(np.float64)
    want = oracle_runs(spec, recs, [req.vector], req.sites, 2 * year_hours, year_hours=year_hours)[0][2]
    err, per = 0.0, {}
    for y in range(2):
        for k, f in enumerate(L.YEARLY):
            w = want[y][f.name] - (want[y - 1][f.name] if y else 0.0)
            scale = max(float(np.max(np.abs(w))), 1e-30)
            e = float(np.max(np.abs(got[:, y, k] - w))) / scale
            per[f"{f.name}.{y}"] = e
            if f.name != "aytrunof":
                err = max(err, e)
    return {"acc": err, "runoff": max(per["aytrunof.0"], per["aytrunof.1"]), "per_field": per}


def test_ensemble_runs_match_oracle(cuda_lib):
    e = _ensemble_vs_oracle(False)
    assert e["temp"] < T_ABS and e["water"] < W_ABS and e["acc"] < ACC_REL, e


def test_daily_form_ensemble_runs_match_oracle(cuda_lib):
    e = _ensemble_vs_oracle(True)
    assert e["temp"] < T_ABS and e["water"] < W_ABS and e["acc"] < ACC_REL, e


def test_release_ensemble_runs_match_oracle(cuda_lib):
    """Runs under the release parameter file's switches (the ensemble kernels
    with the IBIS 3.0 extensions) against the oracle under the same switches:
    the persistent launch over hourly records and over day records, and one
    launch per hour."""
    for daily, hourly in ((False, False), (True, False), (False, True)):
        e = _ensemble_vs_oracle(daily, params=release_params(), hourly=hourly)
        assert e["temp"] < T_ABS and e["water"] < W_ABS and e["acc"] < ACC_REL, (daily, hourly, e)


def test_release_switches_change_ensemble_runs(cuda_lib):
    """The same runs without the switches give other conductances, so the
    extended ensemble kernels are not running the F77 step."""
    from ibis_b200.params import X3_FLAGS
    out = []
    for strip in (False, True):
        P = release_params()
        if strip:
            P.flags &= ~X3_FLAGS
        spec = E.make_ensemble(4, 2, site_hours=np.full(4, 24), seed=3, params=P)
        spec.stat["acclim_x"] = np.full(4, 5.0)
        ens = E.Ensemble(spec, year_steps=24)
        ens.run()
        torch.cuda.synchronize()
        out.append(ens.prog_host())
    d = np.abs(np.asarray(out[0]["gs_upper"]) - np.asarray(out[1]["gs_upper"]))
    assert float(np.max(d)) > 1e-6


def test_served_request_matches_oracle(cuda_lib):
    e = _served_vs_oracle()
    assert e["acc"] < SERVE_REL and e["runoff"] < SERVE_RUNOFF_REL, e


def test_served_request_under_release_switches_matches_oracle(cuda_lib):
    """A request served under the release parameter file's switches (the
    ensemble kernels with the IBIS 3.0 extensions) against the oracle."""
    e = _served_vs_oracle(release_params())
    assert e["acc"] < SERVE_REL and e["runoff"] < SERVE_RUNOFF_REL, e
