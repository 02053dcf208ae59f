"""Known-answer and property tests the reference's own suite applies to this path.

Mirrors python-port/tests/test_thermo.py, test_solvers.py, test_bedrock.py,
test_water_balance.py, test_methane_m1.py and test_f77_verification.py (qglif).
"""
import numpy as np
import pytest

from oracle import physics as ph
from oracle import column as col
import oracle
from ibis_b200 import synth
from ibis_b200.params import StepParams


def test_esat_at_freezing():                      # test_thermo.py:14-17
    assert float(ph.esat(np.array(273.16))) == pytest.approx(610.78, rel=1e-3)


def test_esat_monotonic_and_branches():          # test_thermo.py:19-35
    t = np.linspace(240.0, 320.0, 50)
    assert np.all(np.diff(ph.esat(t)) > 0)
    assert 3000.0 < float(ph.esat(np.array(300.0))) < 5000.0
    assert 0.0 < float(ph.esat(np.array(250.0))) < float(ph.esat(np.array(273.16)))


def test_latent_heats_at_tmelt():                # test_thermo.py:127, 148
    P = StepParams()
    t = np.array([P.tmelt])
    assert ph.hvapf(t, t, P)[0] == pytest.approx(P.hvap, rel=1e-10)
    assert ph.hsubf(t, t, P)[0] == pytest.approx(P.hsub, rel=1e-10)


@pytest.mark.parametrize("n", [3, 6, 9])
def test_thomas_matches_dense(n):                # test_solvers.py:36-60
    rng = np.random.default_rng(n)
    m = 5
    lo, up = rng.uniform(-1, 0, (m, n)), rng.uniform(-1, 0, (m, n))
    di = 3.0 + rng.uniform(0, 1, (m, n))
    r = rng.normal(size=(m, n))
    x = ph.thomas(lo, di, up, r)
    for i in range(m):
        A = np.diag(di[i]) + np.diag(lo[i, 1:], -1) + np.diag(up[i, :-1], 1)
        np.testing.assert_allclose(x[i], np.linalg.solve(A, r[i]), atol=1e-12)


def test_bedrock_heat_solve_conserves_energy_in_float64():   # test_bedrock.py:198-223
    P = StepParams()
    n = 4
    rng = np.random.default_rng(0)
    hs = np.concatenate([P.hsoi, P.hsoi_bed])
    nl = hs.size
    z = np.zeros((n, 3))
    poros = np.concatenate([np.full((n, 6), 0.45), z], 1)
    wsoi = np.concatenate([rng.uniform(0.2, 0.9, (n, 6)), z], 1)
    wisoi = np.concatenate([rng.uniform(0.0, 0.3, (n, 6)), z], 1)
    csoi = np.concatenate([np.full((n, 6), 880.5), np.full((n, 3), P.csoi_bed)], 1)
    rho = np.concatenate([np.full((n, 6), 2636.5), np.full((n, 3), P.rhosoi_bed)], 1)
    con = np.concatenate([rng.uniform(0.5, 2.0, (n, 6)), np.full((n, 3), P.consoi_bed)], 1)
    t = 275.0 + rng.uniform(0, 10, (n, nl))
    fh = rng.normal(0, 50, n)
    zc = np.zeros((n, nl))
    tn, _ = col.soil_heat(t, t, wsoi, wsoi, wisoi, poros, con, csoi, rho, hs, zc, zc, fh,
                          np.zeros((n, nl + 1)), 6, P)
    cv = (1 - poros) * csoi * rho + poros * (1 - wisoi) * P.ch2o * P.rhow * wsoi + poros * wisoi * P.cice * P.rhow
    dE = np.sum(cv * hs[None, :] * (tn - t), axis=1)
    np.testing.assert_allclose(dE, fh * P.dtime, rtol=1e-10)


def test_qglif_partitions_sum_to_one():           # test_f77_verification.py:264
    wl = synth.make_workload(64, 1, seed=3, edge_cases=True)
    wl.prog["wpud"][::3] = 2.0
    wl.prog["wsoi"][::5, 0] = 0.0
    _, q, _, _ = ph.setsoi(wl.stat, wl.prog, wl.prog["tsno"][:, 0], wl.forc["ta"][0], wl.params)
    # with water in the top layer the four sources partition the flux; a dry layer under a puddle
    # gives the puddle only its covered share zwpud (F77 soil.f:135-160), which the reference keeps
    w0, i0 = wl.prog["wsoi"][:, 0], wl.prog["wisoi"][:, 0]
    wet = (1.0 - i0) * w0 + i0 >= wl.params.epsilon
    assert wet.sum() > 40 and (~wet).sum() > 5
    np.testing.assert_allclose(q[wet].sum(axis=1), 1.0, atol=1e-12)


@pytest.mark.parametrize("wsoi,rain", [(0.6, 0.0), (0.98, 2.0e-3), (1.0, 5.0e-3)])
def test_column_water_balance_closes(wsoi, rain):  # test_water_balance.py:36-49
    wl = synth.make_workload(8, 1, seed=4)
    P = wl.params
    wl.prog["wsoi"][:] = wsoi
    F = wl.forcing_at(0)
    F["raina"][:] = rain
    F["snowa"][:] = 0.0

    def water(p):
        por = wl.stat["poros"]
        soil = np.sum(P.hsoi[None, :] * por * P.rhow * ((1 - p["wisoi"]) * p["wsoi"] + p["wisoi"]), axis=1)
        return soil + p["wpud"] + p["wipud"]
    with np.errstate(all="ignore"):
        new, D, _ = oracle.step(wl.prog, wl.stat, F, P)
    resid = (water(new) - water(wl.prog)) - (D["raing_avg"] - (D["gsuvap"] + D["gtrans"] + D["grunof"] + D["gdrain"])) * P.dtime
    scale = np.maximum(np.abs(D["raing_avg"]) + np.abs(D["gsuvap"] + D["gtrans"] + D["grunof"] + D["gdrain"]), 1e-6) * P.dtime
    assert np.all(np.abs(resid) <= 0.02 * scale + 0.05)


def test_methane_zero_when_frozen_and_grows_with_wetness():   # test_methane_m1.py:216-426
    P = StepParams()
    n = 5
    t = np.full((n, 6), 260.0)
    w = np.linspace(0.2, 1.0, n)[:, None] * np.ones((1, 6))
    i = np.zeros((n, 6))
    f = col.methane(np.full(n, 0.2), np.full(n, 1e-3), t, w, i, np.asarray(P.hsoi), P)
    assert np.all(f == 0.0)
    f = col.methane(np.full(n, 0.2), np.full(n, 1e-3), t + 30.0, w, i, np.asarray(P.hsoi), P)
    assert np.all(f > 0.0) and np.all(np.diff(f) >= 0.0)
