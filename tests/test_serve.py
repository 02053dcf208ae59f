"""Serving loop: request generation (CPU) and continuous batching on the GPU.

A request's yearly sums must be the same bits whether it is served alone or
admitted while other requests are in flight, whatever the epoch boundaries and
the slots it lands in: every run is advanced by the same persistent-kernel
code, and the state it carries between epochs is stored and reloaded exactly.
They must also equal the same runs in one ``Ensemble`` launch.
"""
import numpy as np
import pytest
import torch

from ibis_b200 import ensemble as E
from ibis_b200 import layout as L
from ibis_b200 import serve as S


def test_poisson_requests_shape():
    rng = np.random.default_rng(0)
    reqs = S.poisson_requests(rng, rate=50.0, duration=40.0, nsite_lib=356)
    n = len(reqs)
    assert abs(n - 2000) < 4 * np.sqrt(2000)
    arr = np.array([r.arrival for r in reqs])
    assert np.all(np.diff(arr) > 0) and arr[-1] <= 40.0
    gaps = np.diff(arr)
    assert abs(gaps.mean() - 0.02) < 0.002
    ns = np.array([len(r.sites) for r in reqs])
    ys = np.array([r.years for r in reqs])
    assert ns.min() >= 1 and ns.max() <= 64 and ys.min() >= 1 and ys.max() <= 10
    assert all(len(set(r.sites.tolist())) == len(r.sites) for r in reqs)
    assert all(r.vector.shape == (L.N_RUN,) for r in reqs)


def test_slot_bytes():
    assert S.slot_bytes(10) == 4 * (71 + 104 + 31 + 70) + 28


# ---------------------------------------------------------------- GPU

def _library():
    return S.SiteLibrary(nsite=6, years=3, seed=1, year_hours=24)


def _requests(rng, n, t0=0.0, start=1):
    out = []
    for i in range(n):
        k = int(rng.integers(1, 5))
        out.append(S.Request(rid=start + i, sites=np.sort(rng.choice(6, size=k, replace=False)),
                             years=int(rng.integers(1, 4)), vector=E.draw_vectors(rng, 1)[0],
                             arrival=t0 + 0.5 * i))
    return out


@pytest.mark.gpu
def test_request_alone_equals_request_in_mix(cuda_lib):
    lib = _library()
    rng = np.random.default_rng(4)
    r0 = S.Request(rid=0, sites=np.array([1, 3, 4]), years=3, vector=E.draw_vectors(rng, 1)[0], arrival=0.0)
    alone = S.Server(lib, budget_bytes=lib.nbytes + 64 * S.slot_bytes(3), epoch_hours=5)
    st = alone.serve([r0], realtime=False, epoch_seconds=1.0)
    assert st["requests"] == 1
    a = alone.results[0]
    others = _requests(rng, 12)
    mixed_r0 = S.Request(rid=0, sites=r0.sites, years=3, vector=r0.vector, arrival=2.0)
    mix = S.Server(lib, budget_bytes=lib.nbytes + 64 * S.slot_bytes(3), epoch_hours=7)
    st = mix.serve(others + [mixed_r0], realtime=False, epoch_seconds=1.0)
    assert st["requests"] == 13 and st["status"][0] == 0
    b = mix.results[0]
    assert b.admitted > 0.0                    # joined while other requests were running
    np.testing.assert_array_equal(a.yearly, b.yearly)
    assert a.yearly.shape == (3, 3, L.N_YEARLY) and np.isfinite(a.yearly).all()
    assert not a.nonfinite and not b.nonfinite


@pytest.mark.gpu
def test_served_request_equals_ensemble_launch(cuda_lib):
    lib = _library()
    v = E.draw_vectors(np.random.default_rng(9), 1)[0]
    srv = S.Server(lib, budget_bytes=lib.nbytes + 64 * S.slot_bytes(3), epoch_hours=10)
    srv.serve([S.Request(rid=7, sites=np.arange(6), years=3, vector=v)], realtime=False, epoch_seconds=1.0)
    spec = lib.spec
    spec2 = E.EnsembleSpec(nsite=spec.nsite, nparam=1, site_hours=spec.site_hours, stat=spec.stat, prog=spec.prog,
                           forc=spec.forc, site_first=spec.site_first, vectors=v[None].copy(), params=spec.params,
                           latitude=spec.latitude)
    ens = E.Ensemble(spec2, year_steps=24)
    ens.run()
    torch.cuda.synchronize()
    np.testing.assert_array_equal(srv.results[7].yearly, ens.yearly_sums())


@pytest.mark.gpu
def test_admission_waits_for_free_slots(cuda_lib):
    lib = _library()
    rng = np.random.default_rng(11)
    reqs = _requests(rng, 20, start=0)
    big = S.Server(lib, budget_bytes=lib.nbytes + 4096 * S.slot_bytes(3), epoch_hours=6)
    big.serve(reqs, realtime=False, epoch_seconds=1.0)
    small = S.Server(lib, budget_bytes=lib.nbytes + 32 * S.slot_bytes(3) + 100, epoch_hours=6)
    assert small.nslot == 32
    st = small.serve(reqs, realtime=False, epoch_seconds=1.0)
    assert st["requests"] == 20
    for r in reqs:
        np.testing.assert_array_equal(small.results[r.rid].yearly, big.results[r.rid].yearly)
    assert st["p50_s"] <= st["p99_s"]


@pytest.mark.gpu
def test_realtime_loop_reports_latency(cuda_lib):
    lib = _library()
    rng = np.random.default_rng(3)
    reqs = S.poisson_requests(rng, rate=50.0, duration=0.5, nsite_lib=6, max_sites=6, max_years=3)
    srv = S.Server(lib, budget_bytes=lib.nbytes + 1024 * S.slot_bytes(3), epoch_hours=24)
    st = srv.serve(reqs)
    assert st["requests"] == len(reqs) and st["p99_s"] >= st["p50_s"] > 0.0
    assert all(r.done >= r.arrival for r in srv.results.values())


@pytest.mark.gpu
def test_daily_library_request_alone_equals_in_mix_and_ensemble(cuda_lib):
    """A library of day records (hours generated in the kernel): a request's
    result is the same bits alone, in a mix admitted mid-flight, and as one
    persistent daily-form ensemble launch of the same runs."""
    lib = S.SiteLibrary(nsite=6, years=3, seed=1, year_hours=48, daily=True)
    assert lib.forc.shape == (6 * 3 * 2, E.DAILY_WORDS)
    rng = np.random.default_rng(6)
    r0 = S.Request(rid=0, sites=np.array([0, 2, 5]), years=3, vector=E.draw_vectors(rng, 1)[0], arrival=0.0)
    alone = S.Server(lib, budget_bytes=lib.nbytes + 64 * S.slot_bytes(3), epoch_hours=24)
    alone.serve([r0], realtime=False, epoch_seconds=1.0)
    a = alone.results[0]
    others = _requests(rng, 10)
    mix = S.Server(lib, budget_bytes=lib.nbytes + 64 * S.slot_bytes(3), epoch_hours=72)
    st = mix.serve(others + [S.Request(rid=0, sites=r0.sites, years=3, vector=r0.vector, arrival=2.0)],
                   realtime=False, epoch_seconds=1.0)
    assert st["requests"] == 11 and st["status"][0] == 0 and mix.results[0].admitted > 0.0
    np.testing.assert_array_equal(a.yearly, mix.results[0].yearly)
    assert np.isfinite(a.yearly).all() and not a.nonfinite
    spec = lib.spec
    sub = E.EnsembleSpec(nsite=spec.nsite, nparam=1, site_hours=spec.site_hours, stat=spec.stat, prog=spec.prog,
                         forc=None, site_first=spec.site_first, vectors=r0.vector[None].copy(), params=spec.params,
                         latitude=spec.latitude, daily=spec.daily, weather_seed=spec.weather_seed)
    ens = E.Ensemble(sub, year_steps=48)
    ens.run()
    torch.cuda.synchronize()
    np.testing.assert_array_equal(a.yearly, ens.yearly_sums()[r0.sites])
    with pytest.raises(ValueError):
        S.Server(lib, budget_bytes=lib.nbytes + 64 * S.slot_bytes(3), epoch_hours=30)


@pytest.mark.gpu
def test_plain_per_request_form_runs(cuda_lib):
    """serve_plain (one launch per request, one at a time) answers every request
    with a finite latency and runs every hour of every run."""
    lib = _library()
    reqs = _requests(np.random.default_rng(11), 4)
    pl = S.serve_plain(lib, reqs)
    assert pl["requests"] == 4 and np.isfinite(pl["p99_s"]) and pl["p50_s"] > 0.0
    assert pl["cell_steps"] == sum(len(r.sites) * r.years * lib.year_hours for r in reqs)
