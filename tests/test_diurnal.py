"""Daily-to-hourly forcing: the oracle against the reference's own
``compute_precip_timing`` / ``diurnal`` (tests/golden/diurnal.npz, CPU), and the
device generator against the oracle (GPU).

The reference draws its variates from jax.random; the fixture was made with
the counter-based variates the device generator draws, so both are pinned by
the same file.  Tolerances: oracle vs reference 1e-12 relative; the FP32
device generator vs the float64 oracle 2e-5 relative on temperatures,
pressure and longwave, 1e-4 on humidity and wind, absolute 1e-3 W m-2 on
shortwave and 1e-6 on the cosine of the zenith angle; the precipitation event
(length, start, and which hours carry rain or snow) exactly.
"""
import os

import numpy as np
import pytest

from oracle import weather as W

HERE = os.path.dirname(os.path.abspath(__file__))


def _golden():
    z = np.load(os.path.join(HERE, "golden", "diurnal.npz"))
    return {k: z[k] for k in z.files}


def _daily(z):
    return {k[9:]: v for k, v in z.items() if k.startswith("in.daily.")}


def test_uniform24_properties():
    u = W.uniform24(7, np.arange(200000), 3, 9)
    assert u.min() >= 0.0 and u.max() < 1.0 and abs(u.mean() - 0.5) < 0.005
    assert np.all(u * (1 << 24) == np.floor(u * (1 << 24)))          # 24-bit fractions
    assert not np.array_equal(u, W.uniform24(7, np.arange(200000), 3, 10))
    assert not np.array_equal(u, W.uniform24(8, np.arange(200000), 3, 9))
    assert W.uniform24(7, np.array([5]), 3, 9)[0] == u[5]


def test_oracle_matches_reference_diurnal():
    z = _golden()
    d = _daily(z)
    lat, dtime, seed = z["in.lat"], float(z["in.dtime"]), int(z["in.seed"])
    cells = np.arange(lat.size)
    for di, jday in enumerate(z["in.days"]):
        plens, startp, endp = W.precip_timing(W.uniform24(seed, cells, di, 0), W.uniform24(seed, cells, di, 1),
                                              d["precip"], dtime)
        for k, v in (("plens", plens), ("startp", startp), ("endp", endp)):
            np.testing.assert_array_equal(v, z[f"out.{di}.{k}"], err_msg=k)
        for h in range(24):
            f = W.diurnal(h * dtime, int(jday), d, lat, plens, startp, endp, W.uniform24(seed, cells, di, 2 + h),
                          dtime)
            for k in ("coszen", "ta", "qa", "ua", "fira", "raina", "snowa", "solad", "solai"):
                np.testing.assert_allclose(f[k], z[f"out.{di}.{h}.{k}"], rtol=1e-12, atol=1e-300,
                                           err_msg=f"{di} {h} {k}")


def test_fixture_covers_the_regimes():
    z = _golden()
    assert z["out.0.plens"][0] > z["out.0.plens"][5] or z["out.0.plens"][0] == 86400.0   # 400 mm: long event
    assert np.all(np.array([z[f"out.1.{h}.coszen"][2] for h in range(24)]) > 0.0)       # midnight sun (80 N, day 172)
    assert np.all(np.array([z[f"out.1.{h}.coszen"][3] for h in range(24)]) == 0.0)      # polar night (80 S)
    snow = sum(float(z[f"out.0.{h}.snowa"].sum()) for h in range(24))
    rain = sum(float(z[f"out.1.{h}.raina"].sum()) for h in range(24))
    assert snow > 0.0 and rain > 0.0


# ---------------------------------------------------------------- GPU

def _oracle_day(d32, lat32, jday, day, seed, fira_obs=False):
    """Oracle forcing of one day for float32-rounded inputs."""
    d = {k: np.asarray(v, np.float32).astype(np.float64) for k, v in d32.items()}
    lat = np.asarray(lat32, np.float32).astype(np.float64)
    cells = np.arange(lat.size)
    plens, startp, endp = W.precip_timing(W.uniform24(seed, cells, day, 0), W.uniform24(seed, cells, day, 1),
                                          d["precip"], 3600.0)
    hours = [W.diurnal(h * 3600.0, jday, d, lat, plens, startp, endp, W.uniform24(seed, cells, day, 2 + h), 3600.0,
                       fira_obs=d["fira"] if fira_obs else None) for h in range(24)]
    return hours


@pytest.mark.gpu
@pytest.mark.parametrize("observed", [False, True])
def test_device_generator_matches_oracle(cuda_lib, observed):
    import torch
    from ibis_b200 import forcing, layout as L, synth
    z = _golden()
    d, lat = _daily(z), z["in.lat"]
    n = lat.size
    ld = L.leading_dim(n)
    seed = 7
    lat_t = torch.zeros(ld, dtype=torch.float32, device="cuda")
    lat_t[:n] = torch.from_numpy(lat.astype(np.float32)).cuda()
    for di, jday in enumerate(z["in.days"]):
        planes = forcing.daily_planes({k: v[None] for k, v in d.items()}, ld)
        out = forcing.hourly_forcing(torch.from_numpy(planes).cuda(), lat_t, n, jday0=int(jday), day0=di, seed=seed,
                                     observed_fira=observed)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        want = _oracle_day(d, lat, int(jday), di, seed, observed)
        for h in range(24):
            g = synth.from_planes("FORC", got[h], n)
            w = want[h]
            for k, rt in (("ta", 2e-5), ("psurf", 2e-5), ("fira", 2e-5), ("qa", 1e-4), ("ua", 1e-4)):
                np.testing.assert_allclose(g[k], w[k], rtol=rt, err_msg=f"{di} {h} {k}")
            np.testing.assert_allclose(g["coszen"], w["coszen"], atol=1e-6, err_msg=f"{di} {h} coszen")
            for k in ("solad", "solai"):
                np.testing.assert_allclose(g[k], w[k], rtol=1e-4, atol=1e-3, err_msg=f"{di} {h} {k}")
            for k in ("raina", "snowa"):
                np.testing.assert_array_equal(g[k] > 0, w[k] > 0, err_msg=f"{di} {h} {k} event hours")
                np.testing.assert_allclose(g[k], w[k], rtol=1e-6, err_msg=f"{di} {h} {k}")


@pytest.mark.gpu
def test_generated_forcing_drives_the_step(cuda_lib):
    """A day of generated forcing runs through the FP32 step with finite results,
    and regenerating a day (same seed and day index) gives the same bits."""
    import torch
    from ibis_b200 import forcing, synth
    from ibis_b200.columns import Columns
    wl = synth.make_workload(256, 1, seed=3)
    cols = Columns.from_host(wl.prog, wl.stat)
    rng = np.random.default_rng(0)
    daily = {"tmax": np.full((3, 256), 290.0) + rng.uniform(0, 8, (3, 256)), "tmin": np.full((3, 256), 280.0),
             "cloud": rng.uniform(0, 1, (3, 256)), "precip": rng.gamma(0.5, 6.0, (3, 256)),
             "psurf": np.full((3, 256), 101300.0), "qd": np.full((3, 256), 0.008), "ud": np.full((3, 256), 3.0),
             "fira": np.full((3, 256), 330.0)}
    dp = torch.from_numpy(forcing.daily_planes(daily, cols.ld)).cuda()
    lat = torch.from_numpy(np.pad(wl.latitude.astype(np.float32), (0, cols.ld - 256))).cuda()
    f = forcing.hourly_forcing(dp, lat, 256, jday0=100, seed=11)
    again = forcing.hourly_forcing(dp[1:2].contiguous(), lat, 256, jday0=101, day0=1, seed=11)
    assert torch.equal(f[24:48], again)
    cols.run(f, wl.params)
    torch.cuda.synchronize()
    assert not cols.nonfinite()[0]


def _sw_golden():
    z = np.load(os.path.join(HERE, "golden", "observed_sw.npz"))
    return {k: z[k] for k in z.files}


def test_oracle_matches_reference_observed_shortwave():
    z = _sw_golden()
    for d in range(4):
        a, b = W.observed_shortwave(z[f"{d}.sw"], z[f"{d}.use"], z[f"{d}.coszen"], int(z[f"{d}.jday"]),
                                    z[f"{d}.solad_gen"], z[f"{d}.solai_gen"])
        np.testing.assert_allclose(a, z[f"{d}.solad"], rtol=1e-12, atol=1e-300)
        np.testing.assert_allclose(b, z[f"{d}.solai"], rtol=1e-12, atol=1e-300)
    assert (z["0.coszen"] <= 0).any() and z["0.use"].any() and (~z["0.use"]).any()


@pytest.mark.gpu
def test_device_observed_shortwave_matches_oracle(cuda_lib):
    """Generated forcing with an observed hourly shortwave on the cell-days
    marked: shortwave = the oracle's observed_shortwave of the generator's hour
    within 1e-4 relative / 1e-3 W m-2; every other field as without it."""
    import torch
    from ibis_b200 import forcing, layout as L, synth
    z = _golden()
    d, lat = _daily(z), z["in.lat"]
    n = lat.size
    ld = L.leading_dim(n)
    rng = np.random.Generator(np.random.PCG64(5))
    lat_t = torch.zeros(ld, dtype=torch.float32, device="cuda")
    lat_t[:n] = torch.from_numpy(lat.astype(np.float32)).cuda()
    for di, jday in enumerate(z["in.days"]):
        planes = torch.from_numpy(forcing.daily_planes({k: v[None] for k, v in d.items()}, ld)).cuda()
        sw = np.zeros((1, 24, ld), np.float32)
        sw[0, :, :n] = rng.uniform(-20.0, 1100.0, (24, n))
        use = np.zeros((1, ld), np.uint8)
        use[0, :n] = rng.uniform(size=n) < 0.6
        plain = forcing.hourly_forcing(planes, lat_t, n, jday0=int(jday), day0=di, seed=7)
        got = forcing.hourly_forcing(planes, lat_t, n, jday0=int(jday), day0=di, seed=7,
                                     sw_obs=torch.from_numpy(sw).cuda(), use=torch.from_numpy(use).cuda())
        torch.cuda.synchronize()
        got, plain = got.cpu().numpy(), plain.cpu().numpy()
        for h in range(24):
            g = synth.from_planes("FORC", got[h], n)
            p = synth.from_planes("FORC", plain[h], n)
            for k in g:
                if k not in ("solad", "solai"):
                    np.testing.assert_array_equal(g[k], p[k], err_msg=k)
            sd, si = W.observed_shortwave(sw[0, h, :n].astype(np.float64), use[0, :n].astype(bool),
                                          p["coszen"], int(jday), p["solad"], p["solai"])
            np.testing.assert_allclose(g["solad"], sd, rtol=1e-4, atol=1e-3, err_msg=f"{di} {h} solad")
            np.testing.assert_allclose(g["solai"], si, rtol=1e-4, atol=1e-3, err_msg=f"{di} {h} solai")
