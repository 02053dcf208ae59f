"""Monthly wetland methane: the oracle (oracle/month.py) against the
reference's own functions (tests/golden/methane_month.npz, made by
tests/golden/make_golden.py from bgc/methane.py:233-496), CPU; the device
month kernels against the oracle, GPU.

Tolerance: relative 1e-12 (float64 throughout)."""
import os
import types

import numpy as np
import pytest

from oracle import month as OM

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden", "methane_month.npz")
MP_FIELDS = ("sat_crit", "z_max", "r_ch4", "q10p", "t_ref", "z_wt_max", "z_wt_ref", "z_tau", "tau_oxid")


def load():
    z = np.load(GOLD)
    return {k: z[k] for k in z.files}


def mparams(z, tag):
    return types.SimpleNamespace(**{f: float(z[f"param.{tag}.{f}"]) for f in MP_FIELDS})


def close(a, b, rtol=1e-12, atol=1e-300):
    np.testing.assert_allclose(np.asarray(a, np.float64), b, rtol=rtol, atol=atol)


@pytest.mark.parametrize("tag", ["default", "custom"])
def test_oracle_matches_reference_monthly_methane(tag):
    z = load()
    P = mparams(z, tag)
    t, w, i, h = z["in.tsoi"], z["in.wsoi"], z["in.wisoi"], z["in.hsoi"]
    nd = int(z["in.ndays"])
    close(OM.wetland_water_table(w, i, h, P), z[f"{tag}.zwt"])
    close(OM.methane_flux(z["in.f_inund"], z["in.rh"], t, w, i, h, P), z[f"{tag}.flux"])
    close(OM.methane_flux(z["in.f_inund"], z["in.rh"], t, w, i, h, P, z["in.zwt_obs"]), z[f"{tag}.flux_obs"])
    m0 = dict(flux=np.zeros_like(z["in.annual0"]), annual=z["in.annual0"], zwt=np.zeros_like(z["in.annual0"]))
    for obs in (False, True):
        zo = z["in.zwt_obs"] if obs else None
        sfx = "_obs" if obs else ""
        ms = OM.methane_step(m0, z["in.f_inund"], z["in.rh"], t, w, i, h, nd, P, zo)
        mm = OM.methane_step_from_mean(m0, z["in.flux_month"], w, i, h, nd, P, zo)
        sc = OM.scale_month(mm, z["in.annual0"], z["in.scale"])
        for name, st in (("step", ms), ("mean", mm), ("scaled", sc)):
            for leaf in ("flux", "annual", "zwt"):
                close(st[leaf], z[f"{tag}.{name}{sfx}.{leaf}"])
        close(OM.ch4_carbon_from_rh(sc["annual"], z["in.annual0"], z["in.rh_now"], z["in.rh_before"]),
              z[f"{tag}.take{sfx}"])
    close(OM.reset_annual(m0)["annual"], z[f"{tag}.reset.annual"])


def test_observed_water_table_rules():
    """NaN keeps the model's depth; observed depths are clipped to [0, z_max]."""
    z = load()
    P = mparams(z, "default")
    w, i, h, zo = z["in.wsoi"], z["in.wisoi"], z["in.hsoi"], z["in.zwt_obs"]
    model = OM.wetland_water_table(w, i, h, P)
    got = OM.wetland_water_table(w, i, h, P, zo)
    nan = np.isnan(zo)
    assert nan.any() and (zo[~nan] < 0).any() and (zo[~nan] > P.z_max).any()
    np.testing.assert_array_equal(got[nan], model[nan])
    np.testing.assert_array_equal(got[~nan], np.clip(zo[~nan], 0.0, P.z_max))


CKPT = os.path.join(HERE, "golden", "restart_16cells.npz")


def _device_month_setup(tag, dtype):
    import torch
    from ibis_b200 import dropin, restart
    from ibis_b200.columns import Columns
    from ibis_b200.daily import DayLoop
    from ibis_b200.params import FLAG_CH4, DayParams
    z = load()
    n = 16
    leaves, _, _ = restart.load(CKPT)
    tree = restart.as_tree(leaves)
    prog = dropin._leaf_dict(tree, "PROG", n)
    stat = dropin._leaf_dict(tree, "STAT", n)
    prog.update(tsoi=z["in.tsoi"], wsoi=z["in.wsoi"], wisoi=z["in.wisoi"])
    stat.update(f_inund=z["in.f_inund"], tco2mic=z["in.rh"] / OM.RH_CONV, zwt_obs=z["in.zwt_obs"])
    P = restart.params_from_leaves(leaves)
    np.testing.assert_array_equal(np.asarray(P.hsoi), z["in.hsoi"])
    for f in MP_FIELDS:
        setattr(P, f, float(z[f"param.{tag}.{f}"]))
    P.flags |= FLAG_CH4
    cols = Columns.from_host(prog, stat, dtype=dtype, acc=True)
    loop = DayLoop(cols, P, DayParams(), {})
    return z, n, prog, stat, P, cols, loop, torch


@pytest.mark.gpu
@pytest.mark.parametrize("tag", ["default", "custom"])
@pytest.mark.parametrize("obs", [False, True])
def test_device_month_kernels_match_oracle(cuda_lib, tag, obs):
    """ibis_month_begin_f64 / ibis_month_end_f64 against oracle.month.month_end,
    every combination of flux source, scaling and carbon partition: 1e-12."""
    from ibis_b200 import synth
    from ibis_b200.params import FLAG_ZWT_OBS
    z, n, prog, stat, P, cols, loop, torch = _device_month_setup(tag, __import__("torch").float64)
    if obs:
        loop.params.flags |= FLAG_ZWT_OBS
    zo = z["in.zwt_obs"] if obs else None
    nd = int(z["in.ndays"])
    pad = lambda a: torch.from_numpy(np.pad(np.asarray(a, np.float64), (0, cols.ld - n))).cuda()
    stat_o = {**stat}
    for from_mean in (False, True):
        for scaled in (False, True):
            for partition in (False, True):
                wet0 = dict(flux=np.zeros(n), annual=z["in.annual0"].copy(), zwt=np.zeros(n), rh0=np.zeros(n),
                            ch4c=np.full(n, 1e-4))
                loop.set_wet(wet0)
                loop.set_dayst({"ayco2mic": z["in.rh_before"]})
                cols.set_acc({"ch4": np.full(n, 7.0)})                 # cleared by the month's start
                loop.begin_month()
                cols.set_acc({"ch4": z["in.flux_month"] * nd})      # the month's hours
                loop.set_dayst({"ayco2mic": z["in.rh_now"]})
                loop.end_month(nd, from_mean=from_mean, scale=pad(z["in.scale"]) if scaled else None,
                               partition=partition)
                torch.cuda.synchronize()
                want, ay, take = OM.month_end(wet0, prog, stat_o, z["in.flux_month"] * nd, z["in.rh_now"],
                                              z["in.rh_before"], nd, z["in.hsoi"], P, from_mean=from_mean,
                                              scale=z["in.scale"] if scaled else None, partition=partition,
                                              zwt_obs=zo)
                got = loop.wet_host()
                case = (from_mean, scaled, partition)
                for k in ("flux", "annual", "zwt"):
                    close(got[k], want[k])
                np.testing.assert_allclose(got["rh0"], z["in.rh_before"], rtol=0, atol=0, err_msg=str(case))
                close(got["ch4c"], 1e-4 + take)
                close(synth.from_planes("DAYST", loop.dayst.cpu().numpy(), n)["ayco2mic"], ay)


@pytest.mark.gpu
def test_device_month_new_year_resets_annual(cuda_lib):
    z, n, prog, stat, P, cols, loop, torch = _device_month_setup("default", __import__("torch").float64)
    loop.set_wet(dict(annual=np.full(n, 3.0), ch4c=np.full(n, 2.0), flux=np.full(n, 1.0)))
    loop.begin_month(new_year=True)
    torch.cuda.synchronize()
    w = loop.wet_host()
    assert np.all(w["annual"] == 0) and np.all(w["ch4c"] == 0) and np.all(w["flux"] == 1.0)


@pytest.mark.gpu
def test_device_hourly_ch4_with_observed_water_table(cuda_lib):
    """The hourly step's CH4 accumulator with an observed water table
    (FLAG_ZWT_OBS; NaN entries keep the model's) equals the oracle step's,
    float64, over six hours of the day_mixed case: 1e-9."""
    import torch
    import oracle
    from goldens import Case
    from ibis_b200.columns import Columns
    from ibis_b200.params import FLAG_ACC, FLAG_CH4, FLAG_ZWT_OBS
    c = Case("day_mixed")
    n = c.ncell
    rng = np.random.Generator(np.random.PCG64(3))
    stat = dict(c.stat)
    zo = rng.uniform(-0.2, 4.5, n)
    zo[rng.uniform(size=n) < 0.4] = np.nan
    stat["zwt_obs"] = zo
    stat["f_inund"] = rng.uniform(0.0, 1.0, n)
    P = c.params.copy()
    P.flags = (P.flags | FLAG_ACC | FLAG_CH4 | FLAG_ZWT_OBS) & ~(1 << 8)
    nh = min(6, c.nhour)
    cols = Columns.from_host(c.prog, stat, dtype=torch.float64, acc=True)
    cols.run(cols.forcing(c.forc, 0, nh), P)
    torch.cuda.synchronize()
    prog, acc = dict(c.prog), oracle.new_acc(n)
    with np.errstate(all="ignore"):
        for h in range(nh):
            prog, _, acc = oracle.step(prog, stat, c.forcing_at(h), P, acc)
    got = cols.acc_host()["ch4"]
    np.testing.assert_allclose(got, acc["ch4"], rtol=1e-9, atol=1e-300)
    # and the observed depth matters: without the flag the sums differ
    P2 = P.copy()
    P2.flags &= ~FLAG_ZWT_OBS
    prog, acc2 = dict(c.prog), oracle.new_acc(n)
    with np.errstate(all="ignore"):
        for h in range(nh):
            prog, _, acc2 = oracle.step(prog, stat, c.forcing_at(h), P2, acc2)
    assert np.any(np.abs(acc2["ch4"] - acc["ch4"]) > 1e-6 * np.abs(acc["ch4"]).max())


# ---------------------------------------------------------------------------
# per-cell methane parameters by biome (biome_methane_params, methane.py:521-563)
# ---------------------------------------------------------------------------
BANDS_GOLD = os.path.join(HERE, "golden", "methane_bands.npz")
BAND_TAGS = ("biome", "biome_koppen", "release")


def band_params(z, tag):
    """StepParams with the tag's per-band tables (FLAG_CH4_BANDS) and the ch4_band plane,
    built by ibis_b200.params from the tag's base values, Koeppen types and bands."""
    import json
    from ibis_b200.params import StepParams, methane_band_index, with_methane_bands
    base, koppen, with_bands = (str(x) for x in z[f"meta.{tag}"])
    P = StepParams()
    for f in MP_FIELDS:
        setattr(P, f, float(z[f"base.{base}.{f}"]))
    bands = json.loads(str(z["in.bands"])) if with_bands == "1" else None
    band = methane_band_index(z["in.lat"], z["in.band_index"] if koppen == "1" else None)
    return with_methane_bands(P, bands), band


@pytest.mark.parametrize("tag", BAND_TAGS)
def test_band_tables_give_the_reference_per_cell_parameters(tag):
    from oracle.column import methane_params
    z = dict(np.load(BANDS_GOLD))
    P, band = band_params(z, tag)
    per_cell = methane_params(P, {"ch4_band": band})
    for f in MP_FIELDS:
        np.testing.assert_array_equal(np.broadcast_to(getattr(per_cell, f), band.shape), z[f"param.{tag}.{f}"],
                                      err_msg=f)


@pytest.mark.parametrize("tag", BAND_TAGS)
def test_oracle_matches_reference_per_band_methane(tag):
    from oracle.column import methane_params
    z = dict(np.load(BANDS_GOLD))
    P, band = band_params(z, tag)
    m = methane_params(P, {"ch4_band": band})
    t, w, i, h = z["in.tsoi"], z["in.wsoi"], z["in.wisoi"], z["in.hsoi"]
    close(OM.wetland_water_table(w, i, h, m), z[f"{tag}.zwt"])
    close(OM.methane_flux(z["in.f_inund"], z["in.rh"], t, w, i, h, m), z[f"{tag}.flux"])
    close(OM.methane_flux(z["in.f_inund"], z["in.rh"], t, w, i, h, m, z["in.zwt_obs"]), z[f"{tag}.flux_obs"])
    m0 = dict(flux=np.zeros_like(z["in.annual0"]), annual=z["in.annual0"], zwt=np.zeros_like(z["in.annual0"]))
    ms = OM.methane_step(m0, z["in.f_inund"], z["in.rh"], t, w, i, h, int(z["in.ndays"]), m)
    for leaf in ("flux", "annual", "zwt"):
        close(ms[leaf], z[f"{tag}.step.{leaf}"])


def test_band_tables_refuse_what_the_reference_cannot_run():
    from ibis_b200.params import StepParams, with_methane_bands
    with pytest.raises(KeyError):
        with_methane_bands(StepParams(), {"boreal": {"r_ch5": 0.1}})
    with pytest.raises(ValueError):
        with_methane_bands(StepParams(), {"boreal": {"z_wt_ref": 0.3}})


@pytest.mark.gpu
@pytest.mark.parametrize("tag", BAND_TAGS)
def test_device_month_per_band_matches_reference(cuda_lib, tag):
    """ibis_month_end_f64 from the end-of-month state with per-band parameters
    (FLAG_CH4_BANDS, the STAT ch4_band plane) against the reference's own
    methane_step under biome_methane_params: 1e-12."""
    import torch
    from ibis_b200 import dropin, restart
    from ibis_b200.columns import Columns
    from ibis_b200.daily import DayLoop
    from ibis_b200.params import DayParams
    z = dict(np.load(BANDS_GOLD))
    n = 16
    Pb, band = band_params(z, tag)
    leaves, _, _ = restart.load(CKPT)
    tree = restart.as_tree(leaves)
    prog = dropin._leaf_dict(tree, "PROG", n)
    stat = dropin._leaf_dict(tree, "STAT", n)
    prog.update(tsoi=z["in.tsoi"], wsoi=z["in.wsoi"], wisoi=z["in.wisoi"])
    stat.update(f_inund=z["in.f_inund"], tco2mic=z["in.rh"] / OM.RH_CONV, ch4_band=band)
    P = restart.params_from_leaves(leaves)
    np.testing.assert_array_equal(np.asarray(P.hsoi), z["in.hsoi"])
    for f in MP_FIELDS:
        setattr(P, f, getattr(Pb, f))
        setattr(P, "ch4b_" + f, getattr(Pb, "ch4b_" + f))
    P.flags |= Pb.flags
    cols = Columns.from_host(prog, stat, dtype=torch.float64, acc=True)
    loop = DayLoop(cols, P, DayParams(), {})
    loop.set_wet(dict(flux=np.zeros(n), annual=z["in.annual0"].copy(), zwt=np.zeros(n)))
    loop.begin_month()
    loop.end_month(int(z["in.ndays"]), from_mean=False)
    torch.cuda.synchronize()
    got = loop.wet_host()
    for leaf in ("flux", "annual", "zwt"):
        close(got[leaf], z[f"{tag}.step.{leaf}"])


@pytest.mark.gpu
def test_device_hourly_ch4_per_band(cuda_lib):
    """The hourly step's CH4 accumulator with per-band parameters (the release
    file's methane_bands over Koeppen and latitude bands) equals the oracle
    step's, float64 over six hours of the day_mixed case (1e-9) and float32
    within 1e-5 of the largest sum; and the bands matter."""
    import json
    import torch
    import oracle
    from goldens import Case
    from ibis_b200.columns import Columns
    from ibis_b200.params import FLAG_ACC, FLAG_CH4, FLAG_CH4_BANDS, FLAG_KAHAN, methane_band_index, with_methane_bands
    z = dict(np.load(BANDS_GOLD))
    c = Case("day_mixed")
    n = c.ncell
    rng = np.random.Generator(np.random.PCG64(9))
    stat = dict(c.stat)
    stat["f_inund"] = rng.uniform(0.0, 1.0, n)
    stat["ch4_band"] = methane_band_index(rng.uniform(-60.0, 80.0, n), rng.integers(-1, 3, n))
    P = with_methane_bands(c.params, json.loads(str(z["in.bands"])))
    P.flags = (P.flags | FLAG_ACC | FLAG_CH4) & ~FLAG_KAHAN
    nh = min(6, c.nhour)
    prog, acc = dict(c.prog), oracle.new_acc(n)
    with np.errstate(all="ignore"):
        for h in range(nh):
            prog, _, acc = oracle.step(prog, stat, c.forcing_at(h), P, acc)
    for dtype, rtol in ((torch.float64, 1e-9), (torch.float32, None)):
        Pd = P.copy()
        if dtype == torch.float32:
            Pd.flags |= FLAG_KAHAN
        cols = Columns.from_host(c.prog, stat, dtype=dtype, acc=True)
        cols.run(cols.forcing(c.forc, 0, nh), Pd)
        torch.cuda.synchronize()
        got = cols.acc_host()["ch4"]
        if rtol:
            np.testing.assert_allclose(got, acc["ch4"], rtol=rtol, atol=1e-300)
        else:
            assert np.max(np.abs(got - acc["ch4"])) <= 1e-5 * np.abs(acc["ch4"]).max()
    P2 = P.copy()
    P2.flags &= ~FLAG_CH4_BANDS
    prog, acc2 = dict(c.prog), oracle.new_acc(n)
    with np.errstate(all="ignore"):
        for h in range(nh):
            prog, _, acc2 = oracle.step(prog, stat, c.forcing_at(h), P2, acc2)
    assert np.any(np.abs(acc2["ch4"] - acc["ch4"]) > 1e-3 * np.abs(acc["ch4"]).max())


@pytest.mark.parametrize("tag", BAND_TAGS)
def test_dropin_maps_per_cell_methane_parameters(tag):
    """The drop-in reads a reference MethaneParams with per-cell fields (as
    biome_methane_params returns it) into band tables and a band plane that
    give every cell its own values back."""
    import types as _t
    from ibis_b200 import dropin
    from ibis_b200.params import StepParams, FLAG_CH4_BANDS
    from oracle.column import methane_params
    z = dict(np.load(BANDS_GOLD))
    mp = _t.SimpleNamespace(**{f: z[f"param.{tag}.{f}"] for f in MP_FIELDS})
    P, stat = StepParams(), {}
    dropin.apply_methane(P, stat, mp, 16)
    assert P.flags & FLAG_CH4_BANDS
    got = methane_params(P, stat)
    for f in MP_FIELDS:
        np.testing.assert_array_equal(np.broadcast_to(getattr(got, f), (16,)), z[f"param.{tag}.{f}"], err_msg=f)
    scalar = _t.SimpleNamespace(**{f: float(z[f"base.default.{f}"]) for f in MP_FIELDS})
    dropin.apply_methane(P, stat, scalar, 16)
    assert not P.flags & FLAG_CH4_BANDS and P.r_ch4 == float(z["base.default.r_ch4"])
