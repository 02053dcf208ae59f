"""One hourly step of the IBIS column model in float64 -- TEST INFRASTRUCTURE ONLY.

``step(prog, stat, forc, P)`` restates ``timestep_body``
(``python-port/ibis/timestepping/loops.py:234-1284``) followed by the per-step
accumulators and wetland CH4 of ``_run_day_inner._step_body``
(``python-port/ibis/timestepping/loops_gswp3.py:161-318``).

Inputs are dicts of float64 arrays keyed by the field names of
``ibis_b200.layout`` (layer fields as (ncell, k)); ``P`` is an
``ibis_b200.params.StepParams``.  Returns ``(prog_new, diag, acc_new)``.
"""
from __future__ import annotations

import numpy as np

from .physics import clip, cube, setsoi, fwetcal, cascade, radiation, evap_intercepted, FLAG_GPP_CAPACITY
from .canopy import aero_geometry, transfer, weight_veg, weight_snow, stomata, turvap
from .column import (snow_block, water_bounds, soil_water, soil_heat, phase_change, puddle_phase,
                     fire_counters, methane, methane_params)

FLAG_BEDROCK = 1 << 0
FLAG_SUNSHADE_U = 1 << 2
FLAG_SUNSHADE_L = 1 << 3
FLAG_ACC = 1 << 4
FLAG_CH4 = 1 << 5
FLAG_SOIL_MEANS = 1 << 6
FLAG_ZWT_OBS = 1 << 9
FLAG_ETPARTS = 1 << 10
FLAG_NEEPARTS = 1 << 11

ACC_FIELDS = {"adrain": 1, "adsnow": 1, "adaet": 1, "a10ancub": 1, "a10ancls": 1, "a10ancl3": 1,
              "a10ancl4": 1, "aynpp": 12, "aynpptot": 1, "aygpptot": 1, "aytrunof": 1, "aytdrain": 1,
              "ch4": 1, "tsoi_mean": 6, "wsoi_mean": 6, "wisoi_mean": 6, "tg_mean": 1, "afsena": 1,
              "stresstu_last": 1, "stresstl_last": 1, "et_trans": 1, "et_interc": 1, "et_soilev": 1,
              "et_snowsub": 1, "nee_night": 1, "nee_day": 1}


def new_acc(n):
    return {k: (np.zeros(n) if c == 1 else np.zeros((n, c))) for k, c in ACC_FIELDS.items()}


def step(prog, S, F, P, acc=None):
    eps = P.epsilon
    dt = P.dtime
    n = prog["tg"].shape[0]
    hsoi = np.asarray(P.hsoi, dtype=np.float64)
    froot = np.asarray(P.froot, dtype=np.float64).reshape(6, 2)
    fi = prog["fi"]
    lai, sai, fu, fl = S["lai"], S["sai"], S["fu"], S["fl"]
    csoi = np.where(S["csoi"] > 0.0, S["csoi"], P.csoi_mineral_val)
    rhosoi = np.where(S["rhosoi"] > 0.0, S["rhosoi"], P.rhosoi_val)
    D = {}

    # 1-2. diagnostic soil properties and wet fractions (loops.py:318-338)
    consoi, qglif, hvasug, hvasui = setsoi(S, prog, prog["tsno"][:, 0], F["ta"], P)
    wet0 = fwetcal(prog["tu"], prog["ts"], prog["tl"], prog, P)
    # 3. radiation (loops.py:343-354)
    R = radiation(prog, S, F, wet0, P)
    # 4-5. precipitation cascade and wet fractions after it (loops.py:359-389)
    casc = cascade(prog, S, F, P)
    I = {k: casc[k] for k in ("wliqu", "wliqs", "wliql", "wsnou", "wsnos", "wsnol")}
    wet = fwetcal(prog["tu"], prog["ts"], prog["tl"], I, P)

    # 6. canopy exchange (loops.py:396-611)
    A = aero_geometry(F, S, fi, P)
    znorm = 1.0 - np.exp(P.stressfac)
    awc = clip((prog["wsoi"] * (1.0 - prog["wisoi"]) - S["swilt"]) / np.maximum(S["sfield"] - S["swilt"], 1e-10), 0.0, 1.0)
    zwilt = clip((1.0 - np.exp(P.stressfac * awc)) / znorm, 0.0, 1.0)
    stressl = zwilt * froot[None, :, 0]
    stressu = zwilt * froot[None, :, 1]
    stresstl = np.sum(stressl, axis=1)
    stresstu = np.sum(stressu, axis=1)

    X = dict(fi=fi, xu=2.0 * lai[:, 1] * fu, xs=2.0 * sai[:, 1] * fu,
             xl=2.0 * (lai[:, 0] + sai[:, 0]) * fl * (1.0 - fi))
    X["cog"] = consoi[:, 0] / max(0.5 * hsoi[0], eps)
    X["coi"] = P.consno / np.maximum(0.5 * np.maximum(prog["hsno"][:, 0], P.hsnotop), eps)
    X["zirg"] = 4.0 * 0.95 * P.stef * cube(prog["tg"])
    X["ziri"] = 4.0 * 0.95 * P.stef * cube(prog["ti"])
    p0, w0, i0 = S["poros"][:, 0], prog["wsoi"][:, 0], prog["wisoi"][:, 0]
    rwp = p0 * P.rhow
    X["chgx"] = (P.ch2o * prog["wpud"] + P.cice * prog["wipud"]
                 + ((1.0 - p0) * csoi[:, 0] * rhosoi[:, 0] + rwp * (1.0 - i0) * w0 * P.ch2o + rwp * i0 * P.cice) * hsoi[0])
    X["wlgx"] = prog["wpud"] + rwp * (1.0 - i0) * w0 * hsoi[0]
    X["wigx"] = prog["wipud"] + rwp * i0 * hsoi[0]
    X.update(wpud=prog["wpud"], wipud=prog["wipud"], wisoi0=i0, wsoi0=w0, swilt0=S["swilt"][:, 0],
             suction0=S["suction"][:, 0], bex0=S["bex"][:, 0], hvasug=hvasug, hvasui=hvasui,
             tsoi0=prog["tsoi"][:, 0], tsno0=prog["tsno"][:, 0])
    X["chux"] = P.chu + P.ch2o * I["wliqu"] + P.cice * I["wsnou"]
    X["chsx"] = P.chs + P.ch2o * I["wliqs"] + P.cice * I["wsnos"]
    X["chlx"] = P.chl + P.ch2o * I["wliql"] + P.cice * I["wsnol"]

    old = dict(tu=prog["tu"], ts=prog["ts"], tl=prog["tl"], tg=prog["tg"], ti=prog["ti"])
    W = dict(tu=prog["tu"], ts=prog["ts"], tl=prog["tl"], t12=prog["t12"], t34=prog["t34"],
             q12=prog["q12"], q34=prog["q34"], tg=prog["tg"], ti=prog["ti"])
    st = {k: prog[k] for k in ("ci_upper", "gs_upper", "cs_upper", "ci_lower", "gs_lower", "cs_lower",
                               "a10scalparamu", "a10daylightu", "a10scalparaml", "a10daylightl")}
    strat = (None, None, None, None)
    wprev = [None] * 5
    cur = dict(A)
    sun_u = bool(P.flags & FLAG_SUNSHADE_U)
    sun_l = bool(P.flags & FLAG_SUNSHADE_L)
    res = None
    for it in range(3):
        first = it == 0
        T, strat, carry = transfer(cur, F, W["t12"], W["t34"], W["q12"], W["q34"], first, strat, P)
        stom = stomata(W["tu"], W["tl"], W["t12"], W["t34"], W["q12"], W["q34"], T["su"], T["sl"], F["psurf"],
                       R, st, wet["fwetu"], wet["fwetl"], S, stresstu, stresstl, P, sun_u, sun_l)
        for k in st:
            st[k] = stom[k]
        wts = [weight_veg(W["tu"], X["chux"], I["wliqu"], I["wsnou"], wprev[0], first, P),
               weight_veg(W["ts"], X["chsx"], I["wliqs"], I["wsnos"], wprev[1], first, P),
               weight_veg(W["tl"], X["chlx"], I["wliql"], I["wsnol"], wprev[2], first, P),
               weight_veg(W["tg"], X["chgx"], X["wlgx"], X["wigx"], wprev[3], first, P),
               weight_snow(W["ti"], old["ti"], wprev[4], first, P)]
        res = turvap(W, old, T, A, X, wts, I, F, S, wet, stom, R, casc, P)
        for k in W:
            W[k] = res[k]
        cur.update(carry)
        wprev = wts
    ti = np.minimum(res["ti"], P.tmelt)
    tg = W["tg"]

    # 7-8. evaporation of intercepted water, bare-story reset (loops.py:616-640)
    tu, wliqu, wsnou = evap_intercepted(W["tu"], I["wliqu"], I["wsnou"], wet["rliqu"], res["fvapuw"], P.chu, P)
    ts, wliqs, wsnos = evap_intercepted(W["ts"], I["wliqs"], I["wsnos"], wet["rliqs"], res["fvaps"], P.chs, P)
    tl, wliql, wsnol = evap_intercepted(W["tl"], I["wliql"], I["wsnol"], wet["rliql"], res["fvaplw"], P.chl, P)
    tav = (1.0 - fi) * tg + fi * ti
    nou = (lai[:, 1] == 0.0) | (fu == 0.0)
    nos = (sai[:, 1] == 0.0) | (fu == 0.0)
    nol = (2.0 * (lai[:, 0] + sai[:, 0]) == 0.0) | (fl * (1.0 - fi) == 0.0)
    tu = np.where(nou, tav, tu)
    wliqu, wsnou = np.where(nou, 0.0, wliqu), np.where(nou, 0.0, wsnou)
    ts = np.where(nos, tav, ts)
    wliqs, wsnos = np.where(nos, 0.0, wliqs), np.where(nos, 0.0, wsnos)
    tl = np.where(nol, tav, tl)
    wliql, wsnol = np.where(nol, 0.0, wliql), np.where(nol, 0.0, wsnol)

    # 9. surface fluxes into soil and snow (loops.py:665-674)
    fm = P.flux_max
    heatg = R["solg"] + clip(res["firg"], -fm, fm) - clip(res["fseng"], -fm, fm) - hvasug * res["fvapg"]
    heati = R["soli"] + clip(res["firi"], -fm, fm) - clip(res["fseni"], -fm, fm) - hvasui * res["fvapi"]

    # 10. snow (loops.py:676-848)
    sn = snow_block(prog, S, casc, heati, res["fvapi"], tl, wliql, wsnol, consoi[:, 0], P)
    wliql, wsnol = sn["wliql"], sn["wsnol"]
    rdt = 1.0 / dt
    heatg_avg = (1.0 - fi) * heatg + fi * sn["sflo_bot"] + sn["zheat"] * rdt
    fvapg_avg = clip((1.0 - fi) * res["fvapg"], -1.0e-3, 1.0e-3)
    raing_nf = (1.0 - fi) * casc["raing"]
    smr = sn["smelt"] * rdt
    rsum = raing_nf + smr
    zero = rsum < eps
    raing_avg = np.where(zero, 0.0, rsum)
    traing_avg = np.where(zero, 0.0, (raing_nf * casc["traing"] + smr * P.tmelt) / np.maximum(rsum, eps))

    # 11. soil (loops.py:896-1125)
    poros = S["poros"]
    wpud, wipud = prog["wpud"], prog["wipud"]
    c0pud = np.zeros((n, 6))
    grunof = np.minimum(wpud, np.maximum(0.0, wpud + wipud - P.wpudmax)) / dt
    wpw = wpud - grunof * dt
    zfrez = clip((prog["tsoi"][:, 0] - P.tmelt + 0.5) * 2.0, 0.0, 1.0)
    zrunf = zfrez * clip((wpw + wipud) / P.wpudmax, 0.0, 1.0)
    wpw = wpw + (1.0 - zrunf) * raing_avg * dt
    grunof = grunof + zrunf * raing_avg
    evap = fvapg_avg >= 0.0
    edt = fvapg_avg * dt
    fwtop = np.where(evap, -qglif[:, 0] * fvapg_avg, 0.0)
    wpw = np.where(evap, wpw - qglif[:, 2] * edt, wpw)
    wiw = np.where(evap, wipud - qglif[:, 3] * edt, wipud)
    isub = np.where(evap, qglif[:, 1] * edt / np.maximum(P.rhow * poros[:, 0] * hsoi[0], eps), 0.0)
    i0n = np.maximum(0.0, i0 - isub)
    w0a = np.where((1.0 - i0n) > eps, w0 * (1.0 - i0) / (1.0 - i0n), w0)
    wpw = np.where(~evap, wpw - (qglif[:, 0] + qglif[:, 2]) * edt, wpw)
    wiw = np.where(~evap, wiw - (qglif[:, 1] + qglif[:, 3]) * edt, wiw)
    wpw = np.maximum(wpw, 0.0)
    wiw = np.maximum(wiw, 0.0)
    zdpud = P.rhow * dt * np.maximum(1.0 - i0n, 0.0) ** 2 * S["hydraul"][:, 0]
    fwpud = np.maximum(0.0, np.minimum(wpw, zdpud)) / dt
    c0pud[:, 0] = P.ch2o * wpw + P.cice * wiw
    wsw = prog["wsoi"].copy()
    wsw[:, 0] = np.where(evap, w0a, wsw[:, 0])
    wisw = prog["wisoi"].copy()
    wisw[:, 0] = np.where(evap, i0n, wisw[:, 0])
    pflo = np.maximum(poros * np.maximum(1.0 - wisw, eps), eps)
    gtransu = res["fvaput"] * 2.0 * lai[:, 1] * fu
    gtransl = res["fvaplt"] * 2.0 * lai[:, 0] * fl * (1.0 - fi)
    wu_ = np.where(stresstu[:, None] >= 1.0, froot[None, :, 1], stressu / np.maximum(stresstu, eps)[:, None])
    wl_ = np.where(stresstl[:, None] >= 1.0, froot[None, :, 0], stressl / np.maximum(stresstl, eps)[:, None])
    wpt = wsw.copy()
    tpt = prog["tsoi"].copy()
    for k in range(6):
        uu = gtransu * wu_[:, k]
        ul = gtransl * wl_[:, k]
        wpt[:, k] = wpt[:, k] + (-dt * (uu + ul) / (P.rhow * pflo[:, k] * hsoi[k]))
        wpt[:, k] = np.maximum(wpt[:, k], 0.0)
        cx = (c0pud[:, k] + ((1.0 - poros[:, k]) * csoi[:, k] * rhosoi[:, k]
                             + poros[:, k] * (1.0 - wisw[:, k]) * wpt[:, k] * P.ch2o * P.rhow
                             + poros[:, k] * wisw[:, k] * P.cice * P.rhow) * hsoi[k])
        tpt[:, k] = tpt[:, k] + (-dt * P.ch2o * (uu * (tu - tpt[:, k]) + ul * (tl - tpt[:, k])) / np.maximum(cx, eps))
    fhtop_soil = heatg_avg + raing_avg * P.ch2o * (traing_avg - tpt[:, 0]) - grunof * P.ch2o * np.maximum(P.tmelt - tpt[:, 0], 0.0)
    wnew, wpud_h, wflo = soil_water(wpt, wisw, poros, pflo, S, hsoi, fwtop, fwpud, wpw, P)
    c1pud = c0pud.copy()
    c1pud[:, 0] = P.ch2o * wpud_h + P.cice * wiw
    if P.flags & FLAG_BEDROCK:
        nb = 3
        z = np.zeros((n, nb))
        tt, hf = soil_heat(np.concatenate([tpt, prog["tsoi_deep"]], 1), np.concatenate([tpt, prog["tsoi_deep"]], 1),
                           np.concatenate([wpt, z], 1), np.concatenate([wnew, z], 1), np.concatenate([wisw, z], 1),
                           np.concatenate([poros, z], 1), np.concatenate([consoi, np.full((n, nb), P.consoi_bed)], 1),
                           np.concatenate([csoi, np.full((n, nb), P.csoi_bed)], 1),
                           np.concatenate([rhosoi, np.full((n, nb), P.rhosoi_bed)], 1),
                           np.concatenate([hsoi, np.asarray(P.hsoi_bed)]), np.concatenate([c0pud, z], 1),
                           np.concatenate([c1pud, z], 1), fhtop_soil, np.concatenate([wflo, z], 1), 6, P)
        theat, hflo, tdeep = tt[:, :6], hf[:, :7], tt[:, 6:]
    else:
        theat, hflo = soil_heat(tpt, tpt, wpt, wnew, wisw, poros, consoi, csoi, rhosoi, hsoi, c0pud, c1pud,
                                fhtop_soil, wflo, 6, P)
        tdeep = prog.get("tsoi_deep")
    wpre, ipre, gadj1 = water_bounds(wnew, wisw, poros, hsoi, P)
    tft, wft, ift, pflo_ft = phase_change(theat, wpre, ipre, poros, csoi, rhosoi, hsoi, c1pud, P)
    t0, wpud_n, wipud_n = puddle_phase(tft[:, 0], wpud_h, wiw, poros[:, 0], wft[:, 0], ift[:, 0],
                                       csoi[:, 0], rhosoi[:, 0], hsoi[0], P)
    tft[:, 0] = t0
    wadj, iadj, gadj2 = water_bounds(wft, ift, poros, hsoi, P)

    # 12. surface temperature bound (loops.py:1143-1151)
    lo_, hi_ = F["ta"] - P.t_max_dev, F["ta"] + P.t_max_dev
    tu, ts, tl, tg = clip(tu, lo_, hi_), clip(ts, lo_, hi_), clip(tl, lo_, hi_), clip(tg, lo_, hi_)

    new = dict(tsoi=tft, wsoi=wadj, wisoi=iadj, tg=tg, wpud=wpud_n, wipud=wipud_n,
               tsoi_deep=tdeep if tdeep is not None else np.zeros((n, 3)),
               fi=sn["fi"], tsno=sn["tsno"], hsno=sn["hsno"], ti=ti, tlsub=sn["tlsub"],
               tu=tu, ts=ts, tl=tl, t12=W["t12"], t34=W["t34"], q12=W["q12"], q34=W["q34"],
               wliqu=wliqu, wliqs=wliqs, wliql=wliql, wsnou=wsnou, wsnos=wsnos, wsnol=wsnol)
    for k in st:
        new[k] = st[k]
    new.update(fire_counters(prog, wadj[:, 0], iadj[:, 0], S["swilt"][:, 0], F, P))

    # diagnostics (loops.py:1158-1241)
    D.update({k: stom[k] for k in ("an_upper", "ag_upper", "an_lower", "ag_lower")})
    D.update({k: wet[k] for k in ("fwetu", "fwets", "fwetl", "rliqu", "rliqs", "rliql")})
    D.update({k: R[k] for k in ("solu", "sols", "soll", "solg", "soli", "firu", "firs", "firl",
                                "asurd", "asuri", "topparu", "topparl", "scalcoefu", "scalcoefl")})
    D.update({k: res[k] for k in ("firg", "firi", "firb", "fsena", "fsenu", "fsens", "fsenl", "fseng", "fseni",
                                  "fvapg", "fvapi", "ginvap", "gsuvap", "gtrans")})
    D.update(raing=casc["raing"], snowg=casc["snowg"], rhoa=A["rhoa"], consoi=consoi, hflo=hflo, heatg=heatg_avg,
             hvasug=hvasug, qglif=qglif, stresstu=stresstu, stresstl=stresstl, stressu=stressu, stressl=stressl,
             porosflo=pflo_ft, heati=heati, hvasui=hvasui, gtransu=gtransu, gtransl=gtransl, grunof=grunof,
             gdrain=wflo[:, -1], gadjust=gadj1 + gadj2, wtot=np.zeros(n), raing_avg=raing_avg,
             traing_avg=traing_avg, fhtop_soil=fhtop_soil, rainl=casc["rainl"], snowl=casc["snowl"],
             trainl=casc["trainl"], tsnowl=casc["tsnowl"], sflo_bot=sn["sflo_bot"], fhtop_snow=sn["fhtop_snow"])

    acc_new = None
    if acc is not None and (P.flags & (FLAG_ACC | FLAG_CH4 | FLAG_SOIL_MEANS)):
        acc_new = {k: v.copy() for k, v in acc.items()}
        if P.flags & FLAG_ACC:
            accumulate(acc_new, new, D, S, F, P)
        w = np.float64(np.float32(dt / 86400.0))
        if P.flags & FLAG_CH4:
            rh = S["tco2mic"] * np.float64(np.float32(12.0e-3 * 86400.0))
            zo = S["zwt_obs"] if P.flags & FLAG_ZWT_OBS else None
            acc_new["ch4"] = acc_new["ch4"] + methane(S["f_inund"], rh, new["tsoi"], new["wsoi"], new["wisoi"], hsoi,
                                                      methane_params(P, S), zo) * w
        if P.flags & FLAG_SOIL_MEANS:
            acc_new["tsoi_mean"] = acc_new["tsoi_mean"] + new["tsoi"] * w
            acc_new["wsoi_mean"] = acc_new["wsoi_mean"] + new["wsoi"] * w
            acc_new["wisoi_mean"] = acc_new["wisoi_mean"] + new["wisoi"] * w
            acc_new["tg_mean"] = acc_new["tg_mean"] + new["tg"] * w
    return new, D, acc_new


def respiration_rates(P):
    """Per-PFT maintenance respiration rates and the growth-respiration keep factor
    (1 - rgrowth) as the reference forms them: the tables are cast to float32 and the
    arithmetic on them is float32 (loops_gswp3.py:185-190)."""
    f32 = np.float32
    per_s = f32(P.ndaypy * 86400.0)
    mol = f32(1000.0 / 12.0)
    rwood = (np.asarray(P.rwood).astype(f32) / per_s * mol).astype(np.float64)
    rroot = (np.asarray(P.rroot).astype(f32) / per_s * mol).astype(np.float64)
    keep = (f32(1.0) - np.asarray(P.rgrowth).astype(f32)).astype(np.float64)
    return rwood, rroot, keep


def capacity_shares(frac, vp, idx, eps=1e-12):
    """capacity_shares (stomata.py:566-577): a big leaf's GPP shares by leaf area x vmax,
    re-normalised to the leaf-area sum; the leaf-area shares where there is no capacity."""
    ix = list(idx)
    f = frac[:, ix]
    w = f * np.asarray(vp)[ix][None, :]
    tw = np.sum(w, axis=1, keepdims=True)
    tf = np.sum(f, axis=1, keepdims=True)
    return np.where(tw > eps, w / np.maximum(tw, eps) * tf, f)


def gpp_shares(frac, P):
    """Per-PFT shares of the big leaves' GPP in the NPP sums: the leaf-area fractions
    (F77), or with gpp_split_by_capacity the capacity shares (loops_gswp3.py:197-205)."""
    if not P.flags & FLAG_GPP_CAPACITY:
        return frac
    share = frac.copy()
    for idx in ((0, 1, 2, 4, 6), (3, 5, 7), (8, 9)):
        share[:, list(idx)] = capacity_shares(frac, P.vmax_pft, idx)
    return share


def accumulate(acc, new, D, S, F, P):
    """Day/annual accumulators of _step_body (loops_gswp3.py:161-302), with the F77 or
    the capacity split of each big leaf's GPP among its PFTs."""
    dt = P.dtime
    froot = np.asarray(P.froot).reshape(6, 2)
    an_ub, an_uc = D["an_upper"][:, 0], D["an_upper"][:, 1]
    an_ls, an_l3, an_l4 = D["an_lower"][:, 0], D["an_lower"][:, 1], D["an_lower"][:, 2]
    lai_u, lai_l = S["lai"][:, 1], S["lai"][:, 0]
    fu, fl, frac = S["fu"], S["fl"], S["frac"]
    smask = 1.0 - new["fi"]
    rwood, rroot, keep = respiration_rates(P)
    root_t = np.zeros_like(new["ts"])
    for k in range(6):
        root_t = root_t + new["tsoi"][:, k] * 0.5 * (froot[k, 0] + froot[k, 1])
    funca = np.exp(3500.0 * (1.0 / 288.16 - 1.0 / np.maximum(new["ts"], 200.0)))
    funcb = np.exp(3500.0 * (1.0 / 288.16 - 1.0 / np.maximum(root_t, 200.0)))
    cf = 12.0e-3 * dt
    yn_old = acc["aynpp"]
    yn = yn_old.copy()
    cbw, cbr, sap = S["cbiow"], S["cbior"], S["sapfrac"]
    share = gpp_shares(frac, P)
    for j in (0, 1, 2, 4, 6):
        g = an_ub * share[:, j] * lai_u * fu
        r = rwood[j] * cbw[:, j] * sap * funca + rroot[j] * cbr[:, j] * funcb
        yn[:, j] = yn[:, j] + keep[j] * (g - r) * cf
    for j in (3, 5, 7):
        g = an_uc * share[:, j] * lai_u * fu
        r = rwood[j] * cbw[:, j] * sap * funca + rroot[j] * cbr[:, j] * funcb
        yn[:, j] = yn[:, j] + keep[j] * (g - r) * cf
    for j in (8, 9):
        g = an_ls * share[:, j] * lai_l * fl * smask
        r = rwood[j] * cbw[:, j] * funca + rroot[j] * cbr[:, j] * funcb
        yn[:, j] = yn[:, j] + keep[j] * (g - r) * cf
    g = an_l4 * frac[:, 10] * lai_l * fl * smask
    yn[:, 10] = yn[:, 10] + keep[10] * (g - rroot[10] * cbr[:, 10] * funcb) * cf
    g = an_l3 * frac[:, 11] * lai_l * fl * smask
    yn[:, 11] = yn[:, 11] + keep[11] * (g - rroot[11] * cbr[:, 11] * funcb) * cf
    npp = np.sum(yn - yn_old, axis=1)
    ag_ub, ag_uc = D["ag_upper"][:, 0], D["ag_upper"][:, 1]
    ag_ls, ag_l3, ag_l4 = D["ag_lower"][:, 0], D["ag_lower"][:, 1], D["ag_lower"][:, 2]
    gu = (ag_ub * np.sum(frac[:, [0, 1, 2, 4, 6]], axis=1) + ag_uc * np.sum(frac[:, [3, 5, 7]], axis=1)) * lai_u * fu
    gl = (ag_ls * np.sum(frac[:, 8:10], axis=1) + ag_l4 * frac[:, 10] + ag_l3 * frac[:, 11]) * lai_l * fl * smask
    acc["adrain"] = acc["adrain"] + F["raina"] * dt
    acc["adsnow"] = acc["adsnow"] + F["snowa"] * dt
    acc["adaet"] = acc["adaet"] + (D["ginvap"] + D["gsuvap"] + D["gtrans"]) * dt
    acc["a10ancub"] = acc["a10ancub"] + an_ub * dt
    acc["a10ancls"] = acc["a10ancls"] + an_ls * dt
    acc["a10ancl3"] = acc["a10ancl3"] + an_l3 * dt
    acc["a10ancl4"] = acc["a10ancl4"] + an_l4 * dt
    acc["aynpp"] = yn
    acc["aynpptot"] = acc["aynpptot"] + npp
    acc["aygpptot"] = acc["aygpptot"] + (gu + gl) * cf
    acc["aytrunof"] = acc["aytrunof"] + D["grunof"] * dt
    acc["aytdrain"] = acc["aytdrain"] + D["gdrain"] * dt
    # canopy-top sensible heat of turvap (canopy_exchange.py:759), summed like
    # the other fluxes; the reference's day loop does not keep this sum
    acc["afsena"] = acc["afsena"] + D["fsena"] * dt
    acc["stresstu_last"] = D["stresstu"].copy()
    acc["stresstl_last"] = D["stresstl"].copy()
    if P.flags & FLAG_ETPARTS:                      # loops_gswp3.py:263-272
        snowsub = D["fvapi"] * new["fi"] * dt
        acc["et_trans"] = acc["et_trans"] + D["gtrans"] * dt
        acc["et_interc"] = acc["et_interc"] + D["ginvap"] * dt
        acc["et_soilev"] = acc["et_soilev"] + D["gsuvap"] * dt - snowsub
        acc["et_snowsub"] = acc["et_snowsub"] + snowsub
    if P.flags & FLAG_NEEPARTS:                     # loops_gswp3.py:274-281
        nee = S["tco2mic"] * cf - npp
        night = F["coszen"] <= 0.0
        acc["nee_night"] = acc["nee_night"] + np.where(night, nee, 0.0)
        acc["nee_day"] = acc["nee_day"] + np.where(night, 0.0, nee)


def run_steps(prog, S, forcings, P, acc=None):
    """Run len(forcings) hourly steps; returns the final (prog, diag, acc)."""
    D = None
    for F in forcings:
        prog, D, acc = step(prog, S, F, P, acc)
    return prog, D, acc
