"""Float64 restatement of the reference's daily cadence (test infrastructure).

The checker of the device daily kernels (ibis_b200/csrc/ibis_daily.cuh).  One
day of the reference's GSWP3 day loop (``_run_month_scan._day_body``,
python-port/ibis/timestepping/loops_gswp3.py:382-608) around its 24 hourly
steps, with crop and IBIS 3.0 slot types off (their defaults) and one soil-BGC
call per day:

* :func:`day_begin` -- capture the 10-day means, zero the daily sums
  (loops_gswp3.py:402-415), advance the seasonal states when the state
  carries them (loops_gswp3.py:418-437), and ``pheno``
  (physics/phenology.py:89-287);
* :func:`day_end` -- 10-day means and annual sums (loops_gswp3.py:466-492),
  the decomposition factors (loops_gswp3.py:494-562), ``soilbgc``
  (physics/biogeochem.py:23-243), the heterotrophic-respiration sums
  (loops_gswp3.py:575-584) and, when the state carries them, the
  growing-season stress sums (loops_gswp3.py:585-596).

State travels in dicts named as ``ibis_b200.layout`` (STAT, ACC, DAYST
fields).  Float32 constants of the reference's decomposition code are kept as
float32 scalars so the arithmetic promotes exactly as it does there.
"""
from __future__ import annotations

import numpy as np

f32 = np.float32
DAILY_SUMS = ("adrain", "adsnow", "adaet", "a10ancub", "a10ancls", "a10ancl3", "a10ancl4")


def daylength_hours(lat, doy):
    """state/seasonal.py:56-61 (latitude in radians, 1-based day of year)."""
    decl = 0.40910518 * np.sin(2.0 * np.pi * (doy - 81.0) / 365.0)
    return 24.0 / np.pi * np.arccos(np.clip(-np.tan(lat) * np.tan(decl), -1.0, 1.0))


def seasonal_states(day: dict, td, DP):
    """The seasonal states advanced from the day's mean temperature
    (loops_gswp3.py:418-437); returns (day, sen_u, sen_l), the photoperiod
    senescence triggers None where the switch is off."""
    tc = td - 273.16
    dl = daylength_hours(day["latitude"], DP.jday)
    dec = dl < daylength_hours(day["latitude"], DP.jday - 1)
    x = day["acclim_x"] + (tc - day["acclim_x"]) / DP.acclim_tau
    su = np.where(dec & (dl < DP.sen_pstart_u), day["ssen_u"] + np.maximum(DP.sen_tb_u - tc, 0.0), 0.0)
    sl = np.where(dec & (dl < DP.sen_pstart_l), day["ssen_l"] + np.maximum(DP.sen_tb_l - tc, 0.0), 0.0)
    sen_u = su >= DP.sen_ycrit_u if DP.sen_photoperiod_u else None
    sen_l = sl >= DP.sen_ycrit_l if DP.sen_photoperiod_l else None
    return dict(day, acclim_x=x, ssen_u=su, ssen_l=sl), sen_u, sen_l


def pheno(day: dict, stat: dict, means: dict, td, stresstu, stresstl, DP, epsilon, sen_u=None, sen_l=None):
    """Phenology of one day (phenology.py:89-287, habit off); ``sen_u`` /
    ``sen_l`` gate it by photoperiod (phenology.py:148-150, 170-172)."""
    tmelt = 273.16
    ddfac = 1.0 / DP.ddays
    a10td = means["a10td"]
    tthr_u = np.maximum(np.maximum(0.0 + tmelt, day["tc"] + DP.tthresh_u_offset + tmelt), DP.tthresh_u_abs + tmelt)
    gthr_u = DP.gthresh_u_c + tmelt
    cold_u, greset_u = a10td < tthr_u, a10td < gthr_u
    if sen_u is not None:
        cold_u, greset_u = cold_u | sen_u, greset_u | sen_u
    agddu = np.where(greset_u, 0.0, day["agddu"] + td - gthr_u)
    tempu = np.where(cold_u, np.maximum(0.0, day["tempu"] - ddfac),
                     np.minimum(1.0, np.maximum(0.0, agddu - DP.gdd_thresh_u) / DP.gdd_ramp_u))
    tthr_l = DP.tthresh_l_c + tmelt
    gthr_l = DP.gthresh_l_c + tmelt
    cold_l, greset_l = a10td < tthr_l, a10td < gthr_l
    if sen_l is not None:
        cold_l, greset_l = cold_l | sen_l, greset_l | sen_l
    agddl = np.where(greset_l, 0.0, day["agddl"] + td - gthr_l)
    templ = np.where(cold_l, np.maximum(0.0, day["templ"] - ddfac),
                     np.minimum(1.0, np.maximum(0.0, agddl - DP.gdd_thresh_l) / DP.gdd_ramp_l))

    def drop(old, anc, s):
        dry = (anc < DP.drop_thresh) | (s < DP.drop_stress_thresh)
        return np.where(dry, np.maximum(DP.drop_floor, old - ddfac), np.minimum(1.0, old + ddfac))
    dropu = drop(day["dropu"], means["a10ancub"], stresstu)
    dropls = drop(day["dropls"], means["a10ancls"], stresstl)
    dropl4 = drop(day["dropl4"], means["a10ancl4"], stresstl)
    dropl3 = drop(day["dropl3"], means["a10ancl3"], stresstl)
    plai = day["plai"]
    avglaiu = (plai[:, 0] + plai[:, 1] * dropu + plai[:, 2] + plai[:, 3] + plai[:, 4] * tempu + plai[:, 5]
               + plai[:, 6] * tempu + plai[:, 7] * tempu)
    au = np.maximum(avglaiu, epsilon)
    frac = stat["frac"].copy()
    for j, fac in ((0, 1.0), (1, dropu), (2, 1.0), (3, 1.0), (4, tempu), (5, 1.0), (6, tempu), (7, tempu)):
        frac[:, j] = (plai[:, j] * fac if not isinstance(fac, float) else plai[:, j]) / au
    m9, m10, m11 = np.minimum(templ, dropls), np.minimum(templ, dropl4), np.minimum(templ, dropl3)
    avglail = plai[:, 8] + plai[:, 9] * m9 + plai[:, 10] * m10 + plai[:, 11] * m11
    al = np.maximum(avglail, epsilon)
    frac[:, 8] = plai[:, 8] / al
    frac[:, 9] = plai[:, 9] * m9 / al
    frac[:, 10] = plai[:, 10] * m10 / al
    frac[:, 11] = plai[:, 11] * m11 / al
    lai_lower = np.minimum(avglail / np.maximum(stat["fl"], epsilon), 12.0)
    lai_upper = np.minimum(avglaiu / np.maximum(stat["fu"], epsilon), 12.0)
    lai = stat["lai"].copy()
    lai[:, 0], lai[:, 1] = lai_lower, lai_upper
    zbot = stat["zbot"].copy()
    zbot[:, 0] = 0.05
    ztop = stat["ztop"].copy()
    ztop[:, 0] = np.minimum(np.maximum(0.25, lai_lower * 0.25), stat["zbot"][:, 1] - 0.5)
    day = dict(day, tempu=tempu, templ=templ, agddu=agddu, agddl=agddl, dropu=dropu, dropls=dropls, dropl3=dropl3,
               dropl4=dropl4)
    stat = dict(stat, frac=frac, lai=lai, ztop=ztop, zbot=zbot)
    return day, stat


def day_begin(day: dict, stat: dict, acc: dict, td, P, DP):
    """Start of a day: phenology from the standing 10-day means, then the daily sums zeroed."""
    means = {k: day[k] for k in ("a10td", "a10ancub", "a10ancls", "a10ancl3", "a10ancl4")}
    sen_u = sen_l = None
    if DP.seasonal_on:
        day, sen_u, sen_l = seasonal_states(day, td, DP)
        # the day's steps read the advanced acclimation state (loops.py:294-303)
        stat = dict(stat, acclim_x=day["acclim_x"])
    day, stat = pheno(day, stat, means, td, acc["stresstu_last"], acc["stresstl_last"], DP, P.epsilon, sen_u, sen_l)
    acc = dict(acc)
    for k in DAILY_SUMS:
        acc[k] = np.zeros_like(acc[k])
    return day, stat, acc


def decomposition(prog: dict, hsoi, DP):
    """decompl and decomps (loops_gswp3.py:494-562, per-PFT tconst and SOM scaling off)."""
    tconst = f32(DP.lt_e0)
    wshift = DP.wfps_opt - 60.0
    btemp, tzero = f32(288.16), f32(227.13)

    def ftemp(t):
        safe = np.maximum(t, tzero + f32(10.0))
        return np.minimum(np.exp(tconst * (f32(1.0) / (btemp - tzero) - f32(1.0) / (safe - tzero))), f32(10.0))

    def fmoist(w, i):
        wfps = (f32(1.0) - i) * w * f32(100.0) - wshift
        wet = f32(0.000371) * wfps * wfps - f32(0.0748) * wfps + f32(4.13)
        dry = np.exp((wfps - f32(60.0)) ** 2 / f32(-800.0))
        return np.where(wfps >= f32(60.0), wet, dry)

    tsoi, wsoi, wisoi = prog["tsoi"], prog["wsoi"], prog["wisoi"]
    decompl = np.clip(ftemp(tsoi[:, 0]) * fmoist(wsoi[:, 0], wisoi[:, 0]) * DP.k_scale, f32(0.001), f32(10.0))
    h = hsoi
    h4 = h[0] + h[1] + h[2] + h[3]
    avg = lambda a: (a[:, 0] * h[0] + a[:, 1] * h[1] + a[:, 2] * h[2] + a[:, 3] * h[3]) / h4
    decomps = np.clip(ftemp(avg(tsoi)) * fmoist(avg(wsoi), avg(wisoi)) * DP.k_scale, f32(0.001), f32(10.0))
    return decompl, decomps


def soilbgc(d: dict, stat: dict, hsoi, DP, ndaypy):
    """One day of soil C/N (physics/biogeochem.py:23-243); returns the updated DAYST dict and tco2mic."""
    B = DP
    cnr = B.cnr
    totts = 1.0 / ndaypy

    def split(cn, c_last):
        fl = B.bgc_fmax * cn ** 2 / (B.rconst + cn ** 2)
        fs = (1.0 / cn - fl / cnr[4] - (1.0 - fl) / cnr[6]) / (1.0 / cnr[c_last] - 1.0 / cnr[6])
        return 1.0 - fl - fs, fs, fl
    fraclm, fracls, fracll = split(B.cnleaf, 5)
    fracrm, fracrs, fracrl = split(B.cnroot, 5)
    fracwm, fracws, fracwl = split(B.cnwood, 7)
    rdepth = 1.0 / (hsoi[0] + hsoi[1] + hsoi[2] + hsoi[3])
    texfact = np.sum(0.01 * stat["sand"][:, :4] * hsoi[:4], axis=1) * rdepth
    fbpom = 0.50
    totcin = (d["falll"] + d["fallr"] + d["fallw"]) * totts
    totcbegin = (d["clitlm"] + d["clitls"] + d["clitrm"] + d["clitrs"] + d["clitwm"] + d["clitws"] + d["csoislop"]
                 + d["csoislon"] + d["csoipas"] + d["totcmic"] + d["clitll"] + d["clitrl"] + d["clitwl"])
    cmicmx = B.fbsom * totcbegin
    cmicp = np.minimum(d["totcmic"], cmicmx)
    cmicn = np.maximum(0.0, d["totcmic"] - cmicmx)
    clitlm = d["clitlm"] + fraclm * d["falll"] * totts
    clitls = d["clitls"] + fracls * d["falll"] * totts
    clitll = d["clitll"] + fracll * d["falll"] * totts
    clitrm = d["clitrm"] + fracrm * d["fallr"] * totts
    clitrs = d["clitrs"] + fracrs * d["fallr"] * totts
    clitrl = d["clitrl"] + fracrl * d["fallr"] * totts
    clitwm = d["clitwm"] + fracwm * d["fallw"] * totts
    clitws = d["clitws"] + fracws * d["fallw"] * totts
    clitwl = d["clitwl"] + fracwl * d["fallw"] * totts
    dl, ds = d["decompl"], d["decomps"]
    slon, slop, pas = d["csoislon"], d["csoislop"], d["csoipas"]
    outcrs = np.minimum(ds * B.krs * clitrs, clitrs)
    outcws = np.minimum(dl * B.kws * clitws, clitws)
    outcls = np.minimum(dl * B.kls * clitls, clitls)
    outclm = np.minimum(dl * B.klm * clitlm, clitlm)
    outcrm = np.minimum(ds * B.krm * clitrm, clitrm)
    outcwm = np.minimum(dl * B.kwm * clitwm, clitwm)
    outcnb = np.minimum(ds * B.knb * slon, slon)
    outcpb = np.minimum(ds * B.kpb * slop, slop)
    outcsb = np.minimum(ds * B.ksb * pas, pas)
    outcbp = np.minimum(B.kbp * cmicp, cmicp) * B.effac
    outcbn = np.minimum(B.kbn * cmicn, cmicn) * B.effac
    dbdt = (outcrs * B.yrs + outcws * B.yws + outcls * B.yls + outclm * B.ylm + outcrm * B.yrm + outcwm * B.ywm
            + outcnb * B.ynb + outcpb * B.ypb + outcsb * B.ysb - outcbp - outcbn)
    outcll = np.minimum(dl * B.kll * clitll, clitll)
    outcrl = np.minimum(ds * B.krl * clitrl, clitrl)
    outcwl = np.minimum(dl * B.kwl * clitwl, clitwl)
    outcns = np.minimum(ds * B.kns * slon, slon)
    lig = B.lig_frac * (outcll * B.yll + outcrl * B.yrl + outcwl * B.ywl)
    dcndt = lig + (1.0 - fbpom) * (B.ybn * outcbn + B.ybp * outcbp) - outcnb - outcns
    outcps = np.minimum(ds * B.kps * slop, slop)
    dcpdt = lig + fbpom * (B.ybn * outcbn + B.ybp * outcbp) - outcpb - outcps
    fleach = 0.30e-03 / 18.0 * (0.01 + 0.04 * texfact)
    dcsdt = (B.yns * outcns + B.yps * outcps) - outcsb - fleach * pas
    cleach = fleach * (pas + slop + slon)
    ynleach = d["ynleach"] + fleach * pas / cnr[1] + fleach * slop / cnr[2] + fleach * slon / cnr[3]
    dcndt = dcndt - fleach * slon
    dcpdt = dcpdt - fleach * slop
    yrleach = d["yrleach"] + cleach

    def nmi(y, cf, ct, flux):
        net = (1.0 / ct - y / cf) * flux
        up = y / cf > 1.0 / ct
        return np.where(up, 0.0, net), np.where(up, net, 0.0)
    pairs = [nmi(B.yrs, cnr[0], cnr[5], outcrs), nmi(B.yls, cnr[0], cnr[5], outcls),
             nmi(B.yws, cnr[0], cnr[7], outcws), nmi(B.ywm, cnr[0], cnr[7], outcwm),
             nmi(B.ylm, cnr[0], cnr[6], outclm), nmi(B.yrm, cnr[0], cnr[6], outcrm),
             nmi(B.ynb, cnr[0], cnr[3], outcnb), nmi(B.ypb, cnr[0], cnr[2], outcpb),
             nmi(B.ysb, cnr[0], cnr[1], outcsb)]
    totimm = pairs[0][1] + pairs[1][1] + pairs[2][1] + pairs[3][1] + pairs[4][1] + pairs[5][1] + pairs[6][1] \
        + pairs[7][1] + pairs[8][1]
    totmin = pairs[0][0] + pairs[1][0] + pairs[2][0] + pairs[3][0] + pairs[4][0] + pairs[5][0] + pairs[6][0] \
        + pairs[7][0] + pairs[8][0]
    nrelps = outcps * (1.0 / cnr[2] - 1.0 / cnr[1])
    nrelns = outcns * (1.0 / cnr[3] - 1.0 / cnr[1])
    nrelbn = ((1.0 - fbpom) * outcbn * (1.0 / cnr[0] - 1.0 / cnr[3])
              + (1.0 - fbpom) * outcbp * (1.0 / cnr[0] - 1.0 / cnr[3]))
    nrelbp = (fbpom * outcbp * (1.0 / cnr[0] - 1.0 / cnr[2]) + fbpom * outcbn * (1.0 / cnr[0] - 1.0 / cnr[2]))
    lr = lambda o: (B.lig_frac * o * (1.0 / cnr[4] - 1.0 / cnr[2]) + B.lig_frac * o * (1.0 / cnr[4] - 1.0 / cnr[3]))
    totnrel = nrelps + nrelns + nrelbn + nrelbp + lr(outcll) + lr(outcrl) + lr(outcwl)
    netmin = totmin + totimm + totnrel
    tnmin = np.maximum(0.0, netmin) / (86400.0 * 0.014)
    totcmic = np.maximum(0.0, d["totcmic"] + dbdt)
    slon_n = np.maximum(0.0, slon + dcndt)
    slop_n = np.maximum(0.0, slop + dcpdt)
    pas_n = np.maximum(0.0, pas + dcsdt)
    clitlm = np.maximum(0.0, clitlm - outclm)
    clitls = np.maximum(0.0, clitls - outcls)
    clitll = np.maximum(0.0, clitll - outcll)
    clitrm = np.maximum(0.0, clitrm - outcrm)
    clitrs = np.maximum(0.0, clitrs - outcrs)
    clitrl = np.maximum(0.0, clitrl - outcrl)
    clitwm = np.maximum(0.0, clitwm - outcwm)
    clitws = np.maximum(0.0, clitws - outcws)
    clitwl = np.maximum(0.0, clitwl - outcwl)
    totlit = clitlm + clitls + clitll + clitrm + clitrs + clitrl + clitwm + clitws + clitwl
    totalit = clitlm + clitls + clitwm + clitll + clitws + clitwl
    totrlit = clitrm + clitrs + clitrl
    totcsoi = pas_n + slop_n + totcmic + slon_n
    totfall = d["falll"] + d["fallr"] + d["fallw"]
    tco2mic = (totcbegin + totcin - (totlit + totcsoi) - cleach) / (86400.0 * 0.012)
    out = dict(d, clitlm=clitlm, clitls=clitls, clitll=clitll, clitrm=clitrm, clitrs=clitrs, clitrl=clitrl,
               clitwm=clitwm, clitws=clitws, clitwl=clitwl, csoipas=pas_n, csoislon=slon_n, csoislop=slop_n,
               totcmic=totcmic, totlit=totlit, totalit=totalit, totrlit=totrlit, totcsoi=totcsoi, totfall=totfall,
               tnmin=tnmin, storedn=d["storedn"] + tnmin, yrleach=yrleach, ynleach=ynleach)
    return out, tco2mic


def day_end(prog: dict, day: dict, stat: dict, acc: dict, td, P, DP, ndaypy=365, day_sec=86400.0):
    """End of a day: 10-day means, annual sums, decomposition factors, soil BGC, respiration sums."""
    zweight = np.exp(-1.0 / 10.0)
    alpha10 = 1.0 - zweight
    day = dict(day)
    day["a10td"] = zweight * day["a10td"] + alpha10 * td
    for k in ("a10ancub", "a10ancls", "a10ancl3", "a10ancl4"):
        day[k] = zweight * day[k] + alpha10 * (acc[k] / day_sec)
    day["ayprcp"] = day["ayprcp"] + acc["adrain"] + acc["adsnow"]
    day["ayaet"] = day["ayaet"] + acc["adaet"]
    hsoi = np.asarray(P.hsoi, dtype=np.float64)
    day["decompl"], day["decomps"] = decomposition(prog, hsoi, DP)
    day, tco2mic = soilbgc(day, stat, hsoi, DP, ndaypy)
    stat = dict(stat, tco2mic=tco2mic)
    day["ayco2mic"] = day["ayco2mic"] + tco2mic * f32(12.0e-3 * 86400.0)
    day["ayco2root"] = day["ayco2root"] + day["tco2root"] * f32(12.0e-3 * 86400.0)
    if DP.stress_on:
        grow = (td > 273.16 + DP.stress_accum_tmin).astype(np.float64)
        day["aystressu"] = day["aystressu"] + acc["stresstu_last"] * grow
        day["aystressl"] = day["aystressl"] + acc["stresstl_last"] * grow
        day["stress_nday"] = day["stress_nday"] + grow
    return day, stat
