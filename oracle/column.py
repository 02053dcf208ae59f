"""Snow, soil (+bedrock) column solves, fire counters, accumulators and CH4.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).  Restates
``python-port/ibis/physics/snow_physics.py``, ``soil_physics.py``,
``bedrock.py``, the per-step part of ``fire.py``, ``bgc/methane.py`` and the
accumulators of ``timestepping/loops_gswp3.py`` in float64 NumPy.
"""
from __future__ import annotations

import types

import numpy as np

from .physics import clip, esat, thomas


# ---------------------------------------------------------------------------
# snow -- snow_physics.py
# ---------------------------------------------------------------------------


def snow_heat(tsno, tlsub, fhtop, xl, fi, hsno, hsoi0, consoi0, tsoi0, P):
    """snowheat: implicit conduction through snow layers + a buried-vegetation node (snow_physics.py:109-229)."""
    n, ns = tsno.shape
    conbur, hfake = 2.0, 0.01
    temp = np.concatenate([tsno, tlsub[:, None]], axis=1)
    con = np.zeros((n, ns + 2))
    rs = 0.5 / P.consno
    for k in range(1, ns):
        con[:, k] = 1.0 / (np.maximum(hsno[:, k - 1], hfake) * rs + np.maximum(hsno[:, k], hfake) * rs)
    con[:, ns] = 1.0 / (np.maximum(hsno[:, ns - 1], hfake) * rs + 0.5 * xl / conbur)
    con[:, ns + 1] = 1.0 / (xl * (0.5 / conbur) + 0.5 * hsoi0 / np.maximum(consoi0, 1e-12))
    lo = np.zeros((n, ns + 1))
    di = np.zeros((n, ns + 1))
    up = np.zeros((n, ns + 1))
    r = np.zeros((n, ns + 1))
    rdt = P.dtime / (P.rhos * P.cice)
    for k in range(ns):
        dt = rdt / np.maximum(hsno[:, k], hfake)
        lo[:, k] = -dt * con[:, k]
        di[:, k] = 1.0 + dt * (con[:, k] + con[:, k + 1])
        up[:, k] = -dt * con[:, k + 1]
        r[:, k] = temp[:, k]
        if k == 0:
            r[:, k] = r[:, k] + dt * fhtop
    k = ns
    dti = xl * P.chl / P.dtime
    lo[:, k] = -con[:, k]
    di[:, k] = dti + (con[:, k] + con[:, k + 1])
    r[:, k] = dti * temp[:, k] + con[:, k + 1] * tsoi0
    tn = thomas(lo, di, up, r)
    sflo_last = fhtop.copy()
    rh = P.rhos * P.cice / P.dtime
    for k in range(ns):
        sflo_last = sflo_last - rh * hsno[:, k] * (tn[:, k] - tsno[:, k])
    sflo_bot = sflo_last - xl * (P.chl / P.dtime) * (tn[:, ns] - tlsub)
    has = fi > 0.0
    return (np.where(has[:, None], tn[:, :ns], tsno), np.where(has, tn[:, ns], tlsub), sflo_bot)


def readapt_layers(h, t, htop, has, eps):
    """vadapt (snow_physics.py:27-106)."""
    n, ns = h.shape
    zold = np.zeros((n, ns + 1))
    for k in range(ns):
        zold[:, k + 1] = zold[:, k] + h[:, k]
    ht = zold[:, ns]
    thick = ht >= ns * htop
    h1 = np.where(thick, (ht - htop) / (ns - 1), np.maximum(ht / ns, eps))
    hn = np.repeat(h1[:, None], ns, axis=1)
    hn[:, 0] = np.where(thick, htop, h1)
    znew = np.zeros((n, ns + 1))
    for k in range(ns):
        znew[:, k + 1] = znew[:, k] + hn[:, k]
    tn = np.zeros((n, ns))
    for k in range(ns):
        acc = np.zeros(n)
        for ko in range(ns):
            ov = np.maximum(np.minimum(zold[:, ko + 1], znew[:, k + 1]) - np.maximum(zold[:, ko], znew[:, k]), 0.0)
            acc = acc + t[:, ko] * ov
        tn[:, k] = acc / np.maximum(hn[:, k], eps)
    return np.where(has[:, None], hn, h), np.where(has[:, None], tn, t)


def snow_block(prog, S, casc, heati, fvapi, tl_nv, wliql_nv, wsnol_nv, consoi0, P):
    """Snow section of timestep_body (loops.py:676-848); returns updated snow state and ground fluxes."""
    fi = prog["fi"]
    tsno, hsno = prog["tsno"], prog["hsno"]
    ns = tsno.shape[1]
    eps = P.epsilon
    fhtop = (heati + casc["rainl"] * (P.ch2o * (casc["trainl"] - P.tmelt) + P.hfus + P.cice * (P.tmelt - tsno[:, 0]))
             + casc["snowl"] * P.cice * (casc["tsnowl"] - tsno[:, 0]))
    xl = S["fl"] * 2.0 * (S["lai"][:, 0] + S["sai"][:, 0])
    hp = hsno.copy()
    hp[:, 0] = hsno[:, 0] + (casc["rainl"] + casc["snowl"] - fvapi) * (P.dtime / P.rhos)
    hp = np.where(fi[:, None] > 0.0, hp, hsno)
    tsh, tlsub_h, sflo_bot = snow_heat(tsno, prog["tlsub"], fhtop, xl, fi, hp, P.hsoi[0], consoi0,
                                       prog["tsoi"][:, 0], P)
    ht = np.sum(hp, axis=1)
    hts = np.where(ht > 0.0, ht, P.hsnomin)
    dfi = (1.0 - fi) * P.dtime * casc["snowg"] / (P.rhos * hts)
    dfi = np.minimum(dfi, 1.0 - fi)
    fi1 = fi + dfi
    tmix = np.where((fi1 > 0.0)[:, None],
                    (tsh * fi[:, None] + casc["tsnowg"][:, None] * dfi[:, None]) / np.maximum(fi1[:, None], eps), tsh)
    hinit = np.full_like(hp, (P.hsnomin - P.hsnotop) / max(ns - 1, 1))
    hinit[:, 0] = P.hsnotop
    hpm = np.where(((fi < eps) & (dfi > 0.0))[:, None], hinit, hp)
    # snow_melt (snow_physics.py:236-260)
    xh = P.rhos * hpm * P.cice * np.maximum(tmix - P.tmelt, 0.0)
    xm = np.minimum(P.rhos * hpm, xh / P.hfus)
    hm = hpm - xm / P.rhos
    tm = np.minimum(tmix, P.tmelt)
    smelt = np.sum(fi1[:, None] * xm, axis=1)
    zheat = np.sum(fi1[:, None] * (xh - P.hfus * xm), axis=1)
    # snow_coverage (snow_physics.py:263-290)
    ruf = np.minimum(0.70, np.maximum(P.hsnomin + 0.05, S["fl"] * S["ztop"][:, 0]))
    htc = np.sum(hm, axis=1)
    htc = np.where(htc < 1e-10, P.hsnomin, htc)
    zhh = 0.5 * P.hsnomin
    zdh = np.maximum(ruf - P.hsnomin, eps)
    fic = clip((-zhh + np.sqrt(zhh ** 2 + zdh * fi1 * htc)) / zdh, 0.0, P.fimax)
    hc = hm * (fi1 / np.maximum(fic, eps))[:, None]
    hv, tv = readapt_layers(hc, tm, P.hsnotop, np.sum(hc, axis=1) > eps, eps)
    # fimin melt-all
    small = fic < P.fimin
    rmass = P.rhos * np.sum(hv, axis=1) * fic
    rheat = -np.sum(P.rhos * hv * fic[:, None] * (P.cice * (P.tmelt - tv) + P.hfus), axis=1)
    smelt = np.where(small, smelt + rmass, smelt)
    zheat = np.where(small, zheat + rheat, zheat)
    hf = np.where(small[:, None], 0.0, hv)
    tv = np.where(small[:, None], P.tmelt, tv)
    fin = np.where(small, 0.0, fic)
    # buried vegetation (loops.py:781-830)
    dfc = fin - fi
    grow = dfc > 0
    tlsub = np.where(grow, (tlsub_h * fi + tl_nv * dfc) / np.maximum(fin, eps), tlsub_h)
    zheat = np.where(grow, zheat + dfc * xl * (
        wliql_nv * (P.ch2o * (tl_nv - P.tmelt) + P.hfus + P.cice * (P.tmelt - tv[:, -1]))
        + wsnol_nv * P.cice * (tl_nv - tv[:, -1])), zheat)
    hlast = hf[:, -1] + dfc * xl * (wliql_nv + wsnol_nv) / (P.rhos * np.maximum(fin, eps))
    hf[:, -1] = np.where(grow, hlast, hf[:, -1])
    shrink = dfc < 0
    zheat = np.where(shrink, zheat - dfc * xl * P.chl * (tlsub_h - tl_nv), zheat)
    rdec = np.where(shrink, (1.0 - fi) / np.maximum(1.0 - fin, eps), 1.0)
    wliql_nv = wliql_nv * rdec
    wsnol_nv = wsnol_nv * rdec
    tlsub = np.where(fin > 0, tlsub, tl_nv)
    return dict(fi=fin, tsno=tv, hsno=hf, tlsub=tlsub, smelt=smelt, zheat=zheat, sflo_bot=sflo_bot,
                fhtop_snow=fhtop, wliql=wliql_nv, wsnol=wsnol_nv)


# ---------------------------------------------------------------------------
# soil -- soil_physics.py, bedrock.py
# ---------------------------------------------------------------------------


def water_bounds(wsoi, wisoi, poros, hsoi, P):
    """wadjust (soil_physics.py:147-189)."""
    eps = P.epsilon
    z0 = hsoi[None, :] * poros * P.rhow * ((1.0 - wisoi) * wsoi + wisoi)
    w = np.where(wsoi < eps, 0.0, wsoi)
    i = np.where(wisoi < eps, 0.0, wisoi)
    w = np.minimum(1.0, w)
    i = np.minimum(1.0, i)
    w = np.where(i >= 1.0 - eps, 0.0, w)
    z1 = hsoi[None, :] * poros * P.rhow * ((1.0 - i) * w + i)
    return w, i, np.sum(z1 - z0, axis=1) / P.dtime


def soil_water(wsoi, wisoi, poros, porosflo, S, hsoi, fwtop, fwpud, wpud, P):
    """soilh2o: implicit Richards-type moisture solve (soil_physics.py:196-373)."""
    n, nl = wsoi.shape
    hyd, suc, bex = S["hydraul"], S["suction"], S["bex"]
    dmin = 1e-9
    e = np.zeros((n, nl + 1))
    f = np.zeros((n, nl + 1))
    g = np.zeros((n, nl + 1))
    consistent = bool(P.flags & (1 << 1))
    for k in range(1, nl):
        hm = 0.5 * (hsoi[k - 1] + hsoi[k])
        wp = 0.5 * hsoi[k] / hm
        wm = 1.0 - wp
        a = wm * hyd[:, k - 1] + wp * hyd[:, k]
        b = wm * hyd[:, k - 1] * suc[:, k - 1] * bex[:, k - 1] + wp * hyd[:, k] * suc[:, k] * bex[:, k]
        zb = wm * bex[:, k - 1] + wp * bex[:, k]
        nb = np.floor(zb + 0.5).astype(np.int32)
        m = 2 * nb + 3
        nn = nb + 2
        if consistent:
            ws = wp * wsoi[:, k - 1] + wm * wsoi[:, k]
        else:
            ws = wm * wsoi[:, k - 1] + wp * wsoi[:, k]
        wa = np.minimum(ws, 1.0)
        bwn1 = b * (wa ** (nn - 1))
        bwn = bwn1 * wa
        bwn1 = np.where(bwn < dmin, 0.0, bwn1)
        bwn = np.maximum(bwn, dmin)
        dw = (wsoi[:, k] - wsoi[:, k - 1]) / hm
        ek = (-1.0 + m) * a * (wa ** m) + ((0.0 * bwn) - nn * bwn1 * wa) * dw
        fk = -m * a * (wa ** (m - 1)) + nn * bwn1 * dw
        zi = np.maximum(0.0, 1.0 - np.maximum(wisoi[:, k - 1], wisoi[:, k])) ** 2
        e[:, k] = zi * ek
        f[:, k] = zi * fk
        g[:, k] = zi * bwn
    wab = np.minimum(wsoi[:, nl - 1], 1.0)
    mb = 2 * np.floor(bex[:, nl - 1] + 0.5).astype(np.int32) + 3
    e[:, nl] = (np.maximum(0.0, 1.0 - wisoi[:, nl - 1]) ** 2) * (-hyd[:, nl - 1] * (wab ** mb) * P.bperm)

    lo = np.zeros((n, nl))
    di = np.zeros((n, nl))
    up = np.zeros((n, nl))
    r = np.zeros((n, nl))
    for k in range(nl):
        dt = P.dtime / np.maximum(porosflo[:, k] * hsoi[k], 1e-30)
        hm = 0.5 * hsoi[0] if k == 0 else 0.5 * hsoi[k - 1] + 0.5 * hsoi[k]
        hm = max(hm, 1e-30)
        km1 = max(k - 1, 0)
        d1 = dt * (f[:, k] * 0.5 * hsoi[k] / hm - g[:, k] / hm)
        rk = wsoi[:, k] + dt * (e[:, k + 1] - e[:, k])
        if k == 0:
            rk = rk + dt * (fwtop + fwpud) / P.rhow
            d1 = np.zeros(n)
        if k < nl - 1:
            hp = max(0.5 * (hsoi[k] + hsoi[k + 1]), 1e-30)
            d2 = 1.0 + dt * (-f[:, k + 1] * 0.5 * hsoi[k + 1] / hp + f[:, k] * 0.5 * hsoi[km1] / hm
                             + g[:, k + 1] / hp + g[:, k] / hm)
            d3 = dt * (-f[:, k + 1] * 0.5 * hsoi[k] / hp - g[:, k + 1] / hp)
        else:
            d2 = 1.0 + dt * (-f[:, k + 1] + f[:, k] * 0.5 * hsoi[km1] / hm + g[:, k] / hm)
            d3 = np.zeros(n)
        lo[:, k], di[:, k], up[:, k], r[:, k] = d1, d2, d3, rk
    wn = thomas(lo, di, up, r)
    wflo = np.zeros((n, nl + 1))
    wflo[:, nl] = -P.rhow * e[:, nl]
    fsq = np.zeros(n)
    for k in range(nl - 1, -1, -1):
        zz = P.rhow * poros[:, k] * np.maximum(P.epsilon, 1.0 - wisoi[:, k]) * hsoi[k]
        wk = wn[:, k] + P.dtime * fsq / zz
        fsq_n = np.maximum(wk - 1.0, 0.0) * zz / P.dtime
        wk = np.minimum(wk, 1.0)
        wflo[:, k] = wflo[:, k + 1] + (wk - wsoi[:, k]) * zz / P.dtime
        wn[:, k] = wk
        fsq = fsq_n
    wpud_n = np.maximum(wpud + (fsq - fwpud) * P.dtime, 0.0)
    wflo[:, 0] = wflo[:, 0] + fsq - fwpud
    return wn, wpud_n, wflo


def soil_heat(tsoi, otsoi, owsoi, wsoi, wisoi, poros, consoi, csoi, rhosoi, hsoi, c0pud, c1pud, fhtop, wflo,
              n_hyd, P):
    """soilheat with thermal-only layers below n_hyd (soil_physics.py:385-490; bedrock.py:88-153)."""
    n, nl = tsoi.shape
    con = np.zeros((n, nl + 1))
    whf = np.zeros((n, nl + 1))
    whf[:, 0] = wflo[:, 0] * P.ch2o * tsoi[:, 0]
    for k in range(1, nl):
        con[:, k] = 1.0 / (0.5 * (hsoi[k - 1] / np.maximum(consoi[:, k - 1], 1e-12)
                                  + hsoi[k] / np.maximum(consoi[:, k], 1e-12)))
        if k < n_hyd:
            tav = (hsoi[k] * tsoi[:, k - 1] + hsoi[k - 1] * tsoi[:, k]) / (hsoi[k - 1] + hsoi[k])
            whf[:, k] = wflo[:, k] * P.ch2o * tav
    drain = wflo[:, n_hyd] * P.ch2o * tsoi[:, n_hyd - 1]
    for k in range(n_hyd, nl + 1):
        whf[:, k] = drain
    r1 = (1.0 - poros) * csoi * rhosoi
    r2 = poros * (1.0 - wisoi) * P.ch2o * P.rhow
    r3 = poros * wisoi * P.cice * P.rhow
    c0 = c0pud + (r1 + r2 * owsoi + r3) * hsoi[None, :]
    c1 = c1pud + (r1 + r2 * wsoi + r3) * hsoi[None, :]
    lo = np.zeros((n, nl))
    di = np.zeros((n, nl))
    up = np.zeros((n, nl))
    r = np.zeros((n, nl))
    for k in range(nl):
        rw = P.dtime / c1[:, k]
        lo[:, k] = -rw * con[:, k]
        di[:, k] = 1.0 + rw * (con[:, k] + con[:, k + 1])
        up[:, k] = -rw * con[:, k + 1]
        r[:, k] = (c0[:, k] / c1[:, k]) * tsoi[:, k] + rw * (whf[:, k] - whf[:, k + 1])
        if k == 0:
            r[:, k] = r[:, k] + (P.dtime / c1[:, k]) * fhtop
    tn = thomas(lo, di, up, r)
    hflo = np.zeros((n, nl + 1))
    hflo[:, 0] = fhtop
    for k in range(nl):
        hflo[:, k + 1] = hflo[:, k] - (c1[:, k] * tn[:, k] - c0[:, k] * otsoi[:, k]) / P.dtime
    return tn, hflo


def phase_change(tsoi, wsoi, wisoi, poros, csoi, rhosoi, hsoi, c1pud, P):
    """freeze_thaw: heat-conserving layer phase change (soil_physics.py:497-564)."""
    eps = P.epsilon
    t, w, i = tsoi.copy(), wsoi.copy(), wisoi.copy()
    for k in range(t.shape[1]):
        zp = np.maximum(poros[:, k], eps)
        rw = c1pud[:, k] / (P.rhow * hsoi[k]) + (1.0 - zp) * csoi[:, k] * rhosoi[:, k] / P.rhow
        chav = rw + zp * (1.0 - i[:, k]) * w[:, k] * P.ch2o + zp * i[:, k] * P.cice
        zw = np.minimum(1.0, w[:, k])
        dh = chav * (P.tmelt - t[:, k])
        dw = np.minimum(zp * (1.0 - i[:, k]) * zw, np.maximum(0.0, dh / P.hfus))
        ik = i[:, k] + dw / zp
        wk = w[:, k] - (dw / zp) * (1.0 - zw) / np.maximum(eps, 1.0 - ik)
        chav = rw + zp * (1.0 - ik) * wk * P.ch2o + zp * ik * P.cice
        tk = P.tmelt - (dh - P.hfus * dw) / chav
        dh = chav * (tk - P.tmelt)
        dw = np.minimum(zp * ik, np.maximum(0.0, dh / P.hfus))
        ik = ik - dw / zp
        wk = wk + (dw / zp) * (1.0 - wk) / np.maximum(eps, 1.0 - ik)
        chav = rw + zp * (1.0 - ik) * wk * P.ch2o + zp * ik * P.cice
        t[:, k] = P.tmelt + (dh - P.hfus * dw) / chav
        w[:, k] = wk
        i[:, k] = ik
    return t, w, i, poros * np.maximum(eps, 1.0 - i)


def puddle_phase(t0, wpud, wipud, poros0, w0, i0, csoi0, rho0, h0, P):
    """puddle_freeze_thaw (soil_physics.py:567-615)."""
    rw = ((1.0 - poros0) * csoi0 * rho0 + poros0 * (1.0 - i0) * w0 * P.ch2o * P.rhow
          + poros0 * i0 * P.cice * P.rhow) * h0
    chav = P.ch2o * wpud + P.cice * wipud + rw
    dh = chav * (P.tmelt - t0)
    dw = np.minimum(wpud, np.maximum(0.0, dh / P.hfus))
    wipud = wipud + dw
    wpud = wpud - dw
    chav = P.ch2o * wpud + P.cice * wipud + rw
    t0 = P.tmelt - (dh - P.hfus * dw) / chav
    dh = chav * (t0 - P.tmelt)
    dw = np.minimum(wipud, np.maximum(0.0, dh / P.hfus))
    wipud = wipud - dw
    wpud = wpud + dw
    chav = P.ch2o * wpud + P.cice * wipud + rw
    t0 = P.tmelt + (dh - P.hfus * dw) / chav
    return t0, np.maximum(wpud, 0.0), np.maximum(wipud, 0.0)


# ---------------------------------------------------------------------------
# fire counters -- fire.py:88-140, 340-366, 470-514, 583-604
# ---------------------------------------------------------------------------


def fuel_dryness(w0, i0, swilt0):
    water = i0 + (1.0 - i0) * w0
    frac = (water - swilt0) / (1.0 - swilt0)
    return np.minimum(1.0, np.maximum(0.0, -2.0 * (frac - 0.5)))


def fire_counters(prog, wsoi0, wisoi0, swilt0, F, P):
    nyt = prog["nytimes"] + 1.0
    fd = fuel_dryness(wsoi0, wisoi0, swilt0)
    nn = np.maximum(nyt, 1.0)
    out = dict(nytimes=nyt, firefac=((nn - 1.0) * prog["firefac"] + fd) / nn)
    hit = (fd > P.d_crit).astype(np.float64)
    out["nfirestep"] = prog["nfirestep"] + hit
    out["sdry"] = prog["sdry"] + fd * hit
    eact = F["qa"] * F["psurf"] / (0.622 + 0.378 * F["qa"])
    vpd = np.maximum(esat(F["ta"]) - eact, 0.0) / 1000.0
    fl = clip(vpd / P.vpd_ref, 0.0, 1.0)
    hit = (fl > P.d_crit_vpd).astype(np.float64)
    out["nfirestep_vpd"] = prog["nfirestep_vpd"] + hit
    out["sdry_vpd"] = prog["sdry_vpd"] + fl * hit
    return out


# ---------------------------------------------------------------------------
# wetland CH4 -- bgc/methane.py:233-383
# ---------------------------------------------------------------------------


CH4_FIELDS = ("sat_crit", "z_max", "r_ch4", "q10p", "t_ref", "z_wt_max", "z_wt_ref", "z_tau", "tau_oxid")
FLAG_CH4_BANDS = 1 << 23


def methane_params(P, S):
    """The methane parameters each cell uses: ``P``'s, or under FLAG_CH4_BANDS
    per-cell arrays of the ``ch4b_*`` tables at the cell's band (STAT ch4_band:
    0 tropical, 1 temperate, 2 boreal), as biome_methane_params gives every
    cell its band's values (methane.py:521-563)."""
    if not P.flags & FLAG_CH4_BANDS:
        return P
    band = np.asarray(S["ch4_band"], np.float64)
    b = np.where(band >= 1.5, 2, np.where(band >= 0.5, 1, 0))
    return types.SimpleNamespace(**{f: np.asarray(getattr(P, "ch4b_" + f), np.float64)[b] for f in CH4_FIELDS})


def wetland_water_table(wsoi, wisoi, hsoi, P, zwt_obs=None):
    """wetland_water_table (methane.py:233-276), with an observed depth (finite
    entries of ``zwt_obs``, clipped to [0, z_max]) in its place where given
    (methane.py:366-367).  ``P``'s methane fields are scalars or per-cell arrays."""
    theta = clip(wsoi * (1.0 - wisoi) + wisoi, 0.0, 1.0)
    bot = np.cumsum(hsoi)
    top = np.concatenate([[0.0], bot[:-1]])
    zref = np.asarray(P.z_wt_ref, np.float64)
    w = np.minimum(np.maximum(zref[..., None] - top, 0.0), hsoi)         # (nlayer,) or per cell (ncell, nlayer)
    tot = np.maximum(np.sum(w, axis=-1), 1e-12)
    ttop = np.sum(theta * w, axis=1) / tot
    wet = clip(ttop / np.maximum(P.sat_crit, 1e-6), 0.0, 1.0)
    zwt = P.z_wt_max * (1.0 - wet)
    if zwt_obs is not None:
        zo = np.asarray(zwt_obs, dtype=np.float64)
        with np.errstate(invalid="ignore"):
            zwt = np.where(np.isfinite(zo), np.clip(zo, 0.0, P.z_max), zwt)
    return zwt


def methane(f_inund, rh, tsoi, wsoi, wisoi, hsoi, P, zwt_obs=None):
    bot = np.cumsum(hsoi)
    top = np.concatenate([[0.0], bot[:-1]])
    zwt = wetland_water_table(wsoi, wisoi, hsoi, P, zwt_obs)
    below = bot[None, :] - np.maximum(zwt[:, None], top[None, :])
    an = clip(below / hsoi[None, :], 0.0, 1.0) * hsoi[None, :]
    th = an * (tsoi >= 273.15)
    tt = np.sum(th, axis=1)
    tth = np.where(tt > 1e-12, np.sum(th * tsoi, axis=1) / np.maximum(tt, 1e-12), tsoi[:, 0])
    zp = np.maximum(zwt, 0.0)
    rha = np.maximum(rh, 0.0) * np.exp(-zp / np.maximum(P.z_tau, 1e-6))
    q10 = P.q10p ** ((tth - P.t_ref) / 10.0)
    prod = np.maximum(rha, 0.0) * P.r_ch4 * q10 * (tth >= 273.15)
    area = clip(np.maximum(f_inund, 0.0), 0.0, 1.0)
    return area * prod * np.exp(-zp / np.maximum(P.tau_oxid, 1e-6))
