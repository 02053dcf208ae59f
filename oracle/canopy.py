"""Canopy aerodynamics, photosynthesis/stomata and the 9x9 canopy energy solve.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).  Restates
``python-port/ibis/physics/canopy_exchange.py`` and
``python-port/ibis/physics/stomata.py`` in float64 NumPy.
"""
from __future__ import annotations

import numpy as np

from .physics import (clip, cube, esat, qsat, dqsat, hvapf, hsubf, FLAG_VMAX_MIX, FLAG_COEFM_MIX, FLAG_ACCLIM,
                      FLAG_ACCLIM_LIGHT, FLAG_FROST, FLAG_CAP_SCALE_U, FLAG_CAP_SCALE_L, FLAG_LEAF_ONLY, FLAG_CROP)


# ---------------------------------------------------------------------------
# canini -- canopy_exchange.py:192-280
# ---------------------------------------------------------------------------


def aero_geometry(F, S, fi, P):
    ta, qa, ps, ua = F["ta"], F["qa"], F["psurf"], F["ua"]
    lai, sai, ztop, zbot, fu, fl = S["lai"], S["sai"], S["ztop"], S["zbot"], S["fu"], S["fl"]
    z0soi = S["z0soi"]
    A = {}
    siga = 0.999
    A["tfac"] = 1.0 / (siga ** P.cappa)
    pa = ps * siga
    A["rhoa"] = pa / (P.rair * ta * (1.0 + (P.rvap / P.rair - 1.0) * qa))
    A["cp"] = P.cair * (1.0 + (P.cvap / P.cair - 1.0) * qa)
    za = (ps - pa) / (A["rhoa"] * P.grav)
    za = np.maximum(za, ztop[:, 1] + 1.0)
    A["za"] = za

    x = fl * (1.0 - fi) * 2.0 * (lai[:, 0] + sai[:, 0]) / P.alaiml
    x = np.minimum(x, 3.0)
    x1 = np.minimum(x, 1.0)
    rw = np.maximum(ztop[:, 0] - zbot[:, 0], 0.01)
    cveg = (0.4 / rw) * np.maximum(1e-5, x)
    dveg = (0.1 * rw) / np.maximum(1e-5, np.maximum(x, x * x))
    bveg = np.sqrt(2.0 * cveg / dveg)
    A["bdl"] = 0.5 * bveg * dveg
    A["dil"] = 1.0 / dveg
    rw = (1.0 - x1) * (np.maximum(z0soi, P.z0sno) + 0.01)
    z3 = x1 * ztop[:, 0] + rw
    z4 = x1 * zbot[:, 0] + rw
    A["z3"], A["z4"], A["z34"] = z3, z4, 0.5 * (z3 + z4)
    A["exphl"] = np.exp(0.5 * bveg * (z3 - z4))
    A["expl"] = A["exphl"] * A["exphl"]
    displ = x1 * 0.7 * z3

    x = fu * 2.0 * (lai[:, 1] + sai[:, 1]) / P.alaimu
    x = np.minimum(x, 3.0)
    x1 = np.minimum(x, 1.0)
    rw = np.maximum(ztop[:, 1] - zbot[:, 1], 0.01)
    cveg = (0.4 / rw) * np.maximum(1e-5, x)
    dveg = (0.1 * rw) / np.maximum(1e-5, np.maximum(x, x * x))
    rw = 1.0 / dveg
    bveg = np.sqrt(2.0 * cveg * rw)
    A["bdu"] = 0.5 * bveg * dveg
    A["diu"] = rw
    rw = (1.0 - x1) * (z3 + 0.01)
    z1 = x1 * ztop[:, 1] + rw
    z2 = x1 * zbot[:, 1] + rw
    A["z1"], A["z2"], A["z12"] = z1, z2, 0.5 * (z1 + z2)
    A["exphu"] = np.exp(0.5 * bveg * (z1 - z2))
    A["expu"] = A["exphu"] * A["exphu"]
    dispu = x1 * 0.7 * z1 + (1.0 - x1) * displ

    alogg = np.log(z0soi)
    alogi = np.log(P.z0sno)
    A["alogav"] = (1.0 - fi) * alogg + fi * alogi
    A["alog4"] = np.log(np.maximum(z4, np.maximum(1.1 * z0soi, 1.1 * P.z0sno)))
    A["alog3"] = np.log(z3 - displ)
    A["alog2"] = np.log(z2 - displ)
    A["alog1"] = np.log(z1 - dispu)
    A["aloga"] = np.log(za - dispu)
    A["u2"] = ua / A["exphu"]
    A["alogu"] = np.log(np.maximum(0.01, 0.1 * (z1 - z2)))
    A["alogl"] = np.log(np.maximum(0.01, 0.1 * (z3 - z4)))
    return A


# ---------------------------------------------------------------------------
# fstrat / turcof -- canopy_exchange.py:287-426
# ---------------------------------------------------------------------------


def stability(tb, tt, ttfac, qb, qt, zb, zt, alb, alt, u, first, sm_prev, sh_prev, P):
    zht = tt * ttfac * (1.0 + 0.622 * qt)
    zhb = tb * (1.0 + 0.622 * qb)
    rich = P.grav * np.maximum(zt - zb, 0.0) * (zht - zhb) / (0.5 * (zht + zhb) * (u * u))
    rich = clip(rich, -2.0, 1.0)
    xm = np.maximum(alt - alb, 0.5)
    rw = np.sqrt(np.maximum(-rich, 0.0))
    vx = P.vonk / xm
    ym = (vx * vx) * np.exp(0.5 * xm) * rw
    sm_u = 1.0 - 10.0 * rich / (1.0 + 75.0 * ym)
    sh_u = 1.0 - 15.0 * rich / (1.0 + 75.0 * ym)
    rp = np.maximum(rich, 0.0)
    zz = np.sqrt(1.0 + 5.0 * rp)
    sm_s = 1.0 / (1.0 + 10.0 * rp / zz)
    sh_s = 1.0 / (1.0 + 15.0 * rp * zz)
    sm = np.where(rich <= 0.0, sm_u, sm_s)
    sh = np.where(rich <= 0.0, sh_u, sh_s)
    if not first:
        sm = 0.5 * sm + 0.5 * sm_prev
        sh = 0.5 * sh + 0.5 * sh_prev
    return sm, sh


def transfer(A, F, t12, t34, q12, q34, first, strat, P):
    """turcof; A carries u2/alogu/alogl of the previous pass. Returns coefficients and new strat."""
    ta, qa, ua = F["ta"], F["qa"], F["ua"]
    vonk = P.vonk
    sml, shl = stability(t34, t12, 1.0, q34, q12, A["z3"], A["z2"], A["alogl"], A["alog2"], A["u2"],
                         first, strat[0], strat[1], P)
    smu, shu = stability(t12, ta, A["tfac"], q12, qa, A["z1"], A["za"], A["alogu"], A["aloga"], ua,
                         first, strat[2], strat[3], P)
    v = (A["alog4"] - A["alogav"]) / vonk
    x = (v * v) * A["bdl"]
    rw = 1.0 / A["expl"]
    yl = ((x + 1) * A["expl"] + (x - 1) * rw) / ((x + 1) * A["expl"] - (x - 1) * rw)
    alogl = A["alog3"] - vonk * np.sqrt(yl / A["bdl"])
    v = (A["alog2"] - alogl) / vonk
    x = (v * v) * A["bdu"] / sml
    rw = 1.0 / A["expu"]
    yu = ((x + 1) * A["expu"] + (x - 1) * rw) / ((x + 1) * A["expu"] - (x - 1) * rw)
    alogu = A["alog1"] - vonk * np.sqrt(yu / A["bdu"])
    cdmax = 300.0 / (2.0 * P.dtime)
    v = ua * vonk / (A["aloga"] - alogu)
    tauu = (v * v) * smu
    a = 0.5 * tauu * (yu + 1) / A["bdu"]
    b = 0.5 * tauu * (yu - 1) / A["bdu"]
    taul = A["bdu"] * (a / A["expu"] - b * A["expu"])
    c = 0.5 * taul * (yl + 1) / A["bdl"]
    d = 0.5 * taul * (yl - 1) / A["bdl"]
    us = lambda w: np.maximum(0.01, np.sqrt(np.maximum(0.0, w)))
    u1 = us(a + b)
    u12 = us(a / A["exphu"] + b * A["exphu"])
    u2 = us(a / A["expu"] + b * A["expu"])
    u3 = us(c + d)
    u34 = us(c / A["exphl"] + d * A["exphl"])
    u4 = us(c / A["expl"] + d * A["expl"])
    vk2 = vonk ** 2
    ca = ua * shu * vk2 / ((A["aloga"] - alogu) * (A["aloga"] - A["alog1"]))
    ca = np.minimum(cdmax, ca / (1.0 + ca * 1e-20))
    rhoa = A["rhoa"]
    cai = 1.0 / (rhoa * ca)
    cbi = A["diu"] * (A["z1"] - A["z12"]) / (rhoa * 0.5 * (u1 + u12))
    cci = A["diu"] * (A["z12"] - A["z2"]) / (rhoa * 0.5 * (u12 + u2))
    cdi = (A["alog2"] - alogl) * (A["alog2"] - A["alog3"]) / (rhoa * u2 * shl * vk2)
    cei = A["dil"] * (A["z3"] - A["z34"]) / (rhoa * 0.5 * (u3 + u34))
    cfi = A["dil"] * (A["z34"] - A["z4"]) / (rhoa * 0.5 * (u34 + u4))
    T = dict(cu=1.0 / (cai + cbi), cl=1.0 / (cci + cdi + cei),
             su=rhoa * P.cleaf * np.sqrt(u12 / P.dleaf[1]),
             ss=rhoa * P.cstem * np.sqrt(u12 / P.dstem[1]),
             sl=rhoa * P.cgrass * np.sqrt(u34 / P.dleaf[0]))
    sg0 = rhoa * (0.004 + 0.012 * u4)
    si0 = rhoa * (0.003 + 0.010 * u4)
    T["sg"] = 1.0 / (cfi + 1.0 / sg0)
    T["si"] = 1.0 / (cfi + 1.0 / si0)
    carry = dict(u2=u2, alogu=alogu, alogl=alogl)
    return T, (sml, shl, smu, shu), carry


# ---------------------------------------------------------------------------
# implicit weights -- canopy_exchange.py:433-463
# ---------------------------------------------------------------------------


def weight_veg(t, ch, wliq, wsno, prev, first, P):
    if first:
        return np.ones_like(t)
    h = ch * (t - P.tmelt)
    z = np.maximum(np.abs(h), P.epsilon)
    new = np.where(h > P.epsilon + 1.0e-8, 1.0 - np.minimum(1.0, P.hfus * wsno / z),
                   np.where(h < -P.epsilon - 1.0e-8, 1.0 - np.minimum(1.0, P.hfus * wliq / z), 1.0))
    return 0.5 * (prev + new)


def weight_snow(t, told, prev, first, P):
    if first:
        return np.ones_like(t)
    dt = t - told
    warm = dt > P.epsilon + 1.0e-8
    new = np.where(warm, (P.tmelt - told) / np.where(warm, dt, 1.0), prev)
    return clip(new, 0.0, 1.0)


# ---------------------------------------------------------------------------
# stomata -- stomata.py:198-1080 (F77 branches + optional sunlit/shaded canopy)
# ---------------------------------------------------------------------------


def colimit(j1, j2, theta):
    b = j1 + j2
    c = j1 * j2
    disc = np.maximum(b * b - 4.0 * theta * c, 0.0)
    q = 0.5 * (b + np.sqrt(disc)) + 1.0e-15
    return np.minimum(q / theta, c / q)


def c3_rate(par, ci, vmax, gstar, kc, ko, rdark, P, je_fac=None, f_light=None, f_cap=None):
    """farquhar_c3 (stomata.py:228-276): je_fac scales the light-limited rate
    (acclim_light); f_light / f_cap the canopy-level co-limitation (cap_scale)."""
    je = par * 4.59e-06 * P.alpha3 * (ci - gstar) / (ci + 2.0 * gstar)
    if je_fac is not None:
        je = je * je_fac
    jc = vmax * (ci - gstar) / (ci + kc * (1.0 + P.o2conc / ko))
    js = vmax / 2.2
    if f_cap is not None:
        je, jc, js, rdark = je * f_light, jc * f_cap, js * f_cap, rdark * f_cap
    ag = colimit(colimit(je, jc, P.theta3), js, P.beta3)
    return ag, ag - rdark


def c4_rate(par, ci, vmax, rdark, P, je_fac=None, f_light=None, f_cap=None):
    """farquhar_c4 (stomata.py:279-318), with the same optional factors as c3_rate."""
    je = par * 4.59e-06 * P.alpha4
    if je_fac is not None:
        je = je * je_fac
    jc = vmax
    ji = 18.0e3 * vmax * ci
    if f_cap is not None:
        je, jc, ji, rdark = je * f_light, jc * f_cap, ji * f_cap, rdark * f_cap
    ag = colimit(colimit(je, jc, P.theta4), ji, P.beta4)
    return ag, ag - rdark


BROADLEAF_PFTS = (0, 1, 2, 4, 6)
CONIFER_PFTS = (3, 5, 7)
SHRUB_PFTS = (8, 9)


def mix_pft(frac, vp, idx, fallback, eps=1e-6):
    """_mix_vmax (stomata.py:580-590): the displayed-LAI-weighted mean of a per-PFT
    table over one big leaf's PFTs; ``fallback`` where they have no leaves."""
    ix = list(idx)
    w = frac[:, ix]
    tot = np.sum(w, axis=1)
    vpi = vp[:, ix] if vp.ndim == 2 else vp[ix][None, :]
    mixed = np.sum(w * vpi, axis=1) / np.maximum(tot, eps)
    return np.where(tot > eps, mixed, fallback)


def crop_increments(P):
    """Per-PFT ``g - 1`` per unit cropland share of crop_vfac (loops.py:218-231): the C4
    (PFT 10) and C3 (PFT 11) scales less one, or the share-mixed scale less one; the
    reference forms them on float32 masks, so they are float32 values."""
    f32 = np.float32
    q = P.crop_c4_share
    inc = np.zeros(12)
    if q < 0.0:
        inc[10] = float(f32(P.crop_vmax_scale_c4 - 1.0))
        inc[11] = float(f32(P.crop_vmax_scale_c3 - 1.0))
    else:
        qc = min(max(q, 0.0), 1.0)
        s_mix = (1.0 - qc) * P.crop_vmax_scale_c3 + qc * P.crop_vmax_scale_c4
        inc[10] = inc[11] = float(f32(s_mix - 1.0))
    return inc


def capacity_factor(S, P):
    """The per-PFT factor on vmax (None: the F77 step): temperature acclimation of the
    PFTs in acclim_pfts with the frost ramp (loops.py:291-309), then the cropland
    share's grass capacity (crop_vfac, loops.py:218-231)."""
    vfac = None
    if P.flags & FLAG_ACCLIM:
        m = np.asarray(P.acclim_mask, dtype=np.float64)[None, :]
        fs = clip((S["acclim_x"][:, None] - np.asarray(P.acclim_s0_pft)[None, :])
                  / np.asarray(P.acclim_smax_pft)[None, :], 0.0, 1.0)
        vfac = 1.0 - m + m * fs
        if P.flags & FLAG_FROST:
            ff = clip((S["td"] - 273.16 - P.frost_t0) / (P.frost_t1 - P.frost_t0), 0.0, 1.0)
            vfac = vfac * (1.0 - m + m * ff[:, None])
    if P.flags & FLAG_CROP:
        g = 1.0 + S["cropfrac"][:, None] * crop_increments(P)[None, :]
        vfac = g if vfac is None else vfac * g
    return vfac


def big_leaves(S, P):
    """Nominal vmax, light-rate factor (None: none) and Ball-Berry slope of the five big
    leaves (ub, uc, ls, l3, l4): _select_vmax_upper / _select_vmax_shrub with vmax_mix,
    acclim_light and _slopes with coefm_mix (stomata.py:592-660, 800-835)."""
    exist, frac = S["exist"], S["frac"]
    eps = P.epsilon
    vp = np.asarray(P.vmax_pft, dtype=np.float64)
    vfac = capacity_factor(S, P)
    mix = bool(P.flags & FLAG_VMAX_MIX)

    def select(v):
        col = (lambda k: v[:, k]) if v.ndim == 2 else (lambda k: v[k])
        ub = np.where(exist[:, 0] > 0.5, col(0), np.where(exist[:, 2] > 0.5, col(2), col(4)))
        uc = np.where(exist[:, 3] > 0.5, col(3), col(5))
        ls = np.broadcast_to(col(8), frac.shape[:1])
        if mix:
            ub = mix_pft(frac, v, BROADLEAF_PFTS, ub)
            uc = mix_pft(frac, v, CONIFER_PFTS, uc)
            ls = mix_pft(frac, v, SHRUB_PFTS, ls)
        return ub, uc, ls, np.broadcast_to(col(11), frac.shape[:1]), np.broadcast_to(col(10), frac.shape[:1])

    veff = vp if vfac is None else vp[None, :] * vfac
    vn = select(veff)
    je = (None,) * 5
    if (P.flags & FLAG_ACCLIM_LIGHT) and vfac is not None:
        raw = select(vp[None, :])
        je = tuple(a / np.maximum(b, eps) for a, b in zip(vn, raw))
    cm = np.asarray(P.coefm, dtype=np.float64)
    if P.flags & FLAG_COEFM_MIX:
        cp = np.asarray(P.coefm_pft, dtype=np.float64)
        n = frac.shape[0]
        slopes = (mix_pft(frac, cp, BROADLEAF_PFTS, cm[0]), mix_pft(frac, cp, CONIFER_PFTS, cm[1]),
                  mix_pft(frac, cp, SHRUB_PFTS, cm[2]), np.full(n, cp[11]), np.full(n, cp[10]))
    else:
        slopes = (cm[0], cm[1], cm[2], cm[4], cm[3])
    return vn, je, slopes


def capacity_integral(lai, kn):
    """_capacity_integral (stomata.py:370-375): (1 - e^-Kn L)/(Kn L), 0 without leaves."""
    x = kn * lai
    f = np.where(x > 1.0e-4, -np.expm1(-x) / np.maximum(x, 1.0e-4), 1.0 - 0.5 * x)
    return np.where(lai > 0.0, f, 0.0)


def kinetics(tleaf, P):
    rw = 3.47e-03 - 1.0 / tleaf
    tau = P.tau15 * np.exp(-4500.0 * rw)
    kc = P.kc15 * np.exp(6000.0 * rw)
    ko = P.ko15 * np.exp(1500.0 * rw)
    gstar = P.o2conc / (2.0 * tau)
    tc = tleaf - 273.16
    base = np.exp(3500.0 * rw)
    hot = 1.0 + np.exp(0.40 * (tc - 50.0))
    vm3 = base / ((1.0 + np.exp(0.40 * (5.0 - tc))) * hot)
    vm4 = base / ((1.0 + np.exp(0.40 * (10.0 - tc))) * hot)
    return kc, ko, gstar, vm3, vm4


def ball_berry(an, cs0, gs0, ci0, gb, rh, m, b0, stress, gmin, cmin, imin, P):
    cs = np.maximum(cmin, 0.5 * (cs0 + P.co2conc - an / gb))
    gs = 0.5 * (gs0 + m * an * rh / cs + b0 * stress)
    gs = np.maximum(gs, np.maximum(gmin, b0 * stress))
    ci = clip(0.5 * (ci0 + cs - 1.6 * an / gs), imin, P.cimax)
    return cs, gs, ci


def light_scaling(toppar, k, h, sc, lai, sai, a10s, a10d, P):
    """canopy_scaling (stomata.py:442-512): denominator k*LAI (F77) or, with
    scale_leaf_only, k*(LAI+SAI)."""
    ext = (k * sc[:, 0] + h * sc[:, 1] - h * sc[:, 2]) / np.maximum(sc[:, 3], P.epsilon)
    ext = clip(ext, 0.1, 10.0)
    pxai = ext * (lai + sai)
    plai = ext * lai
    zw = np.exp(-1.0 / (10.0 * 86400.0 / P.dtime))
    has = plai > 0.0
    day = toppar > 10.0
    denom = pxai if P.flags & FLAG_LEAF_ONLY else plai
    sday = (1.0 - np.exp(-pxai)) / np.maximum(denom, P.epsilon)
    upd = has & day
    a10s_n = np.where(upd, zw * a10s + (1.0 - zw) * sday * toppar, a10s)
    a10d_n = np.where(upd, zw * a10d + (1.0 - zw) * toppar, a10d)
    snight = a10s / np.maximum(a10d, P.epsilon)
    return np.where(has, np.where(day, sday, snight), 0.0), a10s_n, a10d_n


def _e1(a, plai):
    x = a * plai
    small = np.abs(x) < 1.0e-5
    asafe = np.where(small, 1.0, a)
    return np.where(small, plai * (1.0 - 0.5 * x), -np.expm1(-x) / asafe)


def sunshade(sc, dbeam, k, h, lai, sai, P):
    """sunshade_canopy (stomata.py:395-427)."""
    A, B, C = sc[:, 0], sc[:, 1], sc[:, 2]
    plai = np.maximum(lai + sai, P.epsilon)
    fl = np.where(lai > 0.0, lai / plai, 0.0)
    ek, e2k = _e1(k, plai), _e1(2.0 * k, plai)
    tot = np.maximum(A * ek + B * _e1(h, plai) + C * _e1(-h, plai), 0.0)
    sun = A * e2k + B * _e1(k + h, plai) + C * _e1(k - h, plai) + dbeam * (ek - e2k)
    sun = clip(sun, 0.0, tot)
    sha = tot - sun
    vs = fl * _e1(P.cap_kn * fl + k, plai)
    vh = np.maximum(fl * _e1(P.cap_kn * fl, plai) - vs, 0.0)
    return sun * fl, sha * fl, vs, vh


def _sunshade_rate(ss, lai, fn):
    ps, ph, vs, vh = ss
    ag_s, an_s = fn(ps, vs)
    ag_h, an_h = fn(ph, vh)
    inv = np.where(lai > 0.0, 1.0 / np.maximum(lai, 1.0e-6), 0.0)
    return (ag_s + ag_h) * inv, (an_s + an_h) * inv


def total_conductance(s, g):
    return 1.0 / (1.0 / s + (1.0 / 0.029) / g)


def stomata(tu, tl, t12, t34, q12, q34, su, sl, ps, R, st, fwetu, fwetl, S, stresstu, stresstl, P,
            sun_u=False, sun_l=False):
    """One stomata pass (stomata.py:732-1080). ``st`` holds the carried ci/gs/cs and a10 values."""
    eps = P.epsilon
    lai, sai = S["lai"], S["sai"]
    gam, cb, gmin = (np.asarray(P.gamma), np.asarray(P.coefb), np.asarray(P.gsmin))
    (vub, vuc, vls, vl3, vl4), (jub, juc, jls, jl3, jl4), (mub, muc, mls, ml3, ml4) = big_leaves(S, P)
    cap_u = bool(P.flags & FLAG_CAP_SCALE_U) and not sun_u
    cap_l = bool(P.flags & FLAG_CAP_SCALE_L) and not sun_l
    out = {}
    # ---- upper canopy: broadleaf (group 0) and conifer (group 1)
    kc, ko, gst, vm3, _ = kinetics(tu, P)
    gmn = 1.05 * gst
    gb = clip(su * 25.5, 0.1, 10.0)
    rh = np.maximum(0.30, q12 / np.maximum(qsat(esat(t12), ps), eps))
    if sun_u:
        ssu = sunshade(R["scalcoefu"], R["dbeamu"], R["termu6"], R["termu7"], lai[:, 1], sai[:, 1], P)
    leaves = {}
    for j, (vn, g, jf, m) in enumerate(((vub, 0, jub, mub), (vuc, 1, juc, muc))):
        ci = clip(st["ci_upper"][:, j], gmn, P.cimax)
        vmax = vn * vm3 * stresstu
        rd = gam[g] * vn * vm3
        ag, an = c3_rate(R["topparu"], ci, vmax, gst, kc, ko, rd, P, je_fac=jf)
        if sun_u:
            agc, anc = _sunshade_rate(ssu, lai[:, 1],
                                      lambda par, v: c3_rate(par, ci, vmax * v, gst, kc, ko, rd * v, P, je_fac=jf))
            bb_an = anc
        else:
            agc = anc = None
            bb_an = an
        cs, gs, ci_n = ball_berry(bb_an, st["cs_upper"][:, j], st["gs_upper"][:, j], ci, gb, rh, m, cb[g],
                                  stresstu, gmin[g], gmn, gmn, P)
        leaves[j] = (ag, an, agc, anc, cs, gs, ci_n, ci, vmax, rd, jf, m)
    scale_u, out["a10scalparamu"], out["a10daylightu"] = light_scaling(
        R["topparu"], R["termu6"], R["termu7"], R["scalcoefu"], lai[:, 1], sai[:, 1],
        st["a10scalparamu"], st["a10daylightu"], P)
    fcap_u = capacity_integral(lai[:, 1], P.cap_kn) if cap_u else None
    ag_u, an_u, tc_u = [], [], []
    for j, g in ((0, 0), (1, 1)):
        ag, an, agc, anc, cs, gs, ci_n, ci0, vmax, rd, jf, m = leaves[j]
        if cap_u:
            agc, anc = c3_rate(R["topparu"], ci0, vmax, gst, kc, ko, rd, P, je_fac=jf, f_light=scale_u, f_cap=fcap_u)
        elif not sun_u:
            agc, anc = ag * scale_u, an * scale_u
        csc = np.maximum(gmn, P.co2conc - anc / gb)
        gsc = np.maximum(np.maximum(gmin[g], cb[g] * stresstu), m * anc * rh / csc + cb[g] * stresstu)
        tc_u.append(total_conductance(su, gsc))
        ag_u.append(agc * (1.0 - fwetu))
        an_u.append(anc * (1.0 - fwetu))
    out["ci_upper"] = np.stack([leaves[0][6], leaves[1][6]], 1)
    out["gs_upper"] = np.stack([leaves[0][5], leaves[1][5]], 1)
    out["cs_upper"] = np.stack([leaves[0][4], leaves[1][4]], 1)
    out["ag_upper"] = np.stack(ag_u, 1)
    out["an_upper"] = np.stack(an_u, 1)
    out["totcondub"], out["totconduc"] = tc_u

    # ---- lower canopy: shrub (C3, group 2), C3 grass (group 4), C4 grass (group 3)
    kc, ko, gst, vm3, vm4 = kinetics(tl, P)
    gmn = 1.05 * gst
    gb = clip(sl * 25.5, 0.1, 10.0)
    rh = np.maximum(0.30, q34 / np.maximum(qsat(esat(t34), ps), eps))
    if sun_l:
        ssl = sunshade(R["scalcoefl"], R["dbeaml"], R["terml6"], R["terml7"], lai[:, 0], sai[:, 0], P)
    spec = ((0, vls, 2, False, jls, mls), (1, vl3, 4, False, jl3, ml3), (2, vl4, 3, True, jl4, ml4))
    leaves = {}
    for j, vn, g, c4, jf, m in spec:
        ci = clip(st["ci_lower"][:, j], 0.0 if c4 else gmn, P.cimax)
        vmax = vn * (vm4 if c4 else vm3) * stresstl
        rd = gam[g] * vn * (vm4 if c4 else vm3)
        if c4:
            ag, an = c4_rate(R["topparl"], ci, vmax, rd, P, je_fac=jf)
            fn = (lambda par, v, ci=ci, vmax=vmax, rd=rd, jf=jf: c4_rate(par, ci, vmax * v, rd * v, P, je_fac=jf))
        else:
            ag, an = c3_rate(R["topparl"], ci, vmax, gst, kc, ko, rd, P, je_fac=jf)
            fn = (lambda par, v, ci=ci, vmax=vmax, rd=rd, jf=jf:
                  c3_rate(par, ci, vmax * v, gst, kc, ko, rd * v, P, je_fac=jf))
        if sun_l:
            agc, anc = _sunshade_rate(ssl, lai[:, 0], fn)
            bb_an = anc
        else:
            agc = anc = None
            bb_an = an
        cs, gs, ci_n = ball_berry(bb_an, st["cs_lower"][:, j], st["gs_lower"][:, j], ci, gb, rh, m, cb[g],
                                  stresstl, gmin[g], 1.0e-8 if c4 else gmn, 0.0 if c4 else gmn, P)
        leaves[j] = (ag, an, agc, anc, cs, gs, ci_n, g, c4, ci, vmax, rd, jf, m)
    scale_l, out["a10scalparaml"], out["a10daylightl"] = light_scaling(
        R["topparl"], R["terml6"], R["terml7"], R["scalcoefl"], lai[:, 0], sai[:, 0],
        st["a10scalparaml"], st["a10daylightl"], P)
    fcap_l = capacity_integral(lai[:, 0], P.cap_kn) if cap_l else None
    ag_l, an_l, tc_l = [], [], []
    for j in range(3):
        ag, an, agc, anc, cs, gs, ci_n, g, c4, ci0, vmax, rd, jf, m = leaves[j]
        if cap_l:
            if c4:
                agc, anc = c4_rate(R["topparl"], ci0, vmax, rd, P, je_fac=jf, f_light=scale_l, f_cap=fcap_l)
            else:
                agc, anc = c3_rate(R["topparl"], ci0, vmax, gst, kc, ko, rd, P, je_fac=jf, f_light=scale_l,
                                   f_cap=fcap_l)
        elif not sun_l:
            agc, anc = ag * scale_l, an * scale_l
        csc = np.maximum(1.0e-8 if c4 else gmn, P.co2conc - anc / gb)
        gsc = np.maximum(np.maximum(gmin[g], cb[g] * stresstl), m * anc * rh / csc + cb[g] * stresstl)
        tc_l.append(total_conductance(sl, gsc))
        ag_l.append(agc * (1.0 - fwetl))
        an_l.append(anc * (1.0 - fwetl))
    out["ci_lower"] = np.stack([leaves[j][6] for j in range(3)], 1)
    out["gs_lower"] = np.stack([leaves[j][5] for j in range(3)], 1)
    out["cs_lower"] = np.stack([leaves[j][4] for j in range(3)], 1)
    out["ag_lower"] = np.stack(ag_l, 1)
    out["an_lower"] = np.stack(an_l, 1)
    out["totcondls"], out["totcondl3"], out["totcondl4"] = tc_l
    return out


# ---------------------------------------------------------------------------
# turvap -- canopy_exchange.py:26-61, 470-811
# ---------------------------------------------------------------------------


def gauss_nopivot(A, r):
    """Forward elimination without pivoting in row order, then back substitution."""
    A = A.copy()
    r = r.copy()
    n = A.shape[1]
    for p in range(n - 1):
        piv = A[:, p, p]
        for i in range(p + 1, n):
            f = A[:, i, p] / piv
            A[:, i, :] = A[:, i, :] - f[:, None] * A[:, p, :]
            r[:, i] = r[:, i] - f * r[:, p]
    x = np.zeros_like(r)
    for i in range(n - 1, -1, -1):
        s = np.zeros(r.shape[0])
        for j in range(i + 1, n):
            s = s + A[:, i, j] * x[:, j]
        x[:, i] = (r[:, i] - s) / A[:, i, i]
    return x


def turvap(W, old, T, A, X, w, I, F, S, wet, stom, R, casc, P):
    """Build and solve the 9x9 canopy system; returns new temperatures/humidities and fluxes.

    W: working temps {tu,ts,tl,t12,t34,q12,q34,tg,ti}; old: step-start {tu,ts,tl,tg,ti};
    T: transfer coefficients; A: aero geometry; X: canopy intermediates; w: implicit weights;
    I: intercepted water after the cascade; F: forcing; S: statics; soil-top inputs in X.
    """
    eps = P.epsilon
    dt = P.dtime
    ta, qa, ps = F["ta"], F["qa"], F["psurf"]
    lai, sai, frac, fu, fl, fi = S["lai"], S["sai"], S["frac"], S["fu"], S["fl"], X["fi"]
    wu, ws, wl, wg, wi = w
    tu = wu * W["tu"] + (1.0 - wu) * old["tu"]
    ts = ws * W["ts"] + (1.0 - ws) * old["ts"]
    tl = wl * W["tl"] + (1.0 - wl) * old["tl"]
    tg = wg * W["tg"] + (1.0 - wg) * old["tg"]
    ti = wi * W["ti"] + (1.0 - wi) * old["ti"]
    t12, t34, q12, q34 = W["t12"], W["t34"], W["q12"], W["q34"]

    def sat(t):
        e = esat(t)
        q = qsat(e, ps)
        return q, np.minimum(dqsat(t, q, e), q * 0.1)
    qu, dqu = sat(tu)
    qs, dqs = sat(ts)
    ql, dql = sat(tl)
    qg, dqg = sat(tg)
    qi, dqi = sat(ti)

    zwpud = clip(0.5 * (X["wpud"] + X["wipud"]) / max(P.wpudmax, eps), 0.0, 0.5)
    zwsoi = (1.0 - X["wisoi0"]) * X["wsoi0"] + X["wisoi0"]
    zwtot = zwpud + (1.0 - zwpud) * zwsoi
    psig = -P.grav * X["suction0"] * (zwtot ** (-X["bex0"]))
    hfac = np.exp(psig / (P.rvap * tg))
    hfac2 = q34 / np.maximum(qg, eps)
    betaw = clip((zwtot - X["swilt0"]) / np.maximum(1.0 - X["swilt0"], eps), 0.0, 1.0)
    if P.soil_beta_power != 1.0:
        betaw = betaw ** P.soil_beta_power
    e34 = esat(t34)
    qs1 = qsat(e34, ps)
    dqs1 = dqsat(t34, qs1)
    xden = A["cp"] + (4.0 * 0.95 * P.stef * cube(t34)) / T["sg"]
    bfac = P.hvap * dqs1 / xden
    betas = betaw / (1.0 + bfac * (1.0 - betaw))
    qgfac0 = np.where(betas > 0.0, betas * hfac + (1.0 - betas) * hfac2, hfac2)
    qeps = 1.0e-10
    qgfac = np.where(q34 > qg + qeps, 1.0, qgfac0)
    fwux = np.where(q12 > qu + qeps, 1.0, wet["fwetu"])
    fwsx = np.where(q12 > qs + qeps, 1.0, wet["fwets"])
    fwlx = np.where(q34 > ql + qeps, 1.0, wet["fwetl"])

    fradu = np.where(lai[:, 1] > eps, (R["solu"] + R["firu"]) / (2.0 * lai[:, 1]), 0.0)
    frads = np.where(sai[:, 1] > eps, (R["sols"] + R["firs"]) / (2.0 * sai[:, 1]), 0.0)
    lsl = lai[:, 0] + sai[:, 0]
    fradl = np.where(lsl > eps, (R["soll"] + R["firl"]) / (2.0 * lsl), 0.0)

    su, ss, sl, sg, si, cu, cl = T["su"], T["ss"], T["sl"], T["sg"], T["si"], T["cu"], T["cl"]
    cp = A["cp"]
    tb, tc = stom["totcondub"], stom["totconduc"]
    suw = np.minimum(fwux * su, 0.8 * (I["wliqu"] + I["wsnou"]) / np.maximum(dt * (qu - q12), eps))
    sut = np.maximum(0.0, (1.0 - fwux) * 0.5 * (
        tb * frac[:, 0] + tb * frac[:, 1] + tb * frac[:, 2] + tc * frac[:, 3]
        + tb * frac[:, 4] + tc * frac[:, 5] + tb * frac[:, 6] + tb * frac[:, 7]))
    hvu = hvapf(tu, ta, P)
    suh = suw * (wet["rliqu"] * hvu + (1.0 - wet["rliqu"]) * hsubf(tu, ta, P)) + sut * hvu
    ssw = np.minimum(fwsx * ss, 0.8 * (I["wliqs"] + I["wsnos"]) / np.maximum(dt * (qs - q12), eps))
    ssh = ssw * (wet["rliqs"] * hvapf(ts, ta, P) + (1.0 - wet["rliqs"]) * hsubf(ts, ta, P))
    slw = np.minimum(fwlx * sl, 0.8 * (I["wliql"] + I["wsnol"]) / np.maximum(dt * (ql - q34), eps))
    slt0 = np.maximum(0.0, (1.0 - fwlx) * 0.5 * (
        stom["totcondls"] * frac[:, 8] + stom["totcondls"] * frac[:, 9]
        + stom["totcondl4"] * frac[:, 10] + stom["totcondl3"] * frac[:, 11]))
    slt = slt0 * lai[:, 0] / np.maximum(lsl, eps)
    hvl = hvapf(tl, ta, P)
    slh = slw * (wet["rliql"] * hvl + (1.0 - wet["rliql"]) * hsubf(tl, ta, P)) + slt * hvl

    n = tu.size
    M = np.zeros((n, 9, 9))
    b = np.zeros((n, 9))
    rdt = 1.0 / dt
    chux, chsx, chlx = X["chux"], X["chsx"], X["chlx"]
    xu, xs, xl = X["xu"], X["xs"], X["xl"]
    r2 = su * cp
    M[:, 0, 0] = chux * rdt + wu * r2 + wu * suh * dqu
    M[:, 0, 3] = -r2
    M[:, 0, 5] = -suh
    b[:, 0] = old["tu"] * chux * rdt - (1.0 - wu) * r2 * tu - suh * (qu - wu * dqu * tu) + fradu - casc["pfluxu"]
    r2 = ss * cp
    M[:, 1, 1] = chsx * rdt + ws * r2 + ws * ssh * dqs
    M[:, 1, 3] = -r2
    M[:, 1, 5] = -ssh
    b[:, 1] = old["ts"] * chsx * rdt - (1.0 - ws) * r2 * ts - ssh * (qs - ws * dqs * ts) + frads - casc["pfluxs"]
    r2 = sl * cp
    M[:, 2, 2] = chlx * rdt + wl * r2 + wl * slh * dql
    M[:, 2, 4] = -r2
    M[:, 2, 6] = -slh
    b[:, 2] = old["tl"] * chlx * rdt - (1.0 - wl) * r2 * tl - slh * (ql - wl * dql * tl) + fradl - casc["pfluxl"]
    ru, rs = xu * su, xs * ss
    M[:, 3, 0] = -wu * ru
    M[:, 3, 1] = -ws * rs
    M[:, 3, 3] = cu + cl + ru + rs
    M[:, 3, 4] = -cl
    b[:, 3] = cu * ta * A["tfac"] + (1.0 - wu) * ru * tu + (1.0 - ws) * rs * ts
    rl, ri = xl * sl, fi * si
    M[:, 4, 2] = -wl * rl
    M[:, 4, 3] = -cl
    M[:, 4, 4] = cl + rl + (1.0 - fi) * sg + ri
    M[:, 4, 7] = -wg * (1.0 - fi) * sg
    M[:, 4, 8] = -wi * ri
    b[:, 4] = (1.0 - wl) * rl * tl + (1.0 - wg) * (1.0 - fi) * sg * tg + (1.0 - wi) * ri * ti
    ruq, rsq = xu * (suw + sut), xs * ssw
    M[:, 5, 0] = -wu * ruq * dqu
    M[:, 5, 1] = -ws * rsq * dqs
    M[:, 5, 5] = cu + cl + ruq + rsq
    M[:, 5, 6] = -cl
    b[:, 5] = cu * qa + ruq * (qu - wu * dqu * tu) + rsq * (qs - ws * dqs * ts)
    rlq, rgq = xl * (slw + slt), (1.0 - fi) * sg
    M[:, 6, 2] = -wl * rlq * dql
    M[:, 6, 5] = -cl
    M[:, 6, 6] = cl + rlq + rgq + fi * si
    M[:, 6, 7] = -wg * rgq * qgfac * dqg
    M[:, 6, 8] = -wi * fi * si * dqi
    b[:, 6] = rlq * (ql - wl * dql * tl) + rgq * qgfac * (qg - wg * dqg * tg) + fi * si * (qi - wi * dqi * ti)
    r1, r2 = sg * cp, sg * X["hvasug"]
    M[:, 7, 4] = -r1
    M[:, 7, 6] = -r2
    M[:, 7, 7] = r1 + r2 * qgfac * dqg + X["cog"] + X["zirg"]
    b[:, 7] = -r2 * qgfac * (qg - dqg * tg) + X["cog"] * X["tsoi0"] + R["solg"] + R["firg"] + X["zirg"] * old["tg"]
    r1, r2 = si * cp, si * X["hvasui"]
    M[:, 8, 4] = -r1
    M[:, 8, 6] = -r2
    M[:, 8, 8] = r1 + r2 * dqi + X["coi"] + X["ziri"]
    b[:, 8] = -r2 * (qi - dqi * ti) + X["coi"] * X["tsno0"] + R["soli"] + R["firi"] + X["ziri"] * old["ti"]

    # bare cells: canopy rows become identity rows pinned to the air (canopy_exchange.py:684-732)
    bare = (xu + xs + xl) < eps
    if np.any(bare):
        Mb = M[bare]
        Mb[:, :7, :] = 0.0
        for r in range(7):
            Mb[:, r, r] = 1.0
        Mb[:, 7, 3] = 0.0
        Mb[:, 7, 5] = 0.0
        Mb[:, 8, 3] = 0.0
        Mb[:, 8, 5] = 0.0
        M[bare] = Mb
        ttf = ta * A["tfac"]
        bb = b[bare]
        for r in range(5):
            bb[:, r] = ttf[bare]
        bb[:, 5] = qa[bare]
        bb[:, 6] = qa[bare]
        red = ((fradu - casc["pfluxu"]) * xu + (frads - casc["pfluxs"]) * xs + (fradl - casc["pfluxl"]) * xl)
        bb[:, 7] = bb[:, 7] + red[bare]
        b[bare] = bb

    v = gauss_nopivot(M, b)
    nu, ns, nl, n12, n34, nq12, nq34, ng, ni = (v[:, i] for i in range(9))
    o = dict(tu=nu, ts=ns, tl=nl, t12=n12, t34=n34, q12=nq12, q34=nq34, tg=ng, ti=ni)
    o["fsena"] = cp * cu * (ta * A["tfac"] - n12)
    o["fsenu"] = cp * su * (wu * nu + (1.0 - wu) * tu - n12)
    o["fsens"] = cp * ss * (ws * ns + (1.0 - ws) * ts - n12)
    o["fsenl"] = cp * sl * (wl * nl + (1.0 - wl) * tl - n12)
    o["fseng"] = cp * sg * (wg * ng + (1.0 - wg) * tg - n34)
    o["fseni"] = cp * si * (wi * ni + (1.0 - wi) * ti - n34)
    quav = qu + wu * dqu * (nu - tu)
    o["fvapuw"] = suw * (quav - nq12)
    o["fvaput"] = np.maximum(0.0, sut * (quav - nq12))
    o["fvaps"] = ssw * (qs + ws * dqs * (ns - ts) - nq12)
    qlav = ql + wl * dql * (nl - tl)
    o["fvaplw"] = slw * (qlav - nq34)
    o["fvaplt"] = np.maximum(0.0, slt0 * (qlav - nq34))
    o["fvapg"] = sg * (qgfac * (qg + wg * dqg * (ng - tg)) - nq34)
    o["fvapi"] = si * (qi + wi * dqi * (ni - ti) - nq34)
    o["firg"] = R["firg"] - wg * X["zirg"] * (ng - old["tg"])
    o["firi"] = R["firi"] - wi * X["ziri"] * (ni - old["ti"])
    o["firb"] = R["firb"] + (1.0 - fi) * wg * X["zirg"] * (ng - old["tg"]) + fi * wi * X["ziri"] * (ni - old["ti"])
    o["ginvap"] = o["fvapuw"] * xu + o["fvaps"] * xs + o["fvaplw"] * xl
    o["gsuvap"] = o["fvapg"] * (1.0 - fi) + o["fvapi"] * fi
    o["gtrans"] = o["fvaput"] * 2.0 * lai[:, 1] * fu + o["fvaplt"] * 2.0 * lai[:, 0] * fl * (1.0 - fi)
    return o
