"""Column physics of the IBIS hourly step, restated in float64 NumPy.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).  Every routine works on
arrays whose first axis is the cell; layer arrays are (ncell, nlayer).
Operation orders follow the reference where it documents that the order
matters (no-pivot Gauss, total conductance, integer powers).
"""
from __future__ import annotations

import numpy as np

# IBIS 3.0 extensions of the step, as carried in ``P.flags`` (the values of
# ibis_b200.params.FLAG_*; off = the F77 step)
FLAG_VMAX_MIX = 1 << 12
FLAG_COEFM_MIX = 1 << 13
FLAG_GPP_CAPACITY = 1 << 14
FLAG_ACCLIM = 1 << 15
FLAG_ACCLIM_LIGHT = 1 << 16
FLAG_FROST = 1 << 17
FLAG_CAP_SCALE_U = 1 << 18
FLAG_CAP_SCALE_L = 1 << 19
FLAG_LEAF_ONLY = 1 << 20
FLAG_CROP = 1 << 21
FLAG_FORGANIC = 1 << 22

# ---------------------------------------------------------------------------
# small helpers
# ---------------------------------------------------------------------------


def clip(x, lo, hi):
    return np.minimum(np.maximum(x, lo), hi)


def cube(x):
    """x**3 evaluated as XLA evaluates an integer power: x * (x * x)."""
    return x * (x * x)


def quart(x):
    """x**4 as (x * x) * (x * x)."""
    x2 = x * x
    return x2 * x2


# ---------------------------------------------------------------------------
# thermodynamics -- python-port/ibis/physics/thermo.py:38-224 (Lowe 1977)
# ---------------------------------------------------------------------------
_LIQ_E = (6.1078000, 4.4365185e-1, 1.4289458e-2, 2.6506485e-4, 3.0312404e-6, 2.0340809e-8, 6.1368209e-11)
_ICE_E = (6.1091780, 5.0346990e-1, 1.8860134e-2, 4.1762237e-4, 5.8247203e-6, 4.8388032e-8, 1.8388269e-10)
_LIQ_D = (4.4381000e-1, 2.8570026e-2, 7.9380540e-4, 1.2152151e-5, 1.0365614e-7, 3.5324218e-10, -7.0902448e-13)
_ICE_D = (5.0303052e-1, 3.7732550e-2, 1.2679954e-3, 2.4775631e-5, 3.0056931e-7, 2.1585425e-9, 7.1310977e-12)


def _lowe(t, liq, ice):
    """Both Lowe branches evaluated on clamped offsets (thermo.py:65-97)."""
    dl = clip(t - 273.16, 0.0, 100.0)
    di = clip(t - 273.16, -60.0, 0.0)
    base = np.where(t >= 273.16, liq[0], ice[0])
    pl = dl * (liq[1] + dl * (liq[2] + dl * (liq[3] + dl * (liq[4] + dl * (liq[5] + dl * liq[6])))))
    pi = di * (ice[1] + di * (ice[2] + di * (ice[3] + di * (ice[4] + di * (ice[5] + di * ice[6])))))
    return 100.0 * (base + pl + pi)


def esat(t):
    return _lowe(t, _LIQ_E, _ICE_E)


def desat(t):
    return _lowe(t, _LIQ_D, _ICE_D)


def qsat(e, p):
    """thermo.py:129-149."""
    return 0.622 * e / np.maximum(p - (1.0 - 0.622) * e, 0.622 * e)


def dqsat(t, q, e=None):
    """thermo.py:152-174."""
    if e is None:
        e = esat(t)
    return desat(t) * q * (1.0 + q * (1.0 / 0.622 - 1.0)) / e


def hvapf(t, tair, P):
    """thermo.py:177-199."""
    return P.hvap + P.cvap * (tair - P.tmelt) - P.ch2o * (t - P.tmelt)


def hsubf(t, tair, P):
    """thermo.py:202-224."""
    return P.hsub + P.cvap * (tair - P.tmelt) - P.cice * (t - P.tmelt)


# ---------------------------------------------------------------------------
# tridiagonal solve -- python-port/ibis/physics/solvers.py:17-83
# ---------------------------------------------------------------------------


def thomas(lo, di, up, r):
    """Thomas algorithm over the last axis (lo[:,0] and up[:,-1] unused)."""
    n = di.shape[1]
    gam = np.empty_like(di)
    x = np.empty_like(di)
    alp = 1.0 / di[:, 0]
    gam[:, 0] = up[:, 0] * alp
    x[:, 0] = r[:, 0] * alp
    for k in range(1, n - 1):
        alp = 1.0 / (di[:, k] - lo[:, k] * gam[:, k - 1])
        gam[:, k] = up[:, k] * alp
        x[:, k] = (r[:, k] - lo[:, k] * x[:, k - 1]) * alp
    k = n - 1
    x[:, k] = (r[:, k] - lo[:, k] * x[:, k - 1]) / (di[:, k] - lo[:, k] * gam[:, k - 1])
    for k in range(n - 2, -1, -1):
        x[:, k] = x[:, k] - gam[:, k] * x[:, k + 1]
    return x


# ---------------------------------------------------------------------------
# setsoi -- python-port/ibis/physics/soil_physics.py:37-140
# ---------------------------------------------------------------------------


def setsoi(S, prog, tsno0, ta, P):
    poros, wsoi, wisoi, tsoi = S["poros"], prog["wsoi"], prog["wisoi"], prog["tsoi"]
    fs = 0.01 * S["sand"]
    fc = 0.01 * S["clay"]
    fsilt = 1.0 - fs - fc
    pliq = poros * wsoi * (1.0 - wisoi)
    pice = poros * wisoi
    dry = fs * 0.300 + fsilt * 0.265 + fc * 0.250
    if P.flags & FLAG_FORGANIC:                 # organic solids (soil_physics.py:74-77)
        fo = S["forganic"]
        dry = (1.0 - fo) * dry + fo * 0.05
    consoi = dry * (56.0 ** pliq) * (224.0 ** pice)

    wpud, wipud = prog["wpud"], prog["wipud"]
    pud = wpud + wipud
    zwpud = clip(P.zwpmax * pud / max(P.wpudmax, P.epsilon), 0.0, P.zwpmax)
    w0, i0 = wsoi[:, 0], wisoi[:, 0]
    zwsoi = (1.0 - i0) * w0 + i0
    soilw = zwsoi >= P.epsilon
    haspud = zwpud >= P.epsilon
    r1 = 1.0 / np.maximum(zwsoi, P.epsilon)
    r2 = 1.0 / np.maximum(pud, P.epsilon)
    q1 = np.where(soilw, np.where(haspud, (1.0 - zwpud) * (1.0 - i0) * w0 * r1, (1.0 - i0) * w0 * r1), 0.0)
    q2 = np.where(soilw, np.where(haspud, (1.0 - zwpud) * i0 * r1, i0 * r1), 0.0)
    warm = tsoi[:, 0] >= P.tmelt - 1.0e-9
    q3 = np.where(haspud, zwpud * wpud * r2, np.where(soilw, 0.0, np.where(warm, 1.0, 0.0)))
    q4 = np.where(haspud, zwpud * wipud * r2, np.where(soilw, 0.0, np.where(warm, 0.0, 1.0)))
    qglif = np.stack([q1, q2, q3, q4], axis=1)
    zvap = hvapf(tsoi[:, 0], ta, P)
    zsub = hsubf(tsoi[:, 0], ta, P)
    hvasug = (q1 + q3) * zvap + (q2 + q4) * zsub
    hvasui = hsubf(tsno0, ta, P)
    return consoi, qglif, hvasug, hvasui


# ---------------------------------------------------------------------------
# interception -- python-port/ibis/physics/interception.py
# ---------------------------------------------------------------------------


def wet_fraction(tveg, wliq, wsno, wliqmax, wsnomax, P):
    """One surface of fwetcal (interception.py:62-94)."""
    xliq = wliq / max(wliqmax, 0.01)
    xtot = xliq + wsno / max(wsnomax, 0.01)
    fwet = np.minimum(P.fmax, xtot)
    rliq = xliq / np.maximum(xtot, P.epsilon)
    rliq = np.where(fwet == 0.0, np.where(tveg < P.tmelt - 1.0e-9, 0.0, 1.0), rliq)
    return fwet, rliq


def fwetcal(tu, ts, tl, w, P):
    fu, ru = wet_fraction(tu, w["wliqu"], w["wsnou"], P.wliqumax, P.wsnoumax, P)
    fs, rs = wet_fraction(ts, w["wliqs"], w["wsnos"], P.wliqsmax, P.wsnosmax, P)
    fl, rl = wet_fraction(tl, w["wliql"], w["wsnol"], P.wliqlmax, P.wsnolmax, P)
    return dict(fwetu=fu, fwets=fs, fwetl=fl, rliqu=ru, rliqs=rs, rliql=rl)


def mix3(x1, t1, x2, t2, x3, t3, eps):
    """Calorimetric mix (interception.py:101-123)."""
    xm = x1 + x2 + x3
    ok = np.abs(xm) >= eps
    den = np.where(ok, xm, 1.0)
    tm = np.where(ok, (t1 * x1 + t2 * x2 + t3 * x3) / den, 0.0)
    return np.where(ok, xm, 0.0), tm


def wet_bulb(tak, q, p, P):
    """twet3: 20 relaxation sweeps latched at |step| < 0.02 K (interception.py:126-171)."""
    qs0 = qsat(esat(tak), p)
    ta = tak - P.tmelt
    twk = ta * q / np.maximum(qs0, 1e-12) + P.tmelt
    done = np.zeros(twk.shape, dtype=bool)
    for _ in range(20):
        twold = twk - P.tmelt
        hv = hvapf(twk, tak, P)
        qw = qsat(esat(twk), p)
        twb = ta - (hv / P.cair) * (qw - q)
        nxt = twold + 0.2 * (twb - twold) + P.tmelt
        conv = np.abs(nxt - P.tmelt - twold) < 0.02
        twk = np.where(done, twk, nxt)
        done = done | conv
    return twk


def intercept(tveg, wliq, wsno, xai, rain, train, snow, tsnow, tdrip, tblow,
              wliqmax, wsnomax, wliqmin, wsnomin, P):
    """steph2o for one surface (interception.py:174-260); returns wliq, wsno, pflux, rain, train, snow, tsnow."""
    dt = P.dtime
    fint = np.where(xai >= P.epsilon, (1.0 - np.exp(-0.5 * xai)) / xai, 0.5)
    rdt = 1.0 / dt
    drip = xai * wliq / tdrip
    wliq = wliq * (1.0 - dt / tdrip)
    wliq = wliq + dt * rain * fint
    pflux = rain * fint * (tveg - train) * P.ch2o
    rain = rain * (1.0 - xai * fint)
    x = wliq
    wliq = np.minimum(wliq, wliqmax)
    wliq = np.where(wliq < wliqmin, 0.0, wliq)
    drip = drip + xai * (x - wliq) * rdt

    blow = xai * wsno / tblow
    wsno = wsno * (1.0 - dt / tblow)
    wsno = wsno + dt * snow * fint
    pflux = pflux + snow * fint * (tveg - tsnow) * P.cice
    snow = snow * (1.0 - xai * fint)
    x = wsno
    wsno = np.minimum(wsno, wsnomax)
    wsno = np.where(wsno < wsnomin, 0.0, wsno)
    blow = blow + xai * (x - wsno) * rdt

    dcp = P.ch2o - P.cice
    dfrz = np.where(tveg < P.tmelt - 1.0e-9, wliq, 0.0)
    pflux = pflux + dfrz * (dcp * (P.tmelt - tveg) - P.hfus) * rdt
    wliq = wliq - dfrz
    wsno = wsno + dfrz
    dmlt = np.where(tveg > P.tmelt + 1.0e-9, wsno, 0.0)
    pflux = pflux + dmlt * (dcp * (tveg - P.tmelt) + P.hfus) * rdt
    wsno = wsno - dmlt
    wliq = wliq + dmlt
    z = np.zeros_like(rain)
    rain, train = mix3(rain, train, drip, tveg, z, z, P.epsilon)
    snow, tsnow = mix3(snow, tsnow, blow, tveg, z, z, P.epsilon)
    return wliq, wsno, pflux, rain, train, snow, tsnow


def cascade(prog, S, F, P):
    """Precipitation through the two canopy stories (interception.py:263-357)."""
    tu, ts, tl, t12, t34 = prog["tu"], prog["ts"], prog["tl"], prog["t12"], prog["t34"]
    lai, sai, fu, fl = S["lai"], S["sai"], S["fu"], S["fl"]
    ta, qa, ps = F["ta"], F["qa"], F["psurf"]
    z = np.zeros_like(tu)
    wliqmin = 0.001 * (P.dtime / 3600.0) * (P.wliqumax / 0.2)
    wsnomin = 0.001 * (P.dtime / 3600.0) * (P.wsnoumax / 2.0)
    tw = np.where(ta > P.tmelt + 1.0e-9, wet_bulb(ta, qa, ps, P), P.tmelt)
    rainu, trainu = mix3(F["raina"], np.maximum(tw, P.tmelt), z, np.maximum(t12, P.tmelt), z, z, P.epsilon)
    snowu, tsnowu = mix3(F["snowa"], np.minimum(ta, P.tmelt), z, np.minimum(t12, P.tmelt), z, z, P.epsilon)

    wu, su_, pu, rain, train, snow, tsnow = intercept(
        tu, prog["wliqu"], prog["wsnou"], 2.0 * lai[:, 1], rainu, trainu, snowu, tsnowu,
        P.tdripu, P.tblowu, P.wliqumax, P.wsnoumax, wliqmin, wsnomin, P)
    ws, ss_, ps_, rain, train, snow, tsnow = intercept(
        ts, prog["wliqs"], prog["wsnos"], 2.0 * sai[:, 1], rain, train, snow, tsnow,
        P.tdrips, P.tblows, P.wliqsmax, P.wsnosmax, wliqmin, wsnomin, P)
    rainl, trainl = mix3(fu * rain, train, (1.0 - fu) * rainu, trainu, z, np.maximum(t34, P.tmelt), P.epsilon)
    snowl, tsnowl = mix3(fu * snow, tsnow, (1.0 - fu) * snowu, tsnowu, z, np.minimum(t34, P.tmelt), P.epsilon)
    wl, sl_, pl, rain3, train3, snow3, tsnow3 = intercept(
        tl, prog["wliql"], prog["wsnol"], 2.0 * (lai[:, 0] + sai[:, 0]), rainl, trainl, snowl, tsnowl,
        P.tdripl, P.tblowl, P.wliqlmax, P.wsnolmax, wliqmin, wsnomin, P)
    raing, traing = mix3(fl * rain3, train3, (1.0 - fl) * rainl, trainl, z, z, P.epsilon)
    snowg, tsnowg = mix3(fl * snow3, tsnow3, (1.0 - fl) * snowl, tsnowl, z, z, P.epsilon)
    return dict(wliqu=wu, wliqs=ws, wliql=wl, wsnou=su_, wsnos=ss_, wsnol=sl_,
                pfluxu=pu, pfluxs=ps_, pfluxl=pl, raing=raing, traing=traing,
                snowg=snowg, tsnowg=tsnowg, rainl=rainl, trainl=trainl, snowl=snowl, tsnowl=tsnowl)


def evap_intercepted(tveg, wliq, wsno, rliq, fvapw, cveg, P):
    """steph2o2 minus its discarded fvapa/fsena outputs (interception.py:364-416)."""
    dt = P.dtime
    wliq = wliq - dt * rliq * fvapw
    wsno = wsno - dt * (1.0 - rliq) * fvapw
    wliq = np.maximum(wliq, 0.0)
    wsno = np.maximum(wsno, 0.0)
    rh = 1.0 / P.hfus
    chav = cveg + P.ch2o * wliq + P.cice * wsno
    cold = (tveg < P.tmelt - 1.0e-9) & (wliq > 0.0)
    dh = chav * (P.tmelt - tveg)
    dw = np.where(cold, np.minimum(wliq, np.maximum(0.0, dh * rh)), 0.0)
    wliq = wliq - dw
    wsno = wsno + dw
    chn = cveg + P.ch2o * wliq + P.cice * wsno
    tveg = np.where(cold, P.tmelt - (dh - P.hfus * dw) / chn, tveg)
    warm = (tveg > P.tmelt + 1.0e-9) & (wsno > 0.0)
    chav = cveg + P.ch2o * wliq + P.cice * wsno
    dh = chav * (tveg - P.tmelt)
    dw = np.where(warm, np.minimum(wsno, np.maximum(0.0, dh * rh)), 0.0)
    wsno = wsno - dw
    wliq = wliq + dw
    chn = cveg + P.ch2o * wliq + P.cice * wsno
    tveg = np.where(warm, P.tmelt + (dh - P.hfus * dw) / chn, tveg)
    return tveg, wliq, wsno


# ---------------------------------------------------------------------------
# radiation -- python-port/ibis/physics/radiation.py
# ---------------------------------------------------------------------------


def optics(coszen, lai, sai, fwet, rliq, tveg, rho, tau, ov, oh, osno, sun, P, stem=None):
    """twoset (radiation.py:75-177); ``stem`` = (fwet, rliq, t) of the upper stems."""
    orand = 1.0 - ov - oh
    om0 = rho + tau
    ztab = 0.5 - coszen / 3.0
    rw = 1.0 / max(om0, 1e-12)
    betad = (ov * 0.5 * (rho + tau) + oh * rho + orand * ((1.0 - ztab) * rho + ztab * tau)) * rw
    betai = (ov * 0.5 * (rho + tau) + oh * rho + orand * ((2.0 / 3.0) * rho + (1.0 / 3.0) * tau)) * rw
    gdir = ov * (2.0 / 3.1415927) * np.sqrt(np.maximum(0.0, 1.0 - coszen * coszen)) + oh * coszen + orand * 0.5
    if stem is not None:
        fws, rls, tst = stem
        xu = lai / np.maximum(lai + sai, 1e-7)
        y = xu * (fwet * (1.0 - rliq)) + (1.0 - xu) * (fws * (1.0 - rls))
        o = (xu * clip((P.tmelt - tveg) / 0.1, 0.6, 1.0) + (1.0 - xu) * clip((P.tmelt - tst) / 0.1, 0.6, 1.0)) * osno
    else:
        y = fwet * (1.0 - rliq)
        o = osno * (0.6 + 0.4 * clip((P.tmelt - tveg) / 1.0, 0.0, 1.0))
    ys = y * o
    om = np.maximum((1.0 - y) * om0 + ys, 1e-12)
    betad = ((1.0 - y) * om0 * betad + ys * 0.5) / om
    betai = ((1.0 - y) * om0 * betai + ys * 0.5) / om
    return (np.where(sun, om, 0.0), np.where(sun, betad, 0.0), np.where(sun, betai, 0.0),
            np.where(sun, 1.0, 1.0), np.where(sun, gdir, 0.0))


def two_stream(coszen, lai, sai, asd, asi, om, betad, betai, avmu, gdir, sun, vis, P):
    """twostr (radiation.py:180-313): returns dict of absorbed/reflected/transmitted fractions."""
    eps = P.epsilon
    b = 1.0 - om * (1.0 - betai)
    c = om * betai
    t0 = b * b - c * c
    q = np.sqrt(np.maximum(0.0, t0))
    k = gdir / np.maximum(coszen, 0.01)
    p = avmu * k
    sgn = np.where(p >= q, 1.0, -1.0)
    p = np.where(np.abs(p - q) < 0.001 * p, (1.0 + sgn * 0.001) * p, p)
    c0 = om * p
    d = c0 * betad
    f = c0 * (1.0 - betad)
    h = q / avmu
    sigma = p * p - t0
    ud1 = b - c / np.maximum(asd, 1e-12)
    ui1 = b - c / np.maximum(asi, 1e-12)
    ud2 = b - c * asd
    ui2 = b - c * asi
    ud3 = f + c * asd
    xai = np.maximum(lai + sai, eps)
    s1 = np.exp(-h * xai)
    s2 = np.exp(-k * xai)
    p1, p2, p3, p4 = b + q, b - q, b + p, b - p
    s1m = np.maximum(s1, 1e-30)
    rw = 1.0 / s1m
    dd1 = p1 * (ud1 - q) * rw - p2 * (ud1 + q) * s1
    di1 = p1 * (ui1 - q) * rw - p2 * (ui1 + q) * s1
    dd2 = (ud2 + q) * rw - (ud2 - q) * s1
    di2 = (ui2 + q) * rw - (ui2 - q) * s1
    tiny = lambda v: np.where(np.abs(v) < 1e-30, 1e-30, v)
    dd1, di1, dd2, di2, sigma = tiny(dd1), tiny(di1), tiny(dd2), tiny(di2), tiny(sigma)
    h1 = -d * p4 - c * f
    rw2 = s2 * (d - c - h1 * (ud1 + p) / sigma)
    h2 = (1.0 / dd1) * ((d - h1 * p3 / sigma) * (ud1 - q) / s1m - p2 * rw2)
    h3 = -(1.0 / dd1) * ((d - h1 * p3 / sigma) * (ud1 + q) * s1 - p1 * rw2)
    h4 = -f * p3 - c * d
    rw3 = s2 * (ud3 - h4 * (ud2 - p) / sigma)
    h5 = -(1.0 / dd2) * (h4 * (ud2 + q) / (sigma * s1m) + rw3)
    h6 = (1.0 / dd2) * (h4 * s1 * (ud2 - q) / sigma + rw3)
    h7 = c * (ui1 - q) / (di1 * s1m)
    h8 = -c * s1 * (ui1 + q) / di1
    h9 = (ui2 + q) / (di2 * s1m)
    h10 = -s1 * (ui2 - q) / di2
    fbeldd = s2
    fbelid = h4 / sigma * s2 + h5 * s1 + h6 / s1m
    fbelii = h9 * s1 + h10 / s1m
    refld = h1 / sigma + h2 + h3
    refli = h7 + h8
    absurd = (1.0 - asd) * fbeldd + (1.0 - asi) * fbelid
    absuri = (1.0 - asi) * fbelii
    abvegd = np.maximum(0.0, 1.0 - refld - absurd)
    abvegi = np.maximum(0.0, 1.0 - refli - absuri)
    noveg = xai < eps
    abvegd = np.where(noveg, 0.0, abvegd)
    abvegi = np.where(noveg, 0.0, abvegi)
    out = dict(abvegd=np.where(sun, abvegd, 0.0), abvegi=np.where(sun, abvegi, 0.0),
               refld=np.where(sun, refld, 0.0), refli=np.where(sun, refli, 0.0),
               fbeldd=np.where(sun, fbeldd, 0.0), fbelid=np.where(sun, fbelid, 0.0),
               fbelii=np.where(sun, fbelii, 0.0), om=om)
    if vis:
        out["term"] = (k * (1.0 + (h4 - h1) / sigma), h * (h5 - h2), h * (h9 - h7),
                       h * (h3 - h6), h * (h8 - h10), k, h)
    return out


def radiation(prog, S, F, wet, P):
    """compute_radiation = solsur + solalb + solarf per band, then irrad (radiation.py:316-761)."""
    coszen = F["coszen"]
    sun = coszen > 0.0
    lai, sai, fu, fl = S["lai"], S["sai"], S["fu"], S["fl"]
    fi = prog["fi"]
    tu, ts, tl = prog["tu"], prog["ts"], prog["tl"]
    eps = P.epsilon
    rhoveg = np.asarray(P.rhoveg).reshape(2, 2)
    tauveg = np.asarray(P.tauveg).reshape(2, 2)
    z = np.zeros_like(coszen)
    R = dict(solu=z.copy(), sols=z.copy(), soll=z.copy(), solg=z.copy(), soli=z.copy(),
             asurd=np.zeros((coszen.size, 2)), asuri=np.zeros((coszen.size, 2)),
             topparu=z.copy(), topparl=z.copy(), scalcoefu=np.zeros((coszen.size, 4)),
             scalcoefl=np.zeros((coszen.size, 4)), dbeamu=z.copy(), dbeaml=z.copy())
    w0 = prog["wsoi"][:, 0]
    i0 = prog["wisoi"][:, 0]
    tsno0 = prog["tsno"][:, 0]
    for ib in range(2):
        # solsur (radiation.py:316-369)
        zw = w0 * (1.0 - i0)
        dinc = 1.0 + clip(1.0 - zw / 0.50, 0.0, 1.0)
        albsod = np.minimum((S["albsav"] if ib == 0 else S["albsan"]) * dinc, 0.80)
        albsoi = albsod
        ahi, alo = (0.70, 0.90) if ib == 0 else (0.40, 0.60)
        x = (ahi * (tsno0 - (P.tmelt - 15.0)) + alo * (P.tmelt - tsno0)) / (P.tmelt - (P.tmelt - 15.0))
        x = clip(x, ahi, alo)
        zfac = np.maximum(0.0, 1.5 / (1.0 + 4.0 * coszen) - 0.5)
        albsnd = np.minimum(0.99, x + (1.0 - x) * zfac)
        albsni = np.minimum(1.0, x)
        albsod, albsoi = np.where(sun, albsod, 0.0), np.where(sun, albsoi, 0.0)
        albsnd, albsni = np.where(sun, albsnd, 0.0), np.where(sun, albsni, 0.0)
        # solalb (radiation.py:372-447)
        o = optics(coszen, lai[:, 0], sai[:, 0], wet["fwetl"], wet["rliql"], tl,
                   rhoveg[ib, 0], tauveg[ib, 0], P.oriev[0], P.orieh[0], P.omegasno[ib], sun, P)
        lo = two_stream(coszen, lai[:, 0], sai[:, 0], albsod, albsoi, *o, sun, ib == 0, P)
        asd = fl * (1.0 - fi) * lo["refld"] + (1.0 - fl) * (1.0 - fi) * albsod + fi * albsnd
        asi = fl * (1.0 - fi) * lo["refli"] + (1.0 - fl) * (1.0 - fi) * albsoi + fi * albsni
        o = optics(coszen, lai[:, 1], sai[:, 1], wet["fwetu"], wet["rliqu"], tu,
                   rhoveg[ib, 1], tauveg[ib, 1], P.oriev[1], P.orieh[1], P.omegasno[ib], sun, P,
                   stem=(wet["fwets"], wet["rliqs"], ts))
        up = two_stream(coszen, lai[:, 1], sai[:, 1], asd, asi, *o, sun, ib == 0, P)
        R["asurd"][:, ib] = np.where(sun, fu * up["refld"] + (1.0 - fu) * asd, 0.0)
        R["asuri"][:, ib] = np.where(sun, fu * up["refli"] + (1.0 - fu) * asi, 0.0)
        # solarf (radiation.py:450-540)
        sd, si = F["solad"][:, ib], F["solai"][:, ib]
        x = sd * up["abvegd"] + si * up["abvegi"]
        y = lai[:, 1] / np.maximum(lai[:, 1] + sai[:, 1], eps)
        solu = x * y
        sols = x * (1.0 - y)
        s2d = sd * up["fbeldd"]
        s2i = sd * up["fbelid"] + si * up["fbelii"]
        s3d = fu * s2d + (1.0 - fu) * sd
        s3i = fu * s2i + (1.0 - fu) * si
        soll = s3d * lo["abvegd"] + s3i * lo["abvegi"]
        xd = (fl * lo["fbeldd"] + 1.0 - fl) * s3d
        xi = fl * (s3d * lo["fbelid"] + s3i * lo["fbelii"]) + (1.0 - fl) * s3i
        solg = (1.0 - albsod) * xd + (1.0 - albsoi) * xi
        soli = (1.0 - albsnd) * s3d + (1.0 - albsni) * s3i
        if ib == 0:
            tu_ = up["term"]
            c0 = tu_[0] * sd
            c1 = tu_[1] * sd + tu_[2] * si
            c2 = tu_[3] * sd + tu_[4] * si
            c3 = c0 + c1 + c2
            R["scalcoefu"] = np.stack([c0, c1, c2, c3], axis=1)
            R["topparu"] = c3 * lai[:, 1] / np.maximum(lai[:, 1] + sai[:, 1], eps)
            R["dbeamu"] = (1.0 - up["om"]) * tu_[5] * sd
            tl_ = lo["term"]
            c0 = tl_[0] * s3d
            c1 = tl_[1] * s3d + tl_[2] * s3i
            c2 = tl_[3] * s3d + tl_[4] * s3i
            c3 = c0 + c1 + c2
            R["scalcoefl"] = np.stack([c0, c1, c2, c3], axis=1)
            R["topparl"] = c3 * lai[:, 0] / np.maximum(lai[:, 0] + sai[:, 0], eps)
            R["dbeaml"] = (1.0 - lo["om"]) * tl_[5] * s3d
            R["termu6"], R["termu7"] = tu_[5], tu_[6]
            R["terml6"], R["terml7"] = tl_[5], tl_[6]
        R["solu"] = R["solu"] + np.where(sun, solu, 0.0)
        R["sols"] = R["sols"] + np.where(sun, sols, 0.0)
        R["soll"] = R["soll"] + np.where(sun, soll, 0.0)
        R["solg"] = R["solg"] + np.where(sun, solg, 0.0)
        R["soli"] = R["soli"] + np.where(sun, soli, 0.0)
    # irrad (radiation.py:543-641)
    emu = 1.0 - np.exp(-lai[:, 1] / 1.0)
    ems = 1.0 - np.exp(-sai[:, 1] / 1.0)
    eml = 1.0 - np.exp(-(lai[:, 0] + sai[:, 0]) / 1.0)
    emg = emi = 0.95
    fira = F["fira"]
    tu4 = P.stef * quart(tu)
    ts4 = P.stef * quart(ts)
    tl4 = P.stef * quart(tl)
    tg4 = P.stef * quart(prog["tg"])
    ti4 = P.stef * quart(prog["ti"])
    fdown = (1.0 - fu) * fira + fu * ((1.0 - emu) * (1.0 - ems) * fira + emu * (1.0 - ems) * tu4 + ems * ts4)
    fdowng = (1.0 - eml) * fdown + eml * tl4
    fupg = (1.0 - emg) * fdowng + emg * tg4
    fupgb = (1.0 - emg) * fdown + emg * tg4
    fupi = (1.0 - emi) * fdown + emi * ti4
    fup = (1.0 - fi) * (fl * (eml * tl4 + (1.0 - eml) * fupg) + (1.0 - fl) * fupgb) + fi * fupi
    R["firb"] = (1.0 - fu) * fup + fu * ((1.0 - emu) * (1.0 - ems) * fup + emu * tu4 + ems * (1.0 - emu) * ts4)
    R["firu"] = emu * ems * ts4 + emu * (1.0 - ems) * fup + emu * fira - 2.0 * emu * tu4
    R["firs"] = ems * emu * tu4 + ems * fup + ems * (1.0 - emu) * fira - 2.0 * ems * ts4
    R["firl"] = eml * fdown + eml * fupg - 2.0 * eml * tl4
    R["firg"] = fl * (fdowng - fupg) + (1.0 - fl) * (fdown - fupgb)
    R["firi"] = fdown - fupi
    return R
