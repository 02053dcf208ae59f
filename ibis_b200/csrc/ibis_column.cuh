// One hourly step of the IBIS 3.0 land-surface column, one cell per thread.
//
// This is the device implementation of the reference's `timestep_body`
// (python-port/ibis/timestepping/loops.py:234-1284) and of the per-step
// accumulators and wetland CH4 of `_run_day_inner._step_body`
// (python-port/ibis/timestepping/loops_gswp3.py:161-318).  Each block cites
// the reference lines it implements.
//
// Precision: R is the bulk type.  The 9x9 canopy energy/vapour system of
// `turvap` (assembly, elimination and the flux diagnostics) and the soil-water
// tridiagonal solve of `soilh2o` are always evaluated in double; everything else
// runs in R.  With R = double the kernel is a float64 run of the whole step.
#pragma once
#include "ibis_math.cuh"
#include "ibis_params.cuh"

namespace ibis {

constexpr int NL = 6;   // soil layers
constexpr int NB = 3;   // bedrock layers
constexpr int NS = 3;   // snow layers

template <typename R>
struct Col {
    R tsoi[NL], wsoi[NL], wisoi[NL], tg, wpud, wipud, tsoi_deep[NB];
    R fi, tsno[NS], hsno[NS], ti, tlsub;
    R tu, ts, tl, t12, t34, q12, q34;
    R wliqu, wliqs, wliql, wsnou, wsnos, wsnol;
    R ci_u[2], gs_u[2], cs_u[2], ci_l[3], gs_l[3], cs_l[3];
    R a10su, a10du, a10sl, a10dl;
    R firefac, nytimes, nfirestep, sdry, nfirestep_vpd, sdry_vpd;
};

template <typename R>
struct Forc {
    R ta, qa, ua, ps, cosz, sd[2], si[2], fira, rain, snow;
};

// Read-only view of one cell's static planes.
template <typename R>
struct Stat {
    const R* __restrict__ base;
    int ld;
    __device__ __forceinline__ R operator()(int plane) const { return __ldg(base + (size_t)plane * ld); }
    __device__ __forceinline__ R operator()(int plane, int k) const { return __ldg(base + (size_t)(plane + k) * ld); }
};

// Optional writer of one cell's diagnostic planes.
template <typename R>
struct Diag {
    R* __restrict__ base;  // nullptr: diagnostics off
    int ld;
    __device__ __forceinline__ void put(int plane, R v) const {
        if (base) base[(size_t)plane * ld] = v;
    }
    __device__ __forceinline__ void put(int plane, int k, R v) const {
        if (base) base[(size_t)(plane + k) * ld] = v;
    }
};

// ===========================================================================
// radiation (reference physics/radiation.py)
// ===========================================================================

template <typename R>
struct Rad {
    R solu, sols, soll, solg, soli;
    R firu, firs, firl, firg, firi, firb;
    R asurd[2], asuri[2];
    R topparu, topparl, scu[4], scl[4], dbeamu, dbeaml;
    R termu6, termu7, terml6, terml7;
};

template <typename R>
struct Optics { R om, betad, betai, avmu, gdir; };

// twoset (radiation.py:75-177)
template <typename R>
__device__ __forceinline__ Optics<R> two_stream_optics(R cosz, R lai, R sai, R fwet, R rliq, R tveg, R rho, R tau,
                                                       R ov, R oh, R osno, bool sun, R tmelt, bool upper,
                                                       R fws, R rls, R tst) {
    R orand = R(1.0) - ov - oh;
    R om0 = rho + tau;
    R ztab = R(0.5) - cosz / R(3.0);
    R rw = R(1.0) / mx(om0, R(1e-12));
    R betad = (ov * R(0.5) * (rho + tau) + oh * rho + orand * ((R(1.0) - ztab) * rho + ztab * tau)) * rw;
    R betai = (ov * R(0.5) * (rho + tau) + oh * rho + orand * (R(2.0 / 3.0) * rho + R(1.0 / 3.0) * tau)) * rw;
    R gdir = ov * R(2.0 / 3.1415927) * sq(mx(R(0.0), R(1.0) - cosz * cosz)) + oh * cosz + orand * R(0.5);
    R y, o;
    if (upper) {
        R xu = lai / mx(lai + sai, R(1e-7));
        y = xu * (fwet * (R(1.0) - rliq)) + (R(1.0) - xu) * (fws * (R(1.0) - rls));
        o = (xu * clip((tmelt - tveg) / R(0.1), R(0.6), R(1.0)) + (R(1.0) - xu) * clip((tmelt - tst) / R(0.1), R(0.6), R(1.0))) * osno;
    } else {
        y = fwet * (R(1.0) - rliq);
        o = osno * (R(0.6) + R(0.4) * clip((tmelt - tveg) / R(1.0), R(0.0), R(1.0)));
    }
    R ys = y * o;
    R om = mx((R(1.0) - y) * om0 + ys, R(1e-12));
    betad = ((R(1.0) - y) * om0 * betad + ys * R(0.5)) / om;
    betai = ((R(1.0) - y) * om0 * betai + ys * R(0.5)) / om;
    Optics<R> r;
    r.om = sun ? om : R(0.0);
    r.betad = sun ? betad : R(0.0);
    r.betai = sun ? betai : R(0.0);
    r.avmu = R(1.0);
    r.gdir = sun ? gdir : R(0.0);
    return r;
}

template <typename R>
struct TwoStr {
    R abvegd, abvegi, refld, refli, fbeldd, fbelid, fbelii, om;
    R term[7];
};

__device__ __forceinline__ float tiny30(float v) { return fabsf(v) < 1e-30f ? 1e-30f : v; }
__device__ __forceinline__ double tiny30(double v) { return fabs(v) < 1e-30 ? 1e-30 : v; }

// twostr (radiation.py:180-313)
template <typename R>
__device__ __forceinline__ TwoStr<R> two_stream(R cosz, R lai, R sai, R asd, R asi, const Optics<R>& o, bool sun,
                                                bool vis, R eps) {
    R om = o.om, betad = o.betad, betai = o.betai, avmu = o.avmu, gdir = o.gdir;
    R b = R(1.0) - om * (R(1.0) - betai);
    R c = om * betai;
    R t0 = b * b - c * c;
    R q = sq(mx(R(0.0), t0));
    R k = gdir / mx(cosz, R(0.01));
    R p = avmu * k;
    R sgn = (p >= q) ? R(1.0) : R(-1.0);
    if (ab(p - q) < R(0.001) * p) p = (R(1.0) + sgn * R(0.001)) * p;
    R c0 = om * p;
    R d = c0 * betad;
    R f = c0 * (R(1.0) - betad);
    R h = q / avmu;
    R sigma = p * p - t0;
    R ud1 = b - c / mx(asd, R(1e-12));
    R ui1 = b - c / mx(asi, R(1e-12));
    R ud2 = b - c * asd;
    R ui2 = b - c * asi;
    R ud3 = f + c * asd;
    R xai = mx(lai + sai, eps);
    R s1 = ex(-h * xai);
    R s2 = ex(-k * xai);
    R p1 = b + q, p2 = b - q, p3 = b + p, p4 = b - p;
    R s1m = mx(s1, R(1e-30));
    R rw = R(1.0) / s1m;
    R dd1 = p1 * (ud1 - q) * rw - p2 * (ud1 + q) * s1;
    R di1 = p1 * (ui1 - q) * rw - p2 * (ui1 + q) * s1;
    R dd2 = (ud2 + q) * rw - (ud2 - q) * s1;
    R di2 = (ui2 + q) * rw - (ui2 - q) * s1;
    dd1 = tiny30(dd1); di1 = tiny30(di1); dd2 = tiny30(dd2); di2 = tiny30(di2); sigma = tiny30(sigma);
    R h1 = -d * p4 - c * f;
    R rw2 = s2 * (d - c - h1 * (ud1 + p) / sigma);
    R h2 = (R(1.0) / dd1) * ((d - h1 * p3 / sigma) * (ud1 - q) / s1m - p2 * rw2);
    R h3 = -(R(1.0) / dd1) * ((d - h1 * p3 / sigma) * (ud1 + q) * s1 - p1 * rw2);
    R h4 = -f * p3 - c * d;
    R rw3 = s2 * (ud3 - h4 * (ud2 - p) / sigma);
    R h5 = -(R(1.0) / dd2) * (h4 * (ud2 + q) / (sigma * s1m) + rw3);
    R h6 = (R(1.0) / dd2) * (h4 * s1 * (ud2 - q) / sigma + rw3);
    R h7 = c * (ui1 - q) / (di1 * s1m);
    R h8 = -c * s1 * (ui1 + q) / di1;
    R h9 = (ui2 + q) / (di2 * s1m);
    R h10 = -s1 * (ui2 - q) / di2;
    TwoStr<R> r;
    R fbeldd = s2;
    R fbelid = h4 / sigma * s2 + h5 * s1 + h6 / s1m;
    R fbelii = h9 * s1 + h10 / s1m;
    R refld = h1 / sigma + h2 + h3;
    R refli = h7 + h8;
    R absurd = (R(1.0) - asd) * fbeldd + (R(1.0) - asi) * fbelid;
    R absuri = (R(1.0) - asi) * fbelii;
    R abvegd = mx(R(0.0), R(1.0) - refld - absurd);
    R abvegi = mx(R(0.0), R(1.0) - refli - absuri);
    if (xai < eps) { abvegd = R(0.0); abvegi = R(0.0); }
    r.abvegd = sun ? abvegd : R(0.0);
    r.abvegi = sun ? abvegi : R(0.0);
    r.refld = sun ? refld : R(0.0);
    r.refli = sun ? refli : R(0.0);
    r.fbeldd = sun ? fbeldd : R(0.0);
    r.fbelid = sun ? fbelid : R(0.0);
    r.fbelii = sun ? fbelii : R(0.0);
    r.om = om;
    if (vis) {
        r.term[0] = k * (R(1.0) + (h4 - h1) / sigma);
        r.term[1] = h * (h5 - h2);
        r.term[2] = h * (h9 - h7);
        r.term[3] = h * (h3 - h6);
        r.term[4] = h * (h8 - h10);
        r.term[5] = k;
        r.term[6] = h;
    }
    return r;
}

// compute_radiation = solsur + solalb + solarf per band, then irrad (radiation.py:316-761)
template <typename R>
__device__ __forceinline__ void radiation(Rad<R>& out, const Col<R>& c, const Forc<R>& F, const Stat<R>& S,
                                          R fwetu, R fwets, R fwetl, R rliqu, R rliqs, R rliql,
                                          const DevParams<R>& P) {
    const R eps = P.epsilon;
    const bool sun = F.cosz > R(0.0);
    const R lai0 = S(IBIS_STAT_LAI, 0), lai1 = S(IBIS_STAT_LAI, 1);
    const R sai0 = S(IBIS_STAT_SAI, 0), sai1 = S(IBIS_STAT_SAI, 1);
    const R fu = S(IBIS_STAT_FU), fl = S(IBIS_STAT_FL), fi = c.fi;
    const R w0 = c.wsoi[0], i0 = c.wisoi[0], tsno0 = c.tsno[0];
    out.solu = out.sols = out.soll = out.solg = out.soli = R(0.0);
#pragma unroll
    for (int ib = 0; ib < 2; ++ib) {
        // solsur (radiation.py:316-369)
        R zw = w0 * (R(1.0) - i0);
        R dinc = R(1.0) + clip(R(1.0) - zw / R(0.50), R(0.0), R(1.0));
        R albsod = mn((ib == 0 ? S(IBIS_STAT_ALBSAV) : S(IBIS_STAT_ALBSAN)) * dinc, R(0.80));
        R albsoi = albsod;
        R ahi = ib == 0 ? R(0.70) : R(0.40), alo = ib == 0 ? R(0.90) : R(0.60);
        R tslo = P.tmelt - R(15.0);
        R x = (ahi * (tsno0 - tslo) + alo * (P.tmelt - tsno0)) / (P.tmelt - tslo);
        x = clip(x, ahi, alo);
        R zfac = mx(R(0.0), R(1.5) / (R(1.0) + R(4.0) * F.cosz) - R(0.5));
        R albsnd = mn(R(0.99), x + (R(1.0) - x) * zfac);
        R albsni = mn(R(1.0), x);
        if (!sun) { albsod = albsoi = albsnd = albsni = R(0.0); }
        // solalb (radiation.py:372-447)
        Optics<R> ol = two_stream_optics(F.cosz, lai0, sai0, fwetl, rliql, c.tl, P.rhoveg[2 * ib + 0],
                                         P.tauveg[2 * ib + 0], P.oriev[0], P.orieh[0], P.omegasno[ib], sun,
                                         P.tmelt, false, R(0), R(0), R(0));
        TwoStr<R> lo = two_stream(F.cosz, lai0, sai0, albsod, albsoi, ol, sun, ib == 0, eps);
        R asd = fl * (R(1.0) - fi) * lo.refld + (R(1.0) - fl) * (R(1.0) - fi) * albsod + fi * albsnd;
        R asi = fl * (R(1.0) - fi) * lo.refli + (R(1.0) - fl) * (R(1.0) - fi) * albsoi + fi * albsni;
        Optics<R> ou = two_stream_optics(F.cosz, lai1, sai1, fwetu, rliqu, c.tu, P.rhoveg[2 * ib + 1],
                                         P.tauveg[2 * ib + 1], P.oriev[1], P.orieh[1], P.omegasno[ib], sun,
                                         P.tmelt, true, fwets, rliqs, c.ts);
        TwoStr<R> up = two_stream(F.cosz, lai1, sai1, asd, asi, ou, sun, ib == 0, eps);
        out.asurd[ib] = sun ? fu * up.refld + (R(1.0) - fu) * asd : R(0.0);
        out.asuri[ib] = sun ? fu * up.refli + (R(1.0) - fu) * asi : R(0.0);
        // solarf (radiation.py:450-540)
        R sd = F.sd[ib], si = F.si[ib];
        R xx = sd * up.abvegd + si * up.abvegi;
        R y = lai1 / mx(lai1 + sai1, eps);
        R solu = xx * y;
        R sols = xx * (R(1.0) - y);
        R s2d = sd * up.fbeldd;
        R s2i = sd * up.fbelid + si * up.fbelii;
        R s3d = fu * s2d + (R(1.0) - fu) * sd;
        R s3i = fu * s2i + (R(1.0) - fu) * si;
        R soll = s3d * lo.abvegd + s3i * lo.abvegi;
        R xd = (fl * lo.fbeldd + R(1.0) - fl) * s3d;
        R xi = fl * (s3d * lo.fbelid + s3i * lo.fbelii) + (R(1.0) - fl) * s3i;
        R solg = (R(1.0) - albsod) * xd + (R(1.0) - albsoi) * xi;
        R soli = (R(1.0) - albsnd) * s3d + (R(1.0) - albsni) * s3i;
        if (ib == 0) {
            R c0 = up.term[0] * sd;
            R c1 = up.term[1] * sd + up.term[2] * si;
            R c2 = up.term[3] * sd + up.term[4] * si;
            R c3 = c0 + c1 + c2;
            out.scu[0] = c0; out.scu[1] = c1; out.scu[2] = c2; out.scu[3] = c3;
            out.topparu = c3 * lai1 / mx(lai1 + sai1, eps);
            out.dbeamu = (R(1.0) - up.om) * up.term[5] * sd;
            c0 = lo.term[0] * s3d;
            c1 = lo.term[1] * s3d + lo.term[2] * s3i;
            c2 = lo.term[3] * s3d + lo.term[4] * s3i;
            c3 = c0 + c1 + c2;
            out.scl[0] = c0; out.scl[1] = c1; out.scl[2] = c2; out.scl[3] = c3;
            out.topparl = c3 * lai0 / mx(lai0 + sai0, eps);
            out.dbeaml = (R(1.0) - lo.om) * lo.term[5] * s3d;
            out.termu6 = up.term[5]; out.termu7 = up.term[6];
            out.terml6 = lo.term[5]; out.terml7 = lo.term[6];
        }
        if (sun) {
            out.solu = out.solu + solu;
            out.sols = out.sols + sols;
            out.soll = out.soll + soll;
            out.solg = out.solg + solg;
            out.soli = out.soli + soli;
        }
    }
    // irrad (radiation.py:543-641)
    R emu = R(1.0) - ex(-lai1 / R(1.0));
    R ems = R(1.0) - ex(-sai1 / R(1.0));
    R eml = R(1.0) - ex(-(lai0 + sai0) / R(1.0));
    const R emg = R(0.95), emi = R(0.95);
    R tu4 = P.stef * quart(c.tu);
    R ts4 = P.stef * quart(c.ts);
    R tl4 = P.stef * quart(c.tl);
    R tg4 = P.stef * quart(c.tg);
    R ti4 = P.stef * quart(c.ti);
    R fira = F.fira;
    R fdown = (R(1.0) - fu) * fira + fu * ((R(1.0) - emu) * (R(1.0) - ems) * fira + emu * (R(1.0) - ems) * tu4 + ems * ts4);
    R fdowng = (R(1.0) - eml) * fdown + eml * tl4;
    R fupg = (R(1.0) - emg) * fdowng + emg * tg4;
    R fupgb = (R(1.0) - emg) * fdown + emg * tg4;
    R fupi = (R(1.0) - emi) * fdown + emi * ti4;
    R fup = (R(1.0) - fi) * (fl * (eml * tl4 + (R(1.0) - eml) * fupg) + (R(1.0) - fl) * fupgb) + fi * fupi;
    out.firb = (R(1.0) - fu) * fup + fu * ((R(1.0) - emu) * (R(1.0) - ems) * fup + emu * tu4 + ems * (R(1.0) - emu) * ts4);
    out.firu = emu * ems * ts4 + emu * (R(1.0) - ems) * fup + emu * fira - R(2.0) * emu * tu4;
    out.firs = ems * emu * tu4 + ems * fup + ems * (R(1.0) - emu) * fira - R(2.0) * ems * ts4;
    out.firl = eml * fdown + eml * fupg - R(2.0) * eml * tl4;
    out.firg = fl * (fdowng - fupg) + (R(1.0) - fl) * (fdown - fupgb);
    out.firi = fdown - fupi;
}

// ===========================================================================
// interception (reference physics/interception.py)
// ===========================================================================

template <typename R>
__device__ __forceinline__ void wet_fraction(R tveg, R wliq, R wsno, R wliqmax, R wsnomax, R fmax,
                                             const DevParams<R>& P, R& fwet, R& rliq) {
    R xliq = wliq / mx(wliqmax, R(0.01));
    R xtot = xliq + wsno / mx(wsnomax, R(0.01));
    fwet = mn(fmax, xtot);
    rliq = xliq / mx(xtot, P.epsilon);
    if (fwet == R(0.0)) rliq = (tveg < P.tmelt - R(1.0e-9)) ? R(0.0) : R(1.0);
}

// mix of two masses (the third of the reference's mix is always zero here)
template <typename R>
__device__ __forceinline__ void mix2(R& xm, R& tm, R x1, R t1, R x2, R t2, R x3, R t3, R eps) {
    R s = x1 + x2 + x3;
    bool ok = ab(s) >= eps;
    tm = ok ? (t1 * x1 + t2 * x2 + t3 * x3) / s : R(0.0);
    xm = ok ? s : R(0.0);
}

// twet3 (interception.py:126-171)
template <typename R>
__device__ R wet_bulb(R tak, R q, R p, const DevParams<R>& P) {
    R qs0 = qsat(esat(tak), p);
    R ta = tak - P.tmelt;
    R twk = ta * q / mx(qs0, R(1e-12)) + P.tmelt;
#pragma unroll 1
    for (int it = 0; it < 20; ++it) {
        R twold = twk - P.tmelt;
        R hv = P.hvap + P.cvap * (tak - P.tmelt) - P.ch2o * (twk - P.tmelt);
        R qw = qsat(esat(twk), p);
        R twb = ta - (hv / P.cair) * (qw - q);
        R nxt = twold + R(0.2) * (twb - twold) + P.tmelt;
        bool conv = fabs((double)(nxt - P.tmelt - twold)) < 0.02;
        twk = nxt;
        if (conv) break;
    }
    return twk;
}

template <typename R>
struct Surf { R wliq, wsno, pflux, rain, train, snow, tsnow; };

// steph2o (interception.py:174-260)
template <typename R>
__device__ __forceinline__ Surf<R> intercept(R tveg, R wliq, R wsno, R xai, R rain, R train, R snow, R tsnow,
                                             R tdrip, R tblow, R wliqmax, R wsnomax, R wliqmin,
                                             const DevParams<R>& P) {
    const R dt = P.dtime, eps = P.epsilon;
    R fint = (xai >= eps) ? (R(1.0) - ex(R(-0.5) * xai)) / xai : R(0.5);
    R rdt = R(1.0) / dt;
    R drip = xai * wliq / tdrip;
    wliq = wliq * (R(1.0) - dt / tdrip);
    wliq = wliq + dt * rain * fint;
    R pflux = rain * fint * (tveg - train) * P.ch2o;
    rain = rain * (R(1.0) - xai * fint);
    R x = wliq;
    wliq = mn(wliq, wliqmax);
    if (wliq < wliqmin) wliq = R(0.0);
    drip = drip + xai * (x - wliq) * rdt;
    R blow = xai * wsno / tblow;
    wsno = wsno * (R(1.0) - dt / tblow);
    wsno = wsno + dt * snow * fint;
    pflux = pflux + snow * fint * (tveg - tsnow) * P.cice;
    snow = snow * (R(1.0) - xai * fint);
    x = wsno;
    wsno = mn(wsno, wsnomax);
    if (wsno < P.wsnomin) wsno = R(0.0);
    blow = blow + xai * (x - wsno) * rdt;
    const R dcp = P.ch2o - P.cice;
    R dfrz = (tveg < P.tmelt - R(1.0e-9)) ? wliq : R(0.0);
    pflux = pflux + dfrz * (dcp * (P.tmelt - tveg) - P.hfus) * rdt;
    wliq = wliq - dfrz;
    wsno = wsno + dfrz;
    R dmlt = (tveg > P.tmelt + R(1.0e-9)) ? wsno : R(0.0);
    pflux = pflux + dmlt * (dcp * (tveg - P.tmelt) + P.hfus) * rdt;
    wsno = wsno - dmlt;
    wliq = wliq + dmlt;
    Surf<R> s;
    s.wliq = wliq; s.wsno = wsno; s.pflux = pflux;
    mix2(s.rain, s.train, rain, train, drip, tveg, R(0.0), R(0.0), eps);
    mix2(s.snow, s.tsnow, snow, tsnow, blow, tveg, R(0.0), R(0.0), eps);
    return s;
}

template <typename R>
struct Casc {
    R wliqu, wliqs, wliql, wsnou, wsnos, wsnol, pfluxu, pfluxs, pfluxl;
    R raing, traing, snowg, tsnowg, rainl, trainl, snowl, tsnowl;
};

// cascade (interception.py:263-357)
template <typename R, typename Q>
__device__ __forceinline__ void cascade(Casc<R>& o, const Col<R>& c, const Forc<R>& F, const Stat<R>& S,
                                        const DevParams<R>& P, const Q& q) {
    const R eps = P.epsilon;
    const R fu = S(IBIS_STAT_FU), fl = S(IBIS_STAT_FL);
    R tw = (F.ta > P.tmelt + R(1.0e-9)) ? wet_bulb(F.ta, F.qa, F.ps, P) : P.tmelt;
    R rainu, trainu, snowu, tsnowu;
    mix2(rainu, trainu, F.rain, mx(tw, P.tmelt), R(0.0), mx(c.t12, P.tmelt), R(0.0), R(0.0), eps);
    mix2(snowu, tsnowu, F.snow, mn(F.ta, P.tmelt), R(0.0), mn(c.t12, P.tmelt), R(0.0), R(0.0), eps);
    Surf<R> u = intercept(c.tu, c.wliqu, c.wsnou, R(2.0) * S(IBIS_STAT_LAI, 1), rainu, trainu, snowu, tsnowu,
                          P.tdripu, P.tblowu, q.wliqumax(), P.wsnoumax, q.wliqmin(), P);
    Surf<R> s = intercept(c.ts, c.wliqs, c.wsnos, R(2.0) * S(IBIS_STAT_SAI, 1), u.rain, u.train, u.snow, u.tsnow,
                          P.tdrips, P.tblows, q.wliqsmax(), P.wsnosmax, q.wliqmin(), P);
    mix2(o.rainl, o.trainl, fu * s.rain, s.train, (R(1.0) - fu) * rainu, trainu, R(0.0), mx(c.t34, P.tmelt), eps);
    mix2(o.snowl, o.tsnowl, fu * s.snow, s.tsnow, (R(1.0) - fu) * snowu, tsnowu, R(0.0), mn(c.t34, P.tmelt), eps);
    Surf<R> l = intercept(c.tl, c.wliql, c.wsnol, R(2.0) * (S(IBIS_STAT_LAI, 0) + S(IBIS_STAT_SAI, 0)), o.rainl,
                          o.trainl, o.snowl, o.tsnowl, P.tdripl, P.tblowl, q.wliqlmax(), P.wsnolmax,
                          q.wliqmin(), P);
    mix2(o.raing, o.traing, fl * l.rain, l.train, (R(1.0) - fl) * o.rainl, o.trainl, R(0.0), R(0.0), eps);
    mix2(o.snowg, o.tsnowg, fl * l.snow, l.tsnow, (R(1.0) - fl) * o.snowl, o.tsnowl, R(0.0), R(0.0), eps);
    o.wliqu = u.wliq; o.wliqs = s.wliq; o.wliql = l.wliq;
    o.wsnou = u.wsno; o.wsnos = s.wsno; o.wsnol = l.wsno;
    o.pfluxu = u.pflux; o.pfluxs = s.pflux; o.pfluxl = l.pflux;
}

// steph2o2 without its discarded fvapa/fsena outputs (interception.py:364-416)
template <typename R>
__device__ __forceinline__ void evap_intercepted(R& tveg, R& wliq, R& wsno, R rliq, R fvapw, R cveg,
                                                 const DevParams<R>& P) {
    const R dt = P.dtime;
    wliq = wliq - dt * rliq * fvapw;
    wsno = wsno - dt * (R(1.0) - rliq) * fvapw;
    wliq = mx(wliq, R(0.0));
    wsno = mx(wsno, R(0.0));
    const R rh = R(1.0) / P.hfus;
    R chav = cveg + P.ch2o * wliq + P.cice * wsno;
    if ((tveg < P.tmelt - R(1.0e-9)) && (wliq > R(0.0))) {
        R dh = chav * (P.tmelt - tveg);
        R dw = mn(wliq, mx(R(0.0), dh * rh));
        wliq = wliq - dw;
        wsno = wsno + dw;
        R chn = cveg + P.ch2o * wliq + P.cice * wsno;
        tveg = P.tmelt - (dh - P.hfus * dw) / chn;
    }
    if ((tveg > P.tmelt + R(1.0e-9)) && (wsno > R(0.0))) {
        chav = cveg + P.ch2o * wliq + P.cice * wsno;
        R dh = chav * (tveg - P.tmelt);
        R dw = mn(wsno, mx(R(0.0), dh * rh));
        wsno = wsno - dw;
        wliq = wliq + dw;
        R chn = cveg + P.ch2o * wliq + P.cice * wsno;
        tveg = P.tmelt + (dh - P.hfus * dw) / chn;
    }
}

// ===========================================================================
// aerodynamics (reference physics/canopy_exchange.py:192-426)
// ===========================================================================

template <typename R>
struct Aero {
    R rhoa, cp, za, z1, z2, z3, z4, z12, z34, bdl, bdu, dil, diu, exphl, expl, exphu, expu;
    R alogav, alog1, alog2, alog3, alog4, aloga;
    R hl, hu;   // the exponents of expl and expu (the FP32 wind profile works from them)
};

// canini (canopy_exchange.py:192-280); u2/alogu/alogl are returned separately (they are carried)
template <typename R>
__device__ __forceinline__ void aero_geometry(Aero<R>& A, R& u2, R& alogu, R& alogl, const Forc<R>& F,
                                              const Stat<R>& S, R fi, const DevParams<R>& P) {
    const R lai0 = S(IBIS_STAT_LAI, 0), lai1 = S(IBIS_STAT_LAI, 1);
    const R sai0 = S(IBIS_STAT_SAI, 0), sai1 = S(IBIS_STAT_SAI, 1);
    const R ztop0 = S(IBIS_STAT_ZTOP, 0), ztop1 = S(IBIS_STAT_ZTOP, 1);
    const R zbot0 = S(IBIS_STAT_ZBOT, 0), zbot1 = S(IBIS_STAT_ZBOT, 1);
    const R fu = S(IBIS_STAT_FU), fl = S(IBIS_STAT_FL), z0soi = S(IBIS_STAT_Z0SOI);
    R pa = F.ps * R(0.999);
    A.rhoa = pa / (P.rair * F.ta * (R(1.0) + R((double)P.rvap / (double)P.rair - 1.0) * F.qa));
    A.cp = P.cair * (R(1.0) + R((double)P.cvap / (double)P.cair - 1.0) * F.qa);
    R za = (F.ps - pa) / (A.rhoa * P.grav);
    A.za = mx(za, ztop1 + R(1.0));
    R x = fl * (R(1.0) - fi) * R(2.0) * (lai0 + sai0) / P.alaiml;
    x = mn(x, R(3.0));
    R x1 = mn(x, R(1.0));
    R rw = mx(ztop0 - zbot0, R(0.01));
    R cveg = (R(0.4) / rw) * mx(R(1e-5), x);
    R dveg = (R(0.1) * rw) / mx(R(1e-5), mx(x, x * x));
    R bveg = sq(R(2.0) * cveg / dveg);
    A.bdl = R(0.5) * bveg * dveg;
    A.dil = R(1.0) / dveg;
    rw = (R(1.0) - x1) * (mx(z0soi, P.z0sno) + R(0.01));
    R z3 = x1 * ztop0 + rw;
    R z4 = x1 * zbot0 + rw;
    A.z3 = z3; A.z4 = z4; A.z34 = R(0.5) * (z3 + z4);
    A.hl = bveg * (z3 - z4);
    A.exphl = ex(R(0.5) * bveg * (z3 - z4));
    A.expl = A.exphl * A.exphl;
    R displ = x1 * R(0.7) * z3;
    x = fu * R(2.0) * (lai1 + sai1) / P.alaimu;
    x = mn(x, R(3.0));
    x1 = mn(x, R(1.0));
    rw = mx(ztop1 - zbot1, R(0.01));
    cveg = (R(0.4) / rw) * mx(R(1e-5), x);
    dveg = (R(0.1) * rw) / mx(R(1e-5), mx(x, x * x));
    rw = R(1.0) / dveg;
    bveg = sq(R(2.0) * cveg * rw);
    A.bdu = R(0.5) * bveg * dveg;
    A.diu = rw;
    rw = (R(1.0) - x1) * (z3 + R(0.01));
    R z1 = x1 * ztop1 + rw;
    R z2 = x1 * zbot1 + rw;
    A.z1 = z1; A.z2 = z2; A.z12 = R(0.5) * (z1 + z2);
    A.hu = bveg * (z1 - z2);
    A.exphu = ex(R(0.5) * bveg * (z1 - z2));
    A.expu = A.exphu * A.exphu;
    R dispu = x1 * R(0.7) * z1 + (R(1.0) - x1) * displ;
    R alogg = lg(z0soi);
    R alogi = lg(P.z0sno);
    A.alogav = (R(1.0) - fi) * alogg + fi * alogi;
    A.alog4 = lg(mx(z4, mx(R(1.1) * z0soi, R(1.1) * P.z0sno)));
    A.alog3 = lg(z3 - displ);
    A.alog2 = lg(z2 - displ);
    A.alog1 = lg(z1 - dispu);
    A.aloga = lg(A.za - dispu);
    u2 = F.ua / A.exphu;
    alogu = lg(mx(R(0.01), R(0.1) * (z1 - z2)));
    alogl = lg(mx(R(0.01), R(0.1) * (z3 - z4)));
}

// fstrat (canopy_exchange.py:287-326); albm == albh at both call sites
template <typename R>
__device__ __forceinline__ void stability(R& sm, R& sh, R tb, R tt, R ttfac, R qb, R qt, R zb, R zt, R alb, R alt,
                                          R u, bool first, const DevParams<R>& P) {
    R zht = tt * ttfac * (R(1.0) + R(0.622) * qt);
    R zhb = tb * (R(1.0) + R(0.622) * qb);
    R rich = P.grav * mx(zt - zb, R(0.0)) * (zht - zhb) / (R(0.5) * (zht + zhb) * (u * u));
    rich = clip(rich, R(-2.0), R(1.0));
    R smn, shn;
    if (rich <= R(0.0)) {
        R xm = mx(alt - alb, R(0.5));
        R rw = sq(mx(-rich, R(0.0)));
        R vx = P.vonk / xm;
        R ym = (vx * vx) * ex(R(0.5) * xm) * rw;
        smn = R(1.0) - R(10.0) * rich / (R(1.0) + R(75.0) * ym);
        shn = R(1.0) - R(15.0) * rich / (R(1.0) + R(75.0) * ym);
    } else {
        R rp = mx(rich, R(0.0));
        R zz = sq(R(1.0) + R(5.0) * rp);
        smn = R(1.0) / (R(1.0) + R(10.0) * rp / zz);
        shn = R(1.0) / (R(1.0) + R(15.0) * rp * zz);
    }
    if (first) { sm = smn; sh = shn; }
    else { sm = R(0.5) * smn + R(0.5) * sm; sh = R(0.5) * shn + R(0.5) * sh; }
}

template <typename R>
struct Trans { R cu, cl, su, ss, sl, sg, si; };

// The exponential wind profile inside one canopy story (canopy_exchange.py:
// 365-392) in closed form, for the FP32 kernels.  With E = exp(h) the
// reference forms y = ((x+1)E + (x-1)/E) / ((x+1)E - (x-1)/E) and then the
// profile coefficients from y + 1 and y - 1.  In float32, y rounds to 1 once E
// passes ~3e3 (a dense canopy), so (y - 1) keeps no correct digit and the wind
// at the story's bottom, proportional to (y - 1) E, comes out wrong by O(1).
// With D = 2x sinh h + 2 cosh h (= the reference's denominator) the same
// quantities are
//   y = (x cosh h + sinh h) / (x sinh h + cosh h),
//   a = k (x+1) E,  b = k (x-1)/E,  k = tau / (D bd),
//   a + b = 2k (x cosh h + sinh h),  a/E^.5 + b E^.5 = 2k (x cosh h/2 + sinh h/2),
//   a/E + b E = 2k x,  bd (a/E - b E) = 2 tau / D,
// with sinh and cosh from expm1, which stay accurate for every h.
template <typename R>
struct Profile {
    R y;       // the reference's y
    R d;       // D / 2
    R top2;    // (a + b) / k
    R mid2;    // (a / E^.5 + b E^.5) / k
};

template <typename R>
__device__ __forceinline__ Profile<R> profile(R x, R h) {
    const R ep = em1(h), em = em1(-h), ep2 = em1(R(0.5) * h), em2 = em1(R(-0.5) * h);
    const R sh = R(0.5) * (ep - em), ch = R(1.0) + R(0.5) * (ep + em);
    const R sh2 = R(0.5) * (ep2 - em2), ch2 = R(1.0) + R(0.5) * (ep2 + em2);
    Profile<R> p;
    p.d = x * sh + ch;
    p.y = (x * ch + sh) / p.d;
    p.top2 = R(2.0) * (x * ch + sh);
    p.mid2 = R(2.0) * (x * ch2 + sh2);
    return p;
}

// turcof (canopy_exchange.py:333-426); strat = (sml, shl, smu, shu) carried across passes
template <typename R>
__device__ __forceinline__ void transfer(Trans<R>& T, R (&strat)[4], R& u2, R& alogu, R& alogl, const Aero<R>& A,
                                         const Forc<R>& F, R t12, R t34, R q12, R q34, bool first,
                                         const DevParams<R>& P) {
    const R vonk = P.vonk;
    stability(strat[0], strat[1], t34, t12, R(1.0), q34, q12, A.z3, A.z2, alogl, A.alog2, u2, first, P);
    stability(strat[2], strat[3], t12, F.ta, P.tfac, q12, F.qa, A.z1, A.za, alogu, A.aloga, F.ua, first, P);
    R v = (A.alog4 - A.alogav) / vonk;
    R u1, u12, nu2, u3, u34, u4, nalogl, nalogu;
    if constexpr (sizeof(R) == 4) {
        // FP32: the closed forms of Profile (no cancellation in y - 1)
        const R xl = (v * v) * A.bdl;
        const Profile<R> pl = profile(xl, A.hl);
        nalogl = A.alog3 - vonk * sq(pl.y / A.bdl);
        v = (A.alog2 - nalogl) / vonk;
        const R xu = (v * v) * A.bdu / strat[0];
        const Profile<R> pu = profile(xu, A.hu);
        nalogu = A.alog1 - vonk * sq(pu.y / A.bdu);
        v = F.ua * vonk / (A.aloga - nalogu);
        const R tauu = (v * v) * strat[2];
        const R ku = R(0.5) * tauu / (pu.d * A.bdu);
        const R taul = tauu / pu.d;
        const R kl = R(0.5) * taul / (pl.d * A.bdl);
        u1 = mx(R(0.01), sq(mx(R(0.0), ku * pu.top2)));
        u12 = mx(R(0.01), sq(mx(R(0.0), ku * pu.mid2)));
        nu2 = mx(R(0.01), sq(mx(R(0.0), R(2.0) * ku * xu)));
        u3 = mx(R(0.01), sq(mx(R(0.0), kl * pl.top2)));
        u34 = mx(R(0.01), sq(mx(R(0.0), kl * pl.mid2)));
        u4 = mx(R(0.01), sq(mx(R(0.0), R(2.0) * kl * xl)));
    } else {
        // FP64: the reference's operations
        R x = (v * v) * A.bdl;
        R rw = R(1.0) / A.expl;
        R yl = ((x + R(1)) * A.expl + (x - R(1)) * rw) / ((x + R(1)) * A.expl - (x - R(1)) * rw);
        nalogl = A.alog3 - vonk * sq(yl / A.bdl);
        v = (A.alog2 - nalogl) / vonk;
        x = (v * v) * A.bdu / strat[0];
        rw = R(1.0) / A.expu;
        R yu = ((x + R(1)) * A.expu + (x - R(1)) * rw) / ((x + R(1)) * A.expu - (x - R(1)) * rw);
        nalogu = A.alog1 - vonk * sq(yu / A.bdu);
        v = F.ua * vonk / (A.aloga - nalogu);
        R tauu = (v * v) * strat[2];
        R a = R(0.5) * tauu * (yu + R(1)) / A.bdu;
        R b = R(0.5) * tauu * (yu - R(1)) / A.bdu;
        R taul = A.bdu * (a / A.expu - b * A.expu);
        R cc = R(0.5) * taul * (yl + R(1)) / A.bdl;
        R d = R(0.5) * taul * (yl - R(1)) / A.bdl;
        u1 = mx(R(0.01), sq(mx(R(0.0), a + b)));
        u12 = mx(R(0.01), sq(mx(R(0.0), a / A.exphu + b * A.exphu)));
        nu2 = mx(R(0.01), sq(mx(R(0.0), a / A.expu + b * A.expu)));
        u3 = mx(R(0.01), sq(mx(R(0.0), cc + d)));
        u34 = mx(R(0.01), sq(mx(R(0.0), cc / A.exphl + d * A.exphl)));
        u4 = mx(R(0.01), sq(mx(R(0.0), cc / A.expl + d * A.expl)));
    }
    R ca = F.ua * strat[3] * P.vonk2 / ((A.aloga - nalogu) * (A.aloga - A.alog1));
    ca = mn(P.cdmax, ca / (R(1.0) + ca * R(1e-20)));
    const R rhoa = A.rhoa;
    R cai = R(1.0) / (rhoa * ca);
    R cbi = A.diu * (A.z1 - A.z12) / (rhoa * R(0.5) * (u1 + u12));
    R cci = A.diu * (A.z12 - A.z2) / (rhoa * R(0.5) * (u12 + nu2));
    R cdi = (A.alog2 - nalogl) * (A.alog2 - A.alog3) / (rhoa * nu2 * strat[1] * P.vonk2);
    R cei = A.dil * (A.z3 - A.z34) / (rhoa * R(0.5) * (u3 + u34));
    R cfi = A.dil * (A.z34 - A.z4) / (rhoa * R(0.5) * (u34 + u4));
    T.cu = R(1.0) / (cai + cbi);
    T.cl = R(1.0) / (cci + cdi + cei);
    T.su = rhoa * P.cleaf * sq(u12 / P.dleaf[1]);
    T.ss = rhoa * P.cstem * sq(u12 / P.dstem[1]);
    T.sl = rhoa * P.cgrass * sq(u34 / P.dleaf[0]);
    R sg0 = rhoa * (R(0.004) + R(0.012) * u4);
    R si0 = rhoa * (R(0.003) + R(0.010) * u4);
    T.sg = R(1.0) / (cfi + R(1.0) / sg0);
    T.si = R(1.0) / (cfi + R(1.0) / si0);
    u2 = nu2; alogu = nalogu; alogl = nalogl;
}

// impexp / impexp2 (canopy_exchange.py:433-463)
template <typename R>
__device__ __forceinline__ R weight_veg(R t, R ch, R wliq, R wsno, R prev, bool first, const DevParams<R>& P) {
    if (first) return R(1.0);
    R h = ch * (t - P.tmelt);
    R z = mx(ab(h), P.epsilon);
    R nw;
    if (h > P.epsilon + R(1.0e-8)) nw = R(1.0) - mn(R(1.0), P.hfus * wsno / z);
    else if (h < -P.epsilon - R(1.0e-8)) nw = R(1.0) - mn(R(1.0), P.hfus * wliq / z);
    else nw = R(1.0);
    return R(0.5) * (prev + nw);
}

template <typename R>
__device__ __forceinline__ R weight_snow(R t, R told, R prev, bool first, const DevParams<R>& P) {
    if (first) return R(1.0);
    R dt = t - told;
    R nw = (dt > P.epsilon + R(1.0e-8)) ? (P.tmelt - told) / dt : prev;
    return clip(nw, R(0.0), R(1.0));
}

}  // namespace ibis
