// The hourly step of one column: timestep_body followed by the day-loop
// accumulators (reference loops.py:234-1284, loops_gswp3.py:161-318).
#pragma once
#include "ibis_canopy.cuh"
#include "ibis_ground.cuh"

namespace ibis {

// Planes below kAccOnChip are the accumulators every day loop keeps; the
// planes from kAccOnChip on (the optional ET and NEE components) are summed
// only under their own flags.  A kernel that holds the accumulators on chip
// holds the first kind and leaves the second in the global buffer.
constexpr int kAccOnChip = IBIS_ACC_ET_TRANS;
static_assert(IBIS_ACC_NEE_DAY + 1 == IBIS_ACC_COUNT && IBIS_ACC_STRESSTL_LAST < kAccOnChip,
              "the optional accumulator planes close the accumulator block");

// Accumulator view of one cell: value planes then compensation planes.  In
// the global form (SLD = 0) ``base`` addresses every plane with leading
// dimension ``ld`` and the compensation term of plane p is plane
// p + IBIS_ACC_COUNT.  In the on-chip form (SLD = the block size) ``base``
// holds planes [0, kAccOnChip) with stride SLD and their compensation terms at
// p + kAccOnChip; the optional planes stay in the global buffer ``far``
// (leading dimension ``ld``).
template <typename R, int SLD = 0>
struct Acc {
    R* __restrict__ base;  // nullptr: no accumulators
    int ld;
    bool kahan;
    bool last = true;      // the launch's last hour for this cell: keep the end-of-hour values
    R* __restrict__ far = nullptr;
    __device__ __forceinline__ R& at(int plane) const {
        if constexpr (SLD > 0) {
            if (plane >= kAccOnChip) return far[(size_t)plane * ld];
            return base[plane * SLD];
        } else {
            return base[(size_t)plane * ld];
        }
    }
    __device__ __forceinline__ R& comp(int plane) const {
        if constexpr (SLD > 0) {
            if (plane >= kAccOnChip) return far[(size_t)(plane + IBIS_ACC_COUNT) * ld];
            return base[(plane + kAccOnChip) * SLD];
        } else {
            return base[(size_t)(plane + IBIS_ACC_COUNT) * ld];
        }
    }
    __device__ __forceinline__ void add(int plane, R x) const {
        R& v = at(plane);
        if (kahan) {
            R& cmp = comp(plane);
            R s = v, cc = cmp;
            R y = x - cc;
            R t = s + y;
            cmp = (t - s) - y;
            v = t;
        } else {
            v = v + x;
        }
    }
    __device__ __forceinline__ R get(int plane) const { return at(plane); }
};

// Values the surface phase (steps 1-9 of timestep_body) hands to the ground
// phase (steps 10-12 and the accumulators).  In the fused kernel they stay in
// registers; the two-kernel form passes them through a scratch buffer of
// IBIS_MID_COUNT planes.
template <typename R>
struct Mid {
    R heatg, heati, fvapg, fvapi, fvaput, fvaplt, ginvap, gsuvap, gtrans;
    R raing, traing, snowg, tsnowg, rainl, trainl, snowl, tsnowl;
    R an_u[2], ag_u[2], an_l[3], ag_l[3];
    R fsena;
};
constexpr int kMidCount = 28;

template <typename R>
__device__ __forceinline__ void mid_store(const Mid<R>& m, R* __restrict__ p, int ld) {
    const R v[kMidCount] = {m.heatg, m.heati, m.fvapg, m.fvapi, m.fvaput, m.fvaplt, m.ginvap, m.gsuvap, m.gtrans,
                            m.raing, m.traing, m.snowg, m.tsnowg, m.rainl, m.trainl, m.snowl, m.tsnowl,
                            m.an_u[0], m.an_u[1], m.ag_u[0], m.ag_u[1], m.an_l[0], m.an_l[1], m.an_l[2],
                            m.ag_l[0], m.ag_l[1], m.ag_l[2], m.fsena};
#pragma unroll
    for (int q = 0; q < kMidCount; ++q) p[(size_t)q * ld] = v[q];
}

template <typename R>
__device__ __forceinline__ void mid_load(Mid<R>& m, const R* __restrict__ p, int ld) {
    R v[kMidCount];
#pragma unroll
    for (int q = 0; q < kMidCount; ++q) v[q] = p[(size_t)q * ld];
    m.heatg = v[0]; m.heati = v[1]; m.fvapg = v[2]; m.fvapi = v[3]; m.fvaput = v[4]; m.fvaplt = v[5];
    m.ginvap = v[6]; m.gsuvap = v[7]; m.gtrans = v[8];
    m.raing = v[9]; m.traing = v[10]; m.snowg = v[11]; m.tsnowg = v[12];
    m.rainl = v[13]; m.trainl = v[14]; m.snowl = v[15]; m.tsnowl = v[16];
    m.an_u[0] = v[17]; m.an_u[1] = v[18]; m.ag_u[0] = v[19]; m.ag_u[1] = v[20];
    m.an_l[0] = v[21]; m.an_l[1] = v[22]; m.an_l[2] = v[23];
    m.ag_l[0] = v[24]; m.ag_l[1] = v[25]; m.ag_l[2] = v[26];
    m.fsena = v[27];
}

// setsoi (soil_physics.py:37-140): conductivity of layer k; with X3 and
// IBIS_FLAG_FORGANIC the dry conductivity of organic solids blended in
// (soil_physics.py:74-77)
template <bool X3, typename R>
__device__ __forceinline__ R layer_conductivity(const Col<R>& c, const Stat<R>& S, const DevParams<R>& P, int k) {
    R fs = R(0.01) * S(IBIS_STAT_SAND, k);
    R fc = R(0.01) * S(IBIS_STAT_CLAY, k);
    R fsilt = R(1.0) - fs - fc;
    R por = S(IBIS_STAT_POROS, k);
    R pliq = por * c.wsoi[k] * (R(1.0) - c.wisoi[k]);
    R pice = por * c.wisoi[k];
    R dry = fs * R(0.300) + fsilt * R(0.265) + fc * R(0.250);
    if constexpr (X3) {
        if (P.flags & IBIS_FLAG_FORGANIC) {
            const R fo = S(IBIS_STAT_FORGANIC, k);
            dry = (R(1.0) - fo) * dry + fo * R(0.05);
        }
    }
    return dry * pw(R(56.0), pliq) * pw(R(224.0), pice);
}

// setsoi (soil_physics.py:37-140): evaporation source fractions and latent heats
template <typename R>
__device__ __forceinline__ void evap_sources(const Col<R>& c, const Forc<R>& F, const DevParams<R>& P, R& q1, R& q2,
                                             R& q3, R& q4, R& hvasug, R& hvasui) {
    const R eps = P.epsilon;
    {
        R pud = c.wpud + c.wipud;
        R zwpud = clip(P.zwpmax * pud / mx(P.wpudmax, eps), R(0.0), P.zwpmax);
        R w0 = c.wsoi[0], i0 = c.wisoi[0];
        R zwsoi = (R(1.0) - i0) * w0 + i0;
        bool soilw = zwsoi >= eps, haspud = zwpud >= eps;
        R r1 = R(1.0) / mx(zwsoi, eps);
        R r2 = R(1.0) / mx(pud, eps);
        q1 = soilw ? (haspud ? (R(1.0) - zwpud) * (R(1.0) - i0) * w0 * r1 : (R(1.0) - i0) * w0 * r1) : R(0.0);
        q2 = soilw ? (haspud ? (R(1.0) - zwpud) * i0 * r1 : i0 * r1) : R(0.0);
        bool warm = c.tsoi[0] >= P.tmelt - R(1.0e-9);
        q3 = haspud ? zwpud * c.wpud * r2 : (soilw ? R(0.0) : (warm ? R(1.0) : R(0.0)));
        q4 = haspud ? zwpud * c.wipud * r2 : (soilw ? R(0.0) : (warm ? R(0.0) : R(1.0)));
        R zvap = P.hvap + P.cvap * (F.ta - P.tmelt) - P.ch2o * (c.tsoi[0] - P.tmelt);
        R zsub = P.hsub + P.cvap * (F.ta - P.tmelt) - P.cice * (c.tsoi[0] - P.tmelt);
        hvasug = (q1 + q3) * zvap + (q2 + q4) * zsub;
        hvasui = P.hsub + P.cvap * (F.ta - P.tmelt) - P.cice * (c.tsno[0] - P.tmelt);
    }
}

// capacity_shares (stomata.py:566-577) of one big leaf: the capacity-weighted
// leaf area (floored at 1e-12), the leaf area, and whether the capacity shares apply
template <typename R, int N, typename Q>
__device__ __forceinline__ void capacity_group(const int (&idx)[N], const Stat<R>& S, const Q& q, R& twm, R& tf,
                                               bool& on) {
    R tw = R(0.0);
    tf = R(0.0);
#pragma unroll
    for (int i = 0; i < N; ++i) {
        const R f = S(IBIS_STAT_FRAC, idx[i]);
        tw = tw + f * q.vmax(idx[i]);
        tf = tf + f;
    }
    on = tw > R(1.0e-12);
    twm = mx(tw, R(1.0e-12));
}

// drystress (stomata.py:515-562)
template <typename R, typename Q>
__device__ __forceinline__ void soil_stress(const Col<R>& c, const Stat<R>& S, const DevParams<R>& P, const Q& q,
                                            R (&stressu)[NL], R (&stressl)[NL], R& stresstu, R& stresstl) {
    stresstu = R(0.0);
    stresstl = R(0.0);
#pragma unroll
    for (int k = 0; k < NL; ++k) {
        R sw = S(IBIS_STAT_SWILT, k);
        R awc = clip((c.wsoi[k] * (R(1.0) - c.wisoi[k]) - sw) / mx(S(IBIS_STAT_SFIELD, k) - sw, R(1e-10)), R(0.0), R(1.0));
        R zw = clip((R(1.0) - ex(q.stressfac() * awc)) / q.znorm(), R(0.0), R(1.0));
        stressl[k] = zw * P.froot[2 * k + 0];
        stressu[k] = zw * P.froot[2 * k + 1];
        stresstl = stresstl + stressl[k];
        stresstu = stresstu + stressu[k];
    }
}

// Steps 1-9 of timestep_body: soil diagnostics, radiation, interception, the
// three canopy passes (turcof + stomata + turvap), evaporation of intercepted
// water, the bare-story reset and the surface fluxes (loops.py:318-674).
// Leaves tu/ts/tl/tg unclamped in `c` (the ground phase clamps them).
template <typename R, bool SUN_U, bool SUN_L, typename Q>
__device__ __forceinline__ void surface_phase(Col<R>& c, const Forc<R>& F, const Stat<R>& S, const Diag<R>& D,
                                              const DevParams<R>& P, const Q& q, Mid<R>& M) {
    const R eps = P.epsilon;
    const R fi = c.fi;
    const R lai0 = S(IBIS_STAT_LAI, 0), lai1 = S(IBIS_STAT_LAI, 1);
    const R sai0 = S(IBIS_STAT_SAI, 0), sai1 = S(IBIS_STAT_SAI, 1);
    const R fu = S(IBIS_STAT_FU), fl = S(IBIS_STAT_FL);
    R q1, q2, q3, q4, hvasug, hvasui;
    evap_sources(c, F, P, q1, q2, q3, q4, hvasug, hvasui);
    const R consoi0 = layer_conductivity<Q::x3>(c, S, P, 0);

    // ---- 2-3. wet fractions and radiation (loops.py:331-354)
    Rad<R> Rd;
    {
        R fwu, fws, fwl, rlu, rls, rll;
        wet_fraction(c.tu, c.wliqu, c.wsnou, q.wliqumax(), P.wsnoumax, q.fmax(), P, fwu, rlu);
        wet_fraction(c.ts, c.wliqs, c.wsnos, q.wliqsmax(), P.wsnosmax, q.fmax(), P, fws, rls);
        wet_fraction(c.tl, c.wliql, c.wsnol, q.wliqlmax(), P.wsnolmax, q.fmax(), P, fwl, rll);
        radiation(Rd, c, F, S, fwu, fws, fwl, rlu, rls, rll, P);
    }

    // ---- 4-5. precipitation cascade and wet fractions after it (loops.py:359-389)
    Casc<R> C;
    cascade(C, c, F, S, P, q);
    R fwetu, fwets, fwetl, rliqu, rliqs, rliql;
    wet_fraction(c.tu, C.wliqu, C.wsnou, q.wliqumax(), P.wsnoumax, q.fmax(), P, fwetu, rliqu);
    wet_fraction(c.ts, C.wliqs, C.wsnos, q.wliqsmax(), P.wsnosmax, q.fmax(), P, fwets, rliqs);
    wet_fraction(c.tl, C.wliql, C.wsnol, q.wliqlmax(), P.wsnolmax, q.fmax(), P, fwetl, rliql);

    // ---- 6. canopy exchange (loops.py:396-611)
    Aero<R> A;
    R u2, alogu, alogl;
    aero_geometry(A, u2, alogu, alogl, F, S, fi, P);
    R stresstu, stresstl;
    {
        R su_[NL], sl_[NL];
        soil_stress(c, S, P, q, su_, sl_, stresstu, stresstl);
    }
    TvFixed<R> X;
    const R csoi0 = S(IBIS_STAT_CSOI, 0) > R(0.0) ? S(IBIS_STAT_CSOI, 0) : P.csoi_mineral_val;
    const R rhosoi0 = S(IBIS_STAT_RHOSOI, 0) > R(0.0) ? S(IBIS_STAT_RHOSOI, 0) : P.rhosoi_val;
    R chgx, wlgx, wigx;
    {
        X.xu = R(2.0) * lai1 * fu;
        X.xs = R(2.0) * sai1 * fu;
        X.xl = R(2.0) * (lai0 + sai0) * fl * (R(1.0) - fi);
        X.fi = (double)fi;
        X.cog = consoi0 / mx(R(0.5) * P.hsoi[0], eps);
        X.coi = P.consno / mx(R(0.5) * mx(c.hsno[0], P.hsnotop), eps);
        X.zirg = P.zir * cube(c.tg);
        X.ziri = P.zir * cube(c.ti);
        const R p0 = S(IBIS_STAT_POROS, 0), w0 = c.wsoi[0], i0 = c.wisoi[0];
        const R rwp = p0 * P.rhow;
        chgx = P.ch2o * c.wpud + P.cice * c.wipud
             + ((R(1.0) - p0) * csoi0 * rhosoi0 + rwp * (R(1.0) - i0) * w0 * P.ch2o + rwp * i0 * P.cice) * P.hsoi[0];
        wlgx = c.wpud + rwp * (R(1.0) - i0) * w0 * P.hsoi[0];
        wigx = c.wipud + rwp * i0 * P.hsoi[0];
        X.wliqu = C.wliqu; X.wliqs = C.wliqs; X.wliql = C.wliql;
        X.wsnou = C.wsnou; X.wsnos = C.wsnos; X.wsnol = C.wsnol;
        X.chux = P.chu + P.ch2o * C.wliqu + P.cice * C.wsnou;
        X.chsx = P.chs + P.ch2o * C.wliqs + P.cice * C.wsnos;
        X.chlx = P.chl + P.ch2o * C.wliql + P.cice * C.wsnol;
        X.rliqu = rliqu; X.rliqs = rliqs; X.rliql = rliql;
        X.fwetu = fwetu; X.fwets = fwets; X.fwetl = fwetl;
        X.hvasug = hvasug; X.hvasui = hvasui;
        X.tsoi0 = c.tsoi[0]; X.tsno0 = c.tsno[0];
        const R zwp = clip(R(0.5) * (c.wpud + c.wipud) / mx(P.wpudmax, eps), R(0.0), R(0.5));
        const R zws = (R(1.0) - i0) * w0 + i0;
        X.zwtot = zwp + (R(1.0) - zwp) * zws;
        X.swilt0 = S(IBIS_STAT_SWILT, 0);
        X.suction0 = S(IBIS_STAT_SUCTION, 0);
        X.bex0 = S(IBIS_STAT_BEX, 0);
        X.fradu = lai1 > eps ? (Rd.solu + Rd.firu) / (R(2.0) * lai1) : R(0.0);
        X.frads = sai1 > eps ? (Rd.sols + Rd.firs) / (R(2.0) * sai1) : R(0.0);
        X.fradl = (lai0 + sai0) > eps ? (Rd.soll + Rd.firl) / (R(2.0) * (lai0 + sai0)) : R(0.0);
        X.pfluxu = C.pfluxu; X.pfluxs = C.pfluxs; X.pfluxl = C.pfluxl;
        X.solg = Rd.solg; X.soli = Rd.soli; X.firg = Rd.firg; X.firi = Rd.firi; X.firb = Rd.firb;
        X.lai1 = lai1; X.lai0 = lai0; X.lsl0 = lai0 + sai0; X.fu = fu; X.fl = fl;
    }
    const double old[5] = {(double)c.tu, (double)c.ts, (double)c.tl, (double)c.tg, (double)c.ti};
    double Wv[9] = {(double)c.tu, (double)c.ts, (double)c.tl, (double)c.t12, (double)c.t34,
                    (double)c.q12, (double)c.q34, (double)c.tg, (double)c.ti};
    R strat[4] = {R(1.0), R(1.0), R(1.0), R(1.0)};
    R wprev[5] = {R(1.0), R(1.0), R(1.0), R(1.0), R(1.0)};
    Stom<R> st;
    TvOut<R> tv;
    const double ta64 = F.ta, qa64 = F.qa, ps64 = F.ps;
#pragma unroll 1
    for (int it = 0; it < 3; ++it) {
        const bool first = (it == 0);
        const R tu = (R)Wv[0], ts = (R)Wv[1], tl = (R)Wv[2], t12 = (R)Wv[3], t34 = (R)Wv[4];
        const R q12 = (R)Wv[5], q34 = (R)Wv[6], tg = (R)Wv[7], ti = (R)Wv[8];
        Trans<R> T;
        transfer(T, strat, u2, alogu, alogl, A, F, t12, t34, q12, q34, first, P);
        stomata<R, SUN_U, SUN_L>(st, c, tu, tl, t12, t34, q12, q34, T.su, T.sl, F.ps, Rd, fwetu, fwetl, S,
                                 stresstu, stresstl, P, q);
        R wu = weight_veg(tu, (R)X.chux, C.wliqu, C.wsnou, wprev[0], first, P);
        R ws = weight_veg(ts, (R)X.chsx, C.wliqs, C.wsnos, wprev[1], first, P);
        R wl = weight_veg(tl, (R)X.chlx, C.wliql, C.wsnol, wprev[2], first, P);
        R wg = weight_veg(tg, chgx, wlgx, wigx, wprev[3], first, P);
        R wi = weight_snow(ti, c.ti, wprev[4], first, P);
        turvap(Wv, tv, old, T, (double)A.cp, (double)P.tfac, wu, ws, wl, wg, wi, X, st, ta64, qa64, ps64, S, P,
               (double)q.beta_power());
        wprev[0] = wu; wprev[1] = ws; wprev[2] = wl; wprev[3] = wg; wprev[4] = wi;
    }
    const R ti_new = mn((R)Wv[8], P.tmelt);
    const R tg_w = (R)Wv[7];

    // ---- 7-8. evaporation of intercepted water, bare-story reset (loops.py:616-640)
    R tu = (R)Wv[0], ts = (R)Wv[1], tl = (R)Wv[2];
    R wliqu = C.wliqu, wliqs = C.wliqs, wliql = C.wliql, wsnou = C.wsnou, wsnos = C.wsnos, wsnol = C.wsnol;
    evap_intercepted(tu, wliqu, wsnou, rliqu, (R)tv.fvapuw, P.chu, P);
    evap_intercepted(ts, wliqs, wsnos, rliqs, (R)tv.fvaps, P.chs, P);
    evap_intercepted(tl, wliql, wsnol, rliql, (R)tv.fvaplw, P.chl, P);
    {
        R tav = (R(1.0) - fi) * tg_w + fi * ti_new;
        if (lai1 == R(0.0) || fu == R(0.0)) { tu = tav; wliqu = R(0.0); wsnou = R(0.0); }
        if (sai1 == R(0.0) || fu == R(0.0)) { ts = tav; wliqs = R(0.0); wsnos = R(0.0); }
        if (R(2.0) * (lai0 + sai0) == R(0.0) || fl * (R(1.0) - fi) == R(0.0)) { tl = tav; wliql = R(0.0); wsnol = R(0.0); }
    }

    // ---- 9. surface fluxes into soil and snow (loops.py:665-674)
    const R fm = P.flux_max;
    M.fvapg = (R)tv.fvapg;
    M.fvapi = (R)tv.fvapi;
    M.heatg = Rd.solg + clip((R)tv.firg, -fm, fm) - clip((R)tv.fseng, -fm, fm) - hvasug * M.fvapg;
    M.heati = Rd.soli + clip((R)tv.firi, -fm, fm) - clip((R)tv.fseni, -fm, fm) - hvasui * M.fvapi;
    M.fvaput = (R)tv.fvaput;
    M.fvaplt = (R)tv.fvaplt;
    M.ginvap = (R)tv.ginvap;
    M.gsuvap = (R)tv.gsuvap;
    M.gtrans = (R)tv.gtrans;
    M.fsena = (R)tv.fsena;
    M.raing = C.raing; M.traing = C.traing; M.snowg = C.snowg; M.tsnowg = C.tsnowg;
    M.rainl = C.rainl; M.trainl = C.trainl; M.snowl = C.snowl; M.tsnowl = C.tsnowl;
#pragma unroll
    for (int j = 0; j < 2; ++j) { M.an_u[j] = st.an_u[j]; M.ag_u[j] = st.ag_u[j]; }
#pragma unroll
    for (int j = 0; j < 3; ++j) { M.an_l[j] = st.an_l[j]; M.ag_l[j] = st.ag_l[j]; }

    // canopy state left for the ground phase (tu/ts/tl/tg unclamped)
    c.tu = tu; c.ts = ts; c.tl = tl; c.tg = tg_w; c.ti = ti_new;
    c.t12 = (R)Wv[3]; c.t34 = (R)Wv[4]; c.q12 = (R)Wv[5]; c.q34 = (R)Wv[6];
    c.wliqu = wliqu; c.wliqs = wliqs; c.wliql = wliql;
    c.wsnou = wsnou; c.wsnos = wsnos; c.wsnol = wsnol;

    // ---- diagnostics of the surface phase (loops.py:1158-1241)
    if (D.base) {
#pragma unroll
        for (int j = 0; j < 2; ++j) { D.put(IBIS_DIAG_AN_UPPER, j, st.an_u[j]); D.put(IBIS_DIAG_AG_UPPER, j, st.ag_u[j]); }
#pragma unroll
        for (int j = 0; j < 3; ++j) { D.put(IBIS_DIAG_AN_LOWER, j, st.an_l[j]); D.put(IBIS_DIAG_AG_LOWER, j, st.ag_l[j]); }
        D.put(IBIS_DIAG_FWETU, fwetu); D.put(IBIS_DIAG_FWETS, fwets); D.put(IBIS_DIAG_FWETL, fwetl);
        D.put(IBIS_DIAG_RLIQU, rliqu); D.put(IBIS_DIAG_RLIQS, rliqs); D.put(IBIS_DIAG_RLIQL, rliql);
        D.put(IBIS_DIAG_SOLU, Rd.solu); D.put(IBIS_DIAG_SOLS, Rd.sols); D.put(IBIS_DIAG_SOLL, Rd.soll);
        D.put(IBIS_DIAG_SOLG, Rd.solg); D.put(IBIS_DIAG_SOLI, Rd.soli);
        D.put(IBIS_DIAG_FIRU, Rd.firu); D.put(IBIS_DIAG_FIRS, Rd.firs); D.put(IBIS_DIAG_FIRL, Rd.firl);
        D.put(IBIS_DIAG_FIRG, (R)tv.firg); D.put(IBIS_DIAG_FIRI, (R)tv.firi); D.put(IBIS_DIAG_FIRB, (R)tv.firb);
#pragma unroll
        for (int b = 0; b < 2; ++b) { D.put(IBIS_DIAG_ASURD, b, Rd.asurd[b]); D.put(IBIS_DIAG_ASURI, b, Rd.asuri[b]); }
        D.put(IBIS_DIAG_TOPPARU, Rd.topparu); D.put(IBIS_DIAG_TOPPARL, Rd.topparl);
#pragma unroll
        for (int j = 0; j < 4; ++j) { D.put(IBIS_DIAG_SCALCOEFU, j, Rd.scu[j]); D.put(IBIS_DIAG_SCALCOEFL, j, Rd.scl[j]); }
        D.put(IBIS_DIAG_FSENU, (R)tv.fsenu); D.put(IBIS_DIAG_FSENS, (R)tv.fsens); D.put(IBIS_DIAG_FSENL, (R)tv.fsenl);
        D.put(IBIS_DIAG_FSENG, (R)tv.fseng); D.put(IBIS_DIAG_FSENI, (R)tv.fseni);
        D.put(IBIS_DIAG_FVAPG, M.fvapg); D.put(IBIS_DIAG_FVAPI, M.fvapi);
        D.put(IBIS_DIAG_RAING, C.raing); D.put(IBIS_DIAG_SNOWG, C.snowg); D.put(IBIS_DIAG_RHOA, A.rhoa);
        D.put(IBIS_DIAG_HVASUG, hvasug); D.put(IBIS_DIAG_HVASUI, hvasui);
        D.put(IBIS_DIAG_QGLIF, 0, q1); D.put(IBIS_DIAG_QGLIF, 1, q2); D.put(IBIS_DIAG_QGLIF, 2, q3); D.put(IBIS_DIAG_QGLIF, 3, q4);
        D.put(IBIS_DIAG_HEATI, M.heati);
        D.put(IBIS_DIAG_GINVAP, M.ginvap); D.put(IBIS_DIAG_GSUVAP, M.gsuvap); D.put(IBIS_DIAG_GTRANS, M.gtrans);
        D.put(IBIS_DIAG_RAINL, C.rainl); D.put(IBIS_DIAG_SNOWL, C.snowl);
        D.put(IBIS_DIAG_TRAINL, C.trainl); D.put(IBIS_DIAG_TSNOWL, C.tsnowl);
        D.put(IBIS_DIAG_FSENA, M.fsena);
    }
}

// Steps 10-12 of timestep_body -- snow, soil water and heat (+ bedrock),
// freeze/thaw, the surface-temperature bound -- then the fire counters and the
// day-loop accumulators (loops.py:676-1275; loops_gswp3.py:161-318).
template <typename R, int NT, typename Q, int SLD>
__device__ __forceinline__ void ground_phase(Col<R>& c, const Forc<R>& F, const Stat<R>& S, const Diag<R>& D,
                                             const Acc<R, SLD>& Ac, const DevParams<R>& P, const Q& q, const Mid<R>& M) {
    const R eps = P.epsilon, dt = P.dtime;
    const R fi = c.fi;
    const R lai0 = S(IBIS_STAT_LAI, 0), lai1 = S(IBIS_STAT_LAI, 1);
    const R sai0 = S(IBIS_STAT_SAI, 0);
    const R fu = S(IBIS_STAT_FU), fl = S(IBIS_STAT_FL);
    const R tu = c.tu, tl = c.tl;
    R wliql = c.wliql, wsnol = c.wsnol;
    R consoi[NL];
#pragma unroll
    for (int k = 0; k < NL; ++k) consoi[k] = layer_conductivity<Q::x3>(c, S, P, k);
    R q1, q2, q3, q4, hvasug_, hvasui_;
    evap_sources(c, F, P, q1, q2, q3, q4, hvasug_, hvasui_);
    R stressu[NL], stressl[NL], stresstu, stresstl;
    soil_stress(c, S, P, q, stressu, stressl, stresstu, stresstl);

    // ---- 10. snow (loops.py:676-848)
    R smelt, zheat, sflo_bot, fhtop_snow;
    {
        fhtop_snow = M.heati + M.rainl * (P.ch2o * (M.trainl - P.tmelt) + P.hfus + P.cice * (P.tmelt - c.tsno[0]))
                   + M.snowl * P.cice * (M.tsnowl - c.tsno[0]);
        const R xlb = fl * R(2.0) * (lai0 + sai0);
        R hp[NS];
#pragma unroll
        for (int k = 0; k < NS; ++k) hp[k] = c.hsno[k];
        if (fi > R(0.0)) hp[0] = c.hsno[0] + (M.rainl + M.snowl - M.fvapi) * (P.dtime / P.rhos);
        R tsh[NS];
#pragma unroll
        for (int k = 0; k < NS; ++k) tsh[k] = c.tsno[k];
        R tlsub_h = c.tlsub;
        snow_heat(tsh, tlsub_h, sflo_bot, fhtop_snow, xlb, fi, hp, P.hsoi[0], consoi[0], c.tsoi[0], P);
        R ht = R(0.0);
#pragma unroll
        for (int k = 0; k < NS; ++k) ht = ht + hp[k];
        R hts = ht > R(0.0) ? ht : P.hsnomin;
        R dfi = (R(1.0) - fi) * P.dtime * M.snowg / (P.rhos * hts);
        dfi = mn(dfi, R(1.0) - fi);
        R fi1 = fi + dfi;
        R tm[NS], hm[NS];
        const bool fresh = (fi < eps) && (dfi > R(0.0));
#pragma unroll
        for (int k = 0; k < NS; ++k) {
            tm[k] = fi1 > R(0.0) ? (tsh[k] * fi + M.tsnowg * dfi) / mx(fi1, eps) : tsh[k];
            R hinit = k == 0 ? P.hsnotop : (P.hsnomin - P.hsnotop) / R(NS - 1);
            hm[k] = fresh ? hinit : hp[k];
        }
        // snow_melt (snow_physics.py:236-260)
        smelt = R(0.0);
        zheat = R(0.0);
#pragma unroll
        for (int k = 0; k < NS; ++k) {
            R xh = P.rhos * hm[k] * P.cice * mx(tm[k] - P.tmelt, R(0.0));
            R xm = mn(P.rhos * hm[k], xh / P.hfus);
            hm[k] = hm[k] - xm / P.rhos;
            tm[k] = mn(tm[k], P.tmelt);
            smelt = smelt + fi1 * xm;
            zheat = zheat + fi1 * (xh - P.hfus * xm);
        }
        // snow_coverage (snow_physics.py:263-290)
        R ruf = mn(R(0.70), mx(P.hsnomin + R(0.05), fl * S(IBIS_STAT_ZTOP, 0)));
        R htc = R(0.0);
#pragma unroll
        for (int k = 0; k < NS; ++k) htc = htc + hm[k];
        if (htc < R(1e-10)) htc = P.hsnomin;
        const R zhh = R(0.5) * P.hsnomin;
        const R zdh = mx(ruf - P.hsnomin, eps);
        R fic = clip((-zhh + sq(zhh * zhh + zdh * fi1 * htc)) / zdh, R(0.0), P.fimax);
        R scl = fi1 / mx(fic, eps);
#pragma unroll
        for (int k = 0; k < NS; ++k) hm[k] = hm[k] * scl;
        readapt_layers(hm, tm, P.hsnotop, eps);
        // fimin melt-all (loops.py:763-777)
        if (fic < P.fimin) {
            R hsum = R(0.0), heat = R(0.0);
#pragma unroll
            for (int k = 0; k < NS; ++k) {
                hsum = hsum + hm[k];
                heat = heat + P.rhos * hm[k] * fic * (P.cice * (P.tmelt - tm[k]) + P.hfus);
            }
            smelt = smelt + P.rhos * hsum * fic;
            zheat = zheat + (-heat);
#pragma unroll
            for (int k = 0; k < NS; ++k) { hm[k] = R(0.0); tm[k] = P.tmelt; }
            fic = R(0.0);
        }
        // buried vegetation (loops.py:781-830)
        R dfc = fic - fi;
        R tlsub = tlsub_h;
        if (dfc > R(0.0)) {
            tlsub = (tlsub_h * fi + tl * dfc) / mx(fic, eps);
            zheat = zheat + dfc * xlb * (wliql * (P.ch2o * (tl - P.tmelt) + P.hfus + P.cice * (P.tmelt - tm[NS - 1]))
                                         + wsnol * P.cice * (tl - tm[NS - 1]));
            hm[NS - 1] = hm[NS - 1] + dfc * xlb * (wliql + wsnol) / (P.rhos * mx(fic, eps));
        }
        if (dfc < R(0.0)) {
            zheat = zheat - dfc * xlb * P.chl * (tlsub_h - tl);
            R rdec = (R(1.0) - fi) / mx(R(1.0) - fic, eps);
            wliql = wliql * rdec;
            wsnol = wsnol * rdec;
        }
        if (!(fic > R(0.0))) tlsub = tl;
        c.fi = fic;
#pragma unroll
        for (int k = 0; k < NS; ++k) { c.hsno[k] = hm[k]; c.tsno[k] = tm[k]; }
        c.tlsub = tlsub;
        c.wliql = wliql;
        c.wsnol = wsnol;
    }
    const R heatg_avg = (R(1.0) - fi) * M.heatg + fi * sflo_bot + zheat * P.rdt;
    const R fvapg_avg = clip((R(1.0) - fi) * M.fvapg, R(-1.0e-3), R(1.0e-3));
    const R raing_nf = (R(1.0) - fi) * M.raing;
    const R smr = smelt * P.rdt;
    const R rsum = raing_nf + smr;
    const bool rzero = rsum < eps;
    const R raing_avg = rzero ? R(0.0) : rsum;
    const R traing_avg = rzero ? R(0.0) : (raing_nf * M.traing + smr * P.tmelt) / mx(rsum, eps);

    // ---- 11. soil (loops.py:896-1125)
    R poros[NL], csoi[NL], rhosoi[NL];
#pragma unroll
    for (int k = 0; k < NL; ++k) {
        poros[k] = S(IBIS_STAT_POROS, k);
        R cs = S(IBIS_STAT_CSOI, k), rs = S(IBIS_STAT_RHOSOI, k);
        csoi[k] = cs > R(0.0) ? cs : P.csoi_mineral_val;
        rhosoi[k] = rs > R(0.0) ? rs : P.rhosoi_val;
    }
    R grunof = mn(c.wpud, mx(R(0.0), c.wpud + c.wipud - P.wpudmax)) / dt;
    R wpw = c.wpud - grunof * dt;
    const R zfrez = clip((c.tsoi[0] - P.tmelt + R(0.5)) * R(2.0), R(0.0), R(1.0));
    const R zrunf = zfrez * clip((wpw + c.wipud) / P.wpudmax, R(0.0), R(1.0));
    wpw = wpw + (R(1.0) - zrunf) * raing_avg * dt;
    grunof = grunof + zrunf * raing_avg;
    const bool evap = fvapg_avg >= R(0.0);
    const R edt = fvapg_avg * dt;
    const R fwtop = evap ? -q1 * fvapg_avg : R(0.0);
    R wiw = c.wipud;
    if (evap) { wpw = wpw - q3 * edt; wiw = c.wipud - q4 * edt; }
    const R isub = evap ? q2 * edt / mx(P.rhow * poros[0] * P.hsoi[0], eps) : R(0.0);
    const R i0n = mx(R(0.0), c.wisoi[0] - isub);
    const R w0a = (R(1.0) - i0n) > eps ? c.wsoi[0] * (R(1.0) - c.wisoi[0]) / (R(1.0) - i0n) : c.wsoi[0];
    if (!evap) { wpw = wpw - (q1 + q3) * edt; wiw = wiw - (q2 + q4) * edt; }
    wpw = mx(wpw, R(0.0));
    wiw = mx(wiw, R(0.0));
    const R z1w = mx(R(1.0) - i0n, R(0.0));
    const R zdpud = P.rhow * dt * (z1w * z1w) * S(IBIS_STAT_HYDRAUL, 0);
    const R fwpud = mx(R(0.0), mn(wpw, zdpud)) / dt;
    const R c0pud0 = P.ch2o * wpw + P.cice * wiw;
    R wsw[NL], wisw[NL], pflo[NL];
#pragma unroll
    for (int k = 0; k < NL; ++k) { wsw[k] = c.wsoi[k]; wisw[k] = c.wisoi[k]; }
    if (evap) { wsw[0] = w0a; wisw[0] = i0n; }
#pragma unroll
    for (int k = 0; k < NL; ++k) pflo[k] = mx(poros[k] * mx(R(1.0) - wisw[k], eps), eps);
    const R gtransu = M.fvaput * R(2.0) * lai1 * fu;
    const R gtransl = M.fvaplt * R(2.0) * lai0 * fl * (R(1.0) - fi);
    const R sstu = mx(stresstu, eps), sstl = mx(stresstl, eps);
    R tpt[NT], dtp[NL];
#pragma unroll
    for (int k = 0; k < NL; ++k) {
        R wu_ = stresstu >= R(1.0) ? P.froot[2 * k + 1] : stressu[k] / sstu;
        R wl_ = stresstl >= R(1.0) ? P.froot[2 * k + 0] : stressl[k] / sstl;
        R uu = gtransu * wu_;
        R ul = gtransl * wl_;
        wsw[k] = wsw[k] + (-dt * (uu + ul) / (P.rhow * pflo[k] * P.hsoi[k]));
        wsw[k] = mx(wsw[k], R(0.0));
        R c0 = k == 0 ? c0pud0 : R(0.0);
        R cx = c0 + ((R(1.0) - poros[k]) * csoi[k] * rhosoi[k] + poros[k] * (R(1.0) - wisw[k]) * wsw[k] * P.ch2o * P.rhow
                     + poros[k] * wisw[k] * P.cice * P.rhow) * P.hsoi[k];
        dtp[k] = -dt * P.ch2o * (uu * (tu - c.tsoi[k]) + ul * (tl - c.tsoi[k])) / mx(cx, eps);
        tpt[k] = c.tsoi[k] + dtp[k];
    }
    const R fhtop_soil = heatg_avg + raing_avg * P.ch2o * (traing_avg - tpt[0])
                       - grunof * P.ch2o * mx(P.tmelt - tpt[0], R(0.0));
    // soil water (soil_physics.py:196-373): increment form in the FP32 kernels,
    // double in the FP64 kernels
    R wnew[NL], wflo[NL + 1], wpud_h;
    if constexpr (sizeof(R) == 4 && IBIS_SOILW_INCREMENTS) {
#pragma unroll
        for (int k = 0; k < NL; ++k) wnew[k] = wsw[k];
        wpud_h = wpw;
        soil_water_increments(wnew, wpud_h, wflo, wisw, poros, pflo, S, fwtop, fwpud, P);
    } else {
        double w64[NL], i64[NL], p64[NL], pf64[NL], wf64[NL + 1];
#pragma unroll
        for (int k = 0; k < NL; ++k) { w64[k] = wsw[k]; i64[k] = wisw[k]; p64[k] = poros[k]; pf64[k] = pflo[k]; }
        double wp64 = wpw;
        soil_water(w64, wp64, wf64, i64, p64, pf64, S, (double)fwtop, (double)fwpud, P);
#pragma unroll
        for (int k = 0; k < NL; ++k) wnew[k] = (R)w64[k];
#pragma unroll
        for (int k = 0; k <= NL; ++k) wflo[k] = (R)wf64[k];
        wpud_h = (R)wp64;
    }
    const R c1pud0 = P.ch2o * wpud_h + P.cice * wiw;
    R hflo[NL + 1];
    // the solve starts from tsoi + dtp, the increment kept apart (soil_heat)
#pragma unroll
    for (int k = 0; k < NL; ++k) tpt[k] = c.tsoi[k];
#pragma unroll
    for (int k = NL; k < NT; ++k) tpt[k] = c.tsoi_deep[k - NL];
    soil_heat<R, NT>(tpt, hflo, dtp, wsw, wnew, wisw, poros, consoi, csoi, rhosoi, c0pud0, c1pud0, fhtop_soil, wflo,
                     P);
    R gadj = water_bounds(wnew, wisw, poros, P);
    R pflo_ft[NL];
    R tft[NL];
#pragma unroll
    for (int k = 0; k < NL; ++k) tft[k] = tpt[k];
    phase_change(tft, wnew, wisw, pflo_ft, poros, csoi, rhosoi, c1pud0, P);
    R wpud_n = wpud_h, wipud_n = wiw;
    puddle_phase(tft[0], wpud_n, wipud_n, poros[0], wnew[0], wisw[0], csoi[0], rhosoi[0], P);
    gadj = gadj + water_bounds(wnew, wisw, poros, P);
#pragma unroll
    for (int k = 0; k < NL; ++k) { c.tsoi[k] = tft[k]; c.wsoi[k] = wnew[k]; c.wisoi[k] = wisw[k]; }
#pragma unroll
    for (int k = NL; k < NT; ++k) c.tsoi_deep[k - NL] = tpt[k];
    c.wpud = wpud_n;
    c.wipud = wipud_n;

    // ---- 12. surface temperature bound (loops.py:1143-1151)
    const R lo_ = F.ta - P.t_max_dev, hi_ = F.ta + P.t_max_dev;
    c.tu = clip(c.tu, lo_, hi_);
    c.ts = clip(c.ts, lo_, hi_);
    c.tl = clip(c.tl, lo_, hi_);
    c.tg = clip(c.tg, lo_, hi_);
    fire_counters(c, S(IBIS_STAT_SWILT, 0), F, P);

    // ---- diagnostics of the ground phase (loops.py:1158-1241)
    if (D.base) {
#pragma unroll
        for (int k = 0; k < NL; ++k) {
            D.put(IBIS_DIAG_CONSOI, k, consoi[k]);
            D.put(IBIS_DIAG_STRESSU, k, stressu[k]);
            D.put(IBIS_DIAG_STRESSL, k, stressl[k]);
            D.put(IBIS_DIAG_POROSFLO, k, pflo_ft[k]);
        }
#pragma unroll
        for (int k = 0; k <= NL; ++k) D.put(IBIS_DIAG_HFLO, k, hflo[k]);
        D.put(IBIS_DIAG_HEATG, heatg_avg);
        D.put(IBIS_DIAG_STRESSTU, stresstu); D.put(IBIS_DIAG_STRESSTL, stresstl);
        D.put(IBIS_DIAG_GTRANSU, gtransu); D.put(IBIS_DIAG_GTRANSL, gtransl); D.put(IBIS_DIAG_GRUNOF, grunof);
        D.put(IBIS_DIAG_GDRAIN, wflo[NL]); D.put(IBIS_DIAG_GADJUST, gadj); D.put(IBIS_DIAG_WTOT, R(0.0));
        D.put(IBIS_DIAG_RAING_AVG, raing_avg); D.put(IBIS_DIAG_TRAING_AVG, traing_avg);
        D.put(IBIS_DIAG_FHTOP_SOIL, fhtop_soil);
        D.put(IBIS_DIAG_SFLO_BOT, sflo_bot); D.put(IBIS_DIAG_FHTOP_SNOW, fhtop_snow);
    }

    // ---- accumulators of the day loop (loops_gswp3.py:161-318)
    if (Ac.base) {
        if (P.flags & IBIS_FLAG_ACC) {
            const R smask = R(1.0) - c.fi;
            R root_t = R(0.0);
#pragma unroll
            for (int k = 0; k < NL; ++k) root_t = root_t + c.tsoi[k] * R(0.5) * (P.froot[2 * k] + P.froot[2 * k + 1]);
            const R funca = ex(R(3500.0) * (R(1.0 / 288.16) - R(1.0) / mx(c.ts, R(200.0))));
            const R funcb = ex(R(3500.0) * (R(1.0 / 288.16) - R(1.0) / mx(root_t, R(200.0))));
            const R cf = R(12.0e-3) * dt;
            const R sap = S(IBIS_STAT_SAPFRAC);
            // with gpp_split_by_capacity (X3), each big leaf's GPP is divided among
            // its PFTs by leaf area x vmax, re-normalised to the leaf-area sum
            // (capacity_shares, stomata.py:566-577; loops_gswp3.py:197-205)
            R twm[3] = {R(1.0), R(1.0), R(1.0)}, tfs[3] = {R(0.0), R(0.0), R(0.0)};
            bool by_cap[3] = {false, false, false};
            if constexpr (Q::x3) {
                if (P.flags & IBIS_FLAG_GPP_CAPACITY) {
                    capacity_group(kBroadleafPfts, S, q, twm[0], tfs[0], by_cap[0]);
                    capacity_group(kConiferPfts, S, q, twm[1], tfs[1], by_cap[1]);
                    capacity_group(kShrubPfts, S, q, twm[2], tfs[2], by_cap[2]);
                }
            }
            R npp = R(0.0);
#pragma unroll
            for (int j = 0; j < 12; ++j) {
                R an, lai_, cov, sp;
                bool wood = true;
                if (j < 8) {
                    const bool con = (j == 3 || j == 5 || j == 7);
                    an = con ? M.an_u[1] : M.an_u[0];
                    lai_ = lai1; cov = fu; sp = sap;
                } else {
                    an = j < 10 ? M.an_l[0] : (j == 10 ? M.an_l[2] : M.an_l[1]);
                    lai_ = lai0; cov = fl * smask; sp = R(1.0);
                    wood = j < 10;
                }
                R share = S(IBIS_STAT_FRAC, j);
                if constexpr (Q::x3) {
                    const int gi = j < 8 ? ((j == 3 || j == 5 || j == 7) ? 1 : 0) : (j < 10 ? 2 : -1);
                    if (gi >= 0 && by_cap[gi]) share = share * q.vmax(j) / twm[gi] * tfs[gi];
                }
                R g;
                if (j < 8) g = an * share * lai_ * cov;
                else g = an * share * lai_ * fl * smask;
                R r = q.rroot(j) * S(IBIS_STAT_CBIOR, j) * funcb;
                if (wood) r = (j < 8 ? q.rwood(j) * S(IBIS_STAT_CBIOW, j) * sp * funca
                                     : q.rwood(j) * S(IBIS_STAT_CBIOW, j) * funca) + r;
                R inc = q.keep(j) * (g - r) * cf;
                if (Ac.kahan) {
                    Ac.add(IBIS_ACC_AYNPP + j, inc);
                    npp = npp + inc;
                } else {
                    R old_ = Ac.get(IBIS_ACC_AYNPP + j);
                    R nw = old_ + inc;
                    Ac.at(IBIS_ACC_AYNPP + j) = nw;
                    npp = npp + (nw - old_);
                }
            }
            R fb = S(IBIS_STAT_FRAC, 0) + S(IBIS_STAT_FRAC, 1) + S(IBIS_STAT_FRAC, 2) + S(IBIS_STAT_FRAC, 4)
                 + S(IBIS_STAT_FRAC, 6);
            R fcn = S(IBIS_STAT_FRAC, 3) + S(IBIS_STAT_FRAC, 5) + S(IBIS_STAT_FRAC, 7);
            R gu = (M.ag_u[0] * fb + M.ag_u[1] * fcn) * lai1 * fu;
            R gl = (M.ag_l[0] * (S(IBIS_STAT_FRAC, 8) + S(IBIS_STAT_FRAC, 9)) + M.ag_l[2] * S(IBIS_STAT_FRAC, 10)
                    + M.ag_l[1] * S(IBIS_STAT_FRAC, 11)) * lai0 * fl * smask;
            Ac.add(IBIS_ACC_ADRAIN, F.rain * dt);
            Ac.add(IBIS_ACC_ADSNOW, F.snow * dt);
            Ac.add(IBIS_ACC_ADAET, (M.ginvap + M.gsuvap + M.gtrans) * dt);
            Ac.add(IBIS_ACC_A10ANCUB, M.an_u[0] * dt);
            Ac.add(IBIS_ACC_A10ANCLS, M.an_l[0] * dt);
            Ac.add(IBIS_ACC_A10ANCL3, M.an_l[1] * dt);
            Ac.add(IBIS_ACC_A10ANCL4, M.an_l[2] * dt);
            Ac.add(IBIS_ACC_AYNPPTOT, npp);
            Ac.add(IBIS_ACC_AYGPPTOT, (gu + gl) * cf);
            Ac.add(IBIS_ACC_AYTRUNOF, grunof * dt);
            Ac.add(IBIS_ACC_AYTDRAIN, wflo[NL] * dt);
            Ac.add(IBIS_ACC_AFSENA, M.fsena * dt);
            // the optional ET components (loops_gswp3.py:263-272): the fluxes
            // summed into adaet, kept apart, sublimation from the snow cover
            // taken out of soil evaporation
            if (P.flags & IBIS_FLAG_ETPARTS) {
                const R snowsub = M.fvapi * c.fi * dt;
                Ac.add(IBIS_ACC_ET_TRANS, M.gtrans * dt);
                Ac.add(IBIS_ACC_ET_INTERC, M.ginvap * dt);
                Ac.add(IBIS_ACC_ET_SOILEV, M.gsuvap * dt - snowsub);
                Ac.add(IBIS_ACC_ET_SNOWSUB, snowsub);
            }
            // the optional day/night NEE (loops_gswp3.py:274-281): the day's Rh
            // rate spread evenly over the steps less this step's NPP, booked to
            // the night when the sun is below the horizon
            if (P.flags & IBIS_FLAG_NEEPARTS) {
                const R nee = S(IBIS_STAT_TCO2MIC) * cf - npp;
                Ac.add(F.cosz <= R(0.0) ? IBIS_ACC_NEE_NIGHT : IBIS_ACC_NEE_DAY, nee);
            }
            if (Ac.last) {
                Ac.at(IBIS_ACC_STRESSTU_LAST) = stresstu;
                Ac.at(IBIS_ACC_STRESSTL_LAST) = stresstl;
            }
        }
        if (P.flags & IBIS_FLAG_CH4) {
            R rh = S(IBIS_STAT_TCO2MIC) * P.rh_conv;
            const R zo = (P.flags & IBIS_FLAG_ZWT_OBS) ? S(IBIS_STAT_ZWT_OBS) : R(NAN);
            const Ch4Par<R> m = ch4_params((P.flags & IBIS_FLAG_CH4_BANDS) ? S(IBIS_STAT_CH4_BAND) : R(0.0), P, q);
            R flux = methane(S(IBIS_STAT_F_INUND), rh, c.tsoi, c.wsoi, c.wisoi, zo, m, P);
            Ac.add(IBIS_ACC_CH4, flux * P.ch4_w);
        }
        if (P.flags & IBIS_FLAG_SOIL_MEANS) {
#pragma unroll
            for (int k = 0; k < NL; ++k) {
                Ac.add(IBIS_ACC_TSOI_MEAN + k, c.tsoi[k] * P.ch4_w);
                Ac.add(IBIS_ACC_WSOI_MEAN + k, c.wsoi[k] * P.ch4_w);
                Ac.add(IBIS_ACC_WISOI_MEAN + k, c.wisoi[k] * P.ch4_w);
            }
            Ac.add(IBIS_ACC_TG_MEAN, c.tg * P.ch4_w);
        }
    }
}

// One full hourly step of a column in one kernel.
template <typename R, int NT, bool SUN_U, bool SUN_L, typename Q, int SLD>
__device__ __forceinline__ void column_step(Col<R>& c, const Forc<R>& F, const Stat<R>& S, const Diag<R>& D,
                                            const Acc<R, SLD>& Ac, const DevParams<R>& P, const Q& q) {
    Mid<R> M;
    surface_phase<R, SUN_U, SUN_L>(c, F, S, D, P, q, M);
    ground_phase<R, NT>(c, F, S, D, Ac, P, q, M);
}

}  // namespace ibis
