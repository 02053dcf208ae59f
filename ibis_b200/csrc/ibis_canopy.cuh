// Photosynthesis / stomatal conductance and the 9x9 canopy energy-vapour solve.
// Reference: python-port/ibis/physics/stomata.py and canopy_exchange.py:470-811.
#pragma once
#include "ibis_column.cuh"
#include "gauss9_gen.cuh"

#ifndef IBIS_FAST_SAT
#define IBIS_FAST_SAT 0
#endif

namespace ibis {

// ---------------------------------------------------------------------------
// stomata (stomata.py:198-1080)
// ---------------------------------------------------------------------------

template <typename R>
__device__ __forceinline__ R colimit(R j1, R j2, R theta) {
    R b = j1 + j2;
    R c = j1 * j2;
    R disc = mx(b * b - R(4.0) * theta * c, R(0.0));
    R q = R(0.5) * (b + sq(disc)) + R(1.0e-15);
    return mn(q / theta, c / q);
}

template <typename R>
__device__ __forceinline__ void c3_rate(R& ag, R& an, R par, R ci, R vmax, R gst, R kc, R ko, R rdark,
                                        const DevParams<R>& P) {
    R je = par * R(4.59e-06) * P.alpha3 * (ci - gst) / (ci + R(2.0) * gst);
    R jc = vmax * (ci - gst) / (ci + kc * (R(1.0) + P.o2conc / ko));
    R js = vmax / R(2.2);
    ag = colimit(colimit(je, jc, P.theta3), js, P.beta3);
    an = ag - rdark;
}

template <typename R>
__device__ __forceinline__ void c4_rate(R& ag, R& an, R par, R ci, R vmax, R rdark, const DevParams<R>& P) {
    R je = par * R(4.59e-06) * P.alpha4;
    R ji = R(18.0e3) * vmax * ci;
    ag = colimit(colimit(je, vmax, P.theta4), ji, P.beta4);
    an = ag - rdark;
}

// farquhar_c3 / farquhar_c4 with the IBIS 3.0 factors (stomata.py:228-318): the
// big leaf's light-rate factor `jf` (acclim_light; 1 when off), and with `cap`
// the canopy-level co-limitation: the light limit times `fl`, the capacity
// limits and dark respiration times `fc` (cap_scale).
template <typename R>
__device__ __forceinline__ void c3_rate_x(R& ag, R& an, R par, R ci, R vmax, R gst, R kc, R ko, R rdark, R jf,
                                          bool jon, bool cap, R fl, R fc, const DevParams<R>& P) {
    R je = par * R(4.59e-06) * P.alpha3 * (ci - gst) / (ci + R(2.0) * gst);
    if (jon) je = je * jf;
    R jc = vmax * (ci - gst) / (ci + kc * (R(1.0) + P.o2conc / ko));
    R js = vmax / R(2.2);
    if (cap) { je = je * fl; jc = jc * fc; js = js * fc; rdark = rdark * fc; }
    ag = colimit(colimit(je, jc, P.theta3), js, P.beta3);
    an = ag - rdark;
}

template <typename R>
__device__ __forceinline__ void c4_rate_x(R& ag, R& an, R par, R ci, R vmax, R rdark, R jf, bool jon, bool cap, R fl,
                                          R fc, const DevParams<R>& P) {
    R je = par * R(4.59e-06) * P.alpha4;
    if (jon) je = je * jf;
    R jc = vmax;
    R ji = R(18.0e3) * vmax * ci;
    if (cap) { je = je * fl; jc = jc * fc; ji = ji * fc; rdark = rdark * fc; }
    ag = colimit(colimit(je, jc, P.theta4), ji, P.beta4);
    an = ag - rdark;
}

// ---------------------------------------------------------------------------
// IBIS 3.0 big-leaf parameters (stomata.py:566-660; loops.py:218-231, 291-309)
// ---------------------------------------------------------------------------

// The per-PFT factor on vmax: acclimation f_S(acclim_x) of the PFTs in the mask,
// times the frost ramp on the day's mean air temperature, times the cropland
// share's grass capacity.  `vf` says whether the reference forms a factor at all.
template <typename R>
struct PftFactor {
    bool acclim, frost, crop;
    R ax, ff, cf;
    __device__ __forceinline__ bool vf() const { return acclim || crop; }
    __device__ __forceinline__ R at(int p, const DevParams<R>& P) const {
        R f = R(1.0);
        if (acclim) {
            const R m = P.acclim_mask[p];
            const R fs = clip((ax - P.acclim_s0_pft[p]) / P.acclim_smax_pft[p], R(0.0), R(1.0));
            f = R(1.0) - m + m * fs;
            if (frost) f = f * (R(1.0) - m + m * ff);
        }
        if (crop) {
            const R g = R(1.0) + cf * P.crop_inc[p];
            f = acclim ? f * g : g;
        }
        return f;
    }
};

template <typename R>
__device__ __forceinline__ PftFactor<R> pft_factor(const Stat<R>& S, const DevParams<R>& P) {
    PftFactor<R> f;
    f.acclim = (P.flags & IBIS_FLAG_ACCLIM) != 0;
    f.frost = f.acclim && (P.flags & IBIS_FLAG_FROST) != 0;
    f.crop = (P.flags & IBIS_FLAG_CROP) != 0;
    f.ax = f.acclim ? S(IBIS_STAT_ACCLIM_X) : R(0.0);
    f.ff = f.frost ? clip((S(IBIS_STAT_TD) - R(273.16) - P.frost_t0) / (P.frost_t1 - P.frost_t0), R(0.0), R(1.0))
                   : R(1.0);
    f.cf = f.crop ? S(IBIS_STAT_CROPFRAC) : R(0.0);
    return f;
}

// _mix_vmax (stomata.py:580-590): the displayed-LAI-weighted mean of a per-PFT
// value over the PFTs idx[0..N), `fallback` where they have no leaves
template <typename R, int N, typename V>
__device__ __forceinline__ R mix_pft(const int (&idx)[N], const Stat<R>& S, const V& val, R fallback) {
    R tot = R(0.0), sw = R(0.0);
#pragma unroll
    for (int i = 0; i < N; ++i) {
        const R w = S(IBIS_STAT_FRAC, idx[i]);
        tot = tot + w;
        sw = sw + w * val(idx[i]);
    }
    return tot > R(1.0e-6) ? sw / mx(tot, R(1.0e-6)) : fallback;
}

__device__ constexpr int kBroadleafPfts[5] = {0, 1, 2, 4, 6};
__device__ constexpr int kConiferPfts[3] = {3, 5, 7};
__device__ constexpr int kShrubPfts[2] = {8, 9};

// Per-PFT values read by the big-leaf selection: the source's vmax, times the
// PFT factor when EFF; or the per-PFT Ball-Berry slopes of the parameter record
// (coefm_pft is not one of the parameters a calibration run varies).
template <typename R, typename Q, int KIND>
struct PftValue {
    const Q& q;
    const PftFactor<R>& pf;
    const DevParams<R>& P;
    __device__ __forceinline__ R operator()(int p) const {
        if constexpr (KIND == 0) return q.vmax(p);
        else if constexpr (KIND == 1) return pf.vf() ? q.vmax(p) * pf.at(p, P) : q.vmax(p);
        else return P.coefm_pft[p];
    }
};

// _select_vmax_upper / _select_vmax_shrub (stomata.py:592-631) over the values v:
// the priority pick, or with vmax_mix the displayed-LAI-weighted mean
template <typename R, bool LOWER, typename V>
__device__ __forceinline__ void select_big_leaves(R (&out)[LOWER ? 3 : 2], const V& v, const Stat<R>& S, bool mix) {
    if constexpr (!LOWER) {
        R ub = S(IBIS_STAT_EXIST, 0) > R(0.5) ? v(0) : (S(IBIS_STAT_EXIST, 2) > R(0.5) ? v(2) : v(4));
        R uc = S(IBIS_STAT_EXIST, 3) > R(0.5) ? v(3) : v(5);
        if (mix) {
            ub = mix_pft(kBroadleafPfts, S, v, ub);
            uc = mix_pft(kConiferPfts, S, v, uc);
        }
        out[0] = ub;
        out[1] = uc;
    } else {
        R ls = v(8);
        if (mix) ls = mix_pft(kShrubPfts, S, v, ls);
        out[0] = ls;
        out[1] = v(11);
        out[2] = v(10);
    }
}

// Nominal vmax (vn), light-rate factor (jf; jon = whether it applies) and
// Ball-Berry slope (cm) of the upper big leaves [broadleaf, conifer] or, with
// LOWER, of the lower ones [shrub, C3 grass, C4 grass] (stomata.py:592-660, 800-835).
template <typename R, bool LOWER, typename Q>
__device__ __forceinline__ void big_leaves(R (&vn)[LOWER ? 3 : 2], R (&jf)[LOWER ? 3 : 2], R (&cm)[LOWER ? 3 : 2],
                                           bool& jon, const Stat<R>& S, const DevParams<R>& P, const Q& q) {
    constexpr int NLF = LOWER ? 3 : 2;
    const PftFactor<R> pf = pft_factor(S, P);
    const bool mix = (P.flags & IBIS_FLAG_VMAX_MIX) != 0;
    select_big_leaves<R, LOWER>(vn, PftValue<R, Q, 1>{q, pf, P}, S, mix);
    jon = pf.vf() && (P.flags & IBIS_FLAG_ACCLIM_LIGHT) != 0;
    if (jon) {
        R rv[NLF];
        select_big_leaves<R, LOWER>(rv, PftValue<R, Q, 0>{q, pf, P}, S, mix);
#pragma unroll
        for (int j = 0; j < NLF; ++j) jf[j] = vn[j] / mx(rv[j], P.epsilon);
    } else {
#pragma unroll
        for (int j = 0; j < NLF; ++j) jf[j] = R(1.0);
    }
    if (P.flags & IBIS_FLAG_COEFM_MIX) {
        const PftValue<R, Q, 2> cp{q, pf, P};
        if constexpr (!LOWER) {
            cm[0] = mix_pft(kBroadleafPfts, S, cp, q.coefm(0));
            cm[1] = mix_pft(kConiferPfts, S, cp, q.coefm(1));
        } else {
            cm[0] = mix_pft(kShrubPfts, S, cp, q.coefm(2));
            cm[1] = P.coefm_pft[11];
            cm[2] = P.coefm_pft[10];
        }
    } else {
        if constexpr (!LOWER) { cm[0] = q.coefm(0); cm[1] = q.coefm(1); }
        else { cm[0] = q.coefm(2); cm[1] = q.coefm(4); cm[2] = q.coefm(3); }
    }
}

// _capacity_integral (stomata.py:370-375): (1 - e^-Kn L)/(Kn L), 0 without leaves
template <typename R>
__device__ __forceinline__ R capacity_integral(R lai, R kn) {
    const R x = kn * lai;
    const R f = x > R(1.0e-4) ? -em1(-x) / mx(x, R(1.0e-4)) : R(1.0) - R(0.5) * x;
    return lai > R(0.0) ? f : R(0.0);
}

template <typename R>
struct Kin { R kc, ko, gst, vm3, vm4; };

template <typename R>
__device__ __forceinline__ Kin<R> kinetics(R tleaf, const DevParams<R>& P) {
    Kin<R> k;
    R rw = R(3.47e-03) - R(1.0) / tleaf;
    R tau = P.tau15 * ex(R(-4500.0) * rw);
    k.kc = P.kc15 * ex(R(6000.0) * rw);
    k.ko = P.ko15 * ex(R(1500.0) * rw);
    k.gst = P.o2conc / (R(2.0) * tau);
    R tc = tleaf - R(273.16);
    R base = ex(R(3500.0) * rw);
    R hot = R(1.0) + ex(R(0.40) * (tc - R(50.0)));
    k.vm3 = base / ((R(1.0) + ex(R(0.40) * (R(5.0) - tc))) * hot);
    k.vm4 = base / ((R(1.0) + ex(R(0.40) * (R(10.0) - tc))) * hot);
    return k;
}

template <typename R>
__device__ __forceinline__ void ball_berry(R& cs, R& gs, R& ci, R an, R gb, R rh, R m, R b0, R stress, R gmin,
                                           R cmin, R imin, const DevParams<R>& P) {
    R csn = mx(cmin, R(0.5) * (cs + P.co2conc - an / gb));
    R gsn = R(0.5) * (gs + m * an * rh / csn + b0 * stress);
    gsn = mx(gsn, mx(gmin, b0 * stress));
    ci = clip(R(0.5) * (ci + csn - R(1.6) * an / gsn), imin, P.cimax);
    cs = csn;
    gs = gsn;
}

// canopy_scaling (stomata.py:442-512): denominator k*LAI (F77) or, with
// LEAF_ONLY (scale_leaf_only), k*(LAI+SAI)
template <typename R>
__device__ __forceinline__ R light_scaling(R toppar, R k, R h, const R (&sc)[4], R lai, R sai, R& a10s, R& a10d,
                                           const DevParams<R>& P, bool leaf_only = false) {
    R ext = (k * sc[0] + h * sc[1] - h * sc[2]) / mx(sc[3], P.epsilon);
    ext = clip(ext, R(0.1), R(10.0));
    R pxai = ext * (lai + sai);
    R plai = ext * lai;
    bool has = plai > R(0.0);
    bool day = toppar > R(10.0);
    R sday = (R(1.0) - ex(-pxai)) / mx(leaf_only ? pxai : plai, P.epsilon);
    R snight = a10s / mx(a10d, P.epsilon);
    if (has && day) {
        a10s = P.zweight * a10s + (R(1.0) - P.zweight) * sday * toppar;
        a10d = P.zweight * a10d + (R(1.0) - P.zweight) * toppar;
    }
    return has ? (day ? sday : snight) : R(0.0);
}

// integral of exp(-a x) over [0, plai] (stomata.py:436-441)
template <typename R>
__device__ __forceinline__ R e1(R a, R plai) {
    R x = a * plai;
    if (fabs((double)x) < 1.0e-5) return plai * (R(1.0) - R(0.5) * x);
    return -em1(-x) / a;
}

template <typename R>
struct SunShade { R psun, psha, vsun, vsha; };

// sunshade_canopy (stomata.py:395-427)
template <typename R>
__device__ __forceinline__ SunShade<R> sunshade(const R (&sc)[4], R dbeam, R k, R h, R lai, R sai,
                                                const DevParams<R>& P) {
    R plai = mx(lai + sai, P.epsilon);
    R fl = lai > R(0.0) ? lai / plai : R(0.0);
    R ek = e1(k, plai), e2k = e1(R(2.0) * k, plai);
    R tot = mx(sc[0] * ek + sc[1] * e1(h, plai) + sc[2] * e1(-h, plai), R(0.0));
    R sun = sc[0] * e2k + sc[1] * e1(k + h, plai) + sc[2] * e1(k - h, plai) + dbeam * (ek - e2k);
    sun = clip(sun, R(0.0), tot);
    SunShade<R> s;
    s.psun = sun * fl;
    s.psha = (tot - sun) * fl;
    s.vsun = fl * e1(P.cap_kn * fl + k, plai);
    s.vsha = mx(fl * e1(P.cap_kn * fl, plai) - s.vsun, R(0.0));
    return s;
}

template <typename R>
__device__ __forceinline__ R total_conductance(R s, R g) {
    return R(1.0) / (R(1.0) / s + R(1.0 / 0.029) / g);
}

template <typename R>
struct Stom {
    R an_u[2], ag_u[2], an_l[3], ag_l[3];
    R tcub, tcuc, tcls, tcl3, tcl4;
};

// One pass of stomata over the five big leaves.  Updates the carried ci/gs/cs
// and a10 running means in `c`.  SUN_U/SUN_L select the sunlit/shaded canopy;
// a parameter source with Q::x3 adds the IBIS 3.0 switches (vmax and slope
// mixing, acclimation with its light-rate factor and frost ramp, cropland
// capacity, canopy-level capacity scaling, leaf-only light scaling).
template <typename R, bool SUN_U, bool SUN_L, typename Q>
__device__ __forceinline__ void stomata(Stom<R>& o, Col<R>& c, R tu, R tl, R t12, R t34, R q12, R q34, R su,
                                        R sl, R ps, const Rad<R>& Rd, R fwetu, R fwetl, const Stat<R>& S,
                                        R stresstu, R stresstl, const DevParams<R>& P, const Q& q) {
    constexpr bool X3 = Q::x3;
    const R eps = P.epsilon;
    const R lai0 = S(IBIS_STAT_LAI, 0), lai1 = S(IBIS_STAT_LAI, 1);
    const R sai0 = S(IBIS_STAT_SAI, 0), sai1 = S(IBIS_STAT_SAI, 1);
    const bool leaf_only = X3 && (P.flags & IBIS_FLAG_LEAF_ONLY) != 0;
    // ---------------- upper canopy: broadleaf (group 0) and conifer (group 1)
    {
        Kin<R> K = kinetics(tu, P);
        R gmn = R(1.05) * K.gst;
        R gb = clip(su * R(25.5), R(0.1), R(10.0));
        R rh = mx(R(0.30), q12 / mx(qsat(esat(t12), ps), eps));
        R vn[2], jf[2], cm[2];
        bool jon = false;
        if constexpr (X3) {
            big_leaves<R, false>(vn, jf, cm, jon, S, P, q);
        } else {
            vn[0] = S(IBIS_STAT_EXIST, 0) > R(0.5) ? q.vmax(0)
                  : (S(IBIS_STAT_EXIST, 2) > R(0.5) ? q.vmax(2) : q.vmax(4));
            vn[1] = S(IBIS_STAT_EXIST, 3) > R(0.5) ? q.vmax(3) : q.vmax(5);
            cm[0] = q.coefm(0);
            cm[1] = q.coefm(1);
        }
        const bool cap = X3 && !SUN_U && (P.flags & IBIS_FLAG_CAP_SCALE_U) != 0;
        SunShade<R> ss;
        if (SUN_U) ss = sunshade(Rd.scu, Rd.dbeamu, Rd.termu6, Rd.termu7, lai1, sai1, P);
        R ag[2], an[2], ci0[2], vmx[2], rdk[2];
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            R ci = clip(c.ci_u[j], gmn, P.cimax);
            R vmax = vn[j] * K.vm3 * stresstu;
            R rd = P.gamma[j] * vn[j] * K.vm3;
            if constexpr (X3) c3_rate_x(ag[j], an[j], Rd.topparu, ci, vmax, K.gst, K.kc, K.ko, rd, jf[j], jon, false,
                                        R(0.0), R(0.0), P);
            else c3_rate(ag[j], an[j], Rd.topparu, ci, vmax, K.gst, K.kc, K.ko, rd, P);
            R bb = an[j];
            if (SUN_U) {
                R ags, ans, agh, anh;
                if constexpr (X3) {
                    c3_rate_x(ags, ans, ss.psun, ci, vmax * ss.vsun, K.gst, K.kc, K.ko, rd * ss.vsun, jf[j], jon,
                              false, R(0.0), R(0.0), P);
                    c3_rate_x(agh, anh, ss.psha, ci, vmax * ss.vsha, K.gst, K.kc, K.ko, rd * ss.vsha, jf[j], jon,
                              false, R(0.0), R(0.0), P);
                } else {
                    c3_rate(ags, ans, ss.psun, ci, vmax * ss.vsun, K.gst, K.kc, K.ko, rd * ss.vsun, P);
                    c3_rate(agh, anh, ss.psha, ci, vmax * ss.vsha, K.gst, K.kc, K.ko, rd * ss.vsha, P);
                }
                R inv = lai1 > R(0.0) ? R(1.0) / mx(lai1, R(1.0e-6)) : R(0.0);
                ag[j] = (ags + agh) * inv;
                an[j] = (ans + anh) * inv;
                bb = an[j];
            }
            ci0[j] = ci;
            vmx[j] = vmax;
            rdk[j] = rd;
            c.ci_u[j] = ci;
            ball_berry(c.cs_u[j], c.gs_u[j], c.ci_u[j], bb, gb, rh, cm[j], P.coefb[j], stresstu, P.gsmin[j],
                       gmn, gmn, P);
        }
        R scale = light_scaling(Rd.topparu, Rd.termu6, Rd.termu7, Rd.scu, lai1, sai1, c.a10su, c.a10du, P, leaf_only);
        const R fcap = cap ? capacity_integral(lai1, P.cap_kn) : R(0.0);
        R tcs[2];
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            R agc = ag[j], anc = an[j];
            if (cap) c3_rate_x(agc, anc, Rd.topparu, ci0[j], vmx[j], K.gst, K.kc, K.ko, rdk[j], jf[j], jon, true,
                               scale, fcap, P);
            else if (!SUN_U) { agc = ag[j] * scale; anc = an[j] * scale; }
            R csc = mx(gmn, P.co2conc - anc / gb);
            R gsc = mx(mx(P.gsmin[j], P.coefb[j] * stresstu), cm[j] * anc * rh / csc + P.coefb[j] * stresstu);
            tcs[j] = total_conductance(su, gsc);
            o.ag_u[j] = agc * (R(1.0) - fwetu);
            o.an_u[j] = anc * (R(1.0) - fwetu);
        }
        o.tcub = tcs[0];
        o.tcuc = tcs[1];
    }
    // ---------------- lower canopy: shrub (group 2, C3), C3 grass (group 4), C4 grass (group 3)
    {
        Kin<R> K = kinetics(tl, P);
        R gmn = R(1.05) * K.gst;
        R gb = clip(sl * R(25.5), R(0.1), R(10.0));
        R rh = mx(R(0.30), q34 / mx(qsat(esat(t34), ps), eps));
        const int grp[3] = {2, 4, 3};
        R vn[3], jf[3], cm[3];
        bool jon = false;
        if constexpr (X3) {
            big_leaves<R, true>(vn, jf, cm, jon, S, P, q);
        } else {
            vn[0] = q.vmax(8);
            vn[1] = q.vmax(11);
            vn[2] = q.vmax(10);
#pragma unroll
            for (int j = 0; j < 3; ++j) cm[j] = q.coefm(grp[j]);
        }
        const bool cap = X3 && !SUN_L && (P.flags & IBIS_FLAG_CAP_SCALE_L) != 0;
        SunShade<R> ss;
        if (SUN_L) ss = sunshade(Rd.scl, Rd.dbeaml, Rd.terml6, Rd.terml7, lai0, sai0, P);
        R ag[3], an[3], ci0[3], vmx[3], rdk[3];
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const bool c4 = (j == 2);
            const int g = grp[j];
            R ci = clip(c.ci_l[j], c4 ? R(0.0) : gmn, P.cimax);
            R vm = c4 ? K.vm4 : K.vm3;
            R vmax = vn[j] * vm * stresstl;
            R rd = P.gamma[g] * vn[j] * vm;
            if constexpr (X3) {
                if (c4) c4_rate_x(ag[j], an[j], Rd.topparl, ci, vmax, rd, jf[j], jon, false, R(0.0), R(0.0), P);
                else c3_rate_x(ag[j], an[j], Rd.topparl, ci, vmax, K.gst, K.kc, K.ko, rd, jf[j], jon, false, R(0.0),
                               R(0.0), P);
            } else {
                if (c4) c4_rate(ag[j], an[j], Rd.topparl, ci, vmax, rd, P);
                else c3_rate(ag[j], an[j], Rd.topparl, ci, vmax, K.gst, K.kc, K.ko, rd, P);
            }
            R bb = an[j];
            if (SUN_L) {
                R ags, ans, agh, anh;
                if constexpr (X3) {
                    if (c4) {
                        c4_rate_x(ags, ans, ss.psun, ci, vmax * ss.vsun, rd * ss.vsun, jf[j], jon, false, R(0.0),
                                  R(0.0), P);
                        c4_rate_x(agh, anh, ss.psha, ci, vmax * ss.vsha, rd * ss.vsha, jf[j], jon, false, R(0.0),
                                  R(0.0), P);
                    } else {
                        c3_rate_x(ags, ans, ss.psun, ci, vmax * ss.vsun, K.gst, K.kc, K.ko, rd * ss.vsun, jf[j], jon,
                                  false, R(0.0), R(0.0), P);
                        c3_rate_x(agh, anh, ss.psha, ci, vmax * ss.vsha, K.gst, K.kc, K.ko, rd * ss.vsha, jf[j], jon,
                                  false, R(0.0), R(0.0), P);
                    }
                } else if (c4) {
                    c4_rate(ags, ans, ss.psun, ci, vmax * ss.vsun, rd * ss.vsun, P);
                    c4_rate(agh, anh, ss.psha, ci, vmax * ss.vsha, rd * ss.vsha, P);
                } else {
                    c3_rate(ags, ans, ss.psun, ci, vmax * ss.vsun, K.gst, K.kc, K.ko, rd * ss.vsun, P);
                    c3_rate(agh, anh, ss.psha, ci, vmax * ss.vsha, K.gst, K.kc, K.ko, rd * ss.vsha, P);
                }
                R inv = lai0 > R(0.0) ? R(1.0) / mx(lai0, R(1.0e-6)) : R(0.0);
                ag[j] = (ags + agh) * inv;
                an[j] = (ans + anh) * inv;
                bb = an[j];
            }
            ci0[j] = ci;
            vmx[j] = vmax;
            rdk[j] = rd;
            c.ci_l[j] = ci;
            ball_berry(c.cs_l[j], c.gs_l[j], c.ci_l[j], bb, gb, rh, cm[j], P.coefb[g], stresstl, P.gsmin[g],
                       c4 ? R(1.0e-8) : gmn, c4 ? R(0.0) : gmn, P);
        }
        R scale = light_scaling(Rd.topparl, Rd.terml6, Rd.terml7, Rd.scl, lai0, sai0, c.a10sl, c.a10dl, P, leaf_only);
        const R fcap = cap ? capacity_integral(lai0, P.cap_kn) : R(0.0);
        R tcs[3];
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const bool c4 = (j == 2);
            const int g = grp[j];
            R agc = ag[j], anc = an[j];
            if (cap) {
                if (c4) c4_rate_x(agc, anc, Rd.topparl, ci0[j], vmx[j], rdk[j], jf[j], jon, true, scale, fcap, P);
                else c3_rate_x(agc, anc, Rd.topparl, ci0[j], vmx[j], K.gst, K.kc, K.ko, rdk[j], jf[j], jon, true, scale,
                               fcap, P);
            } else if (!SUN_L) {
                agc = ag[j] * scale;
                anc = an[j] * scale;
            }
            R csc = mx(c4 ? R(1.0e-8) : gmn, P.co2conc - anc / gb);
            R gsc = mx(mx(P.gsmin[g], P.coefb[g] * stresstl), cm[j] * anc * rh / csc + P.coefb[g] * stresstl);
            tcs[j] = total_conductance(sl, gsc);
            o.ag_l[j] = agc * (R(1.0) - fwetl);
            o.an_l[j] = anc * (R(1.0) - fwetl);
        }
        o.tcls = tcs[0];
        o.tcl3 = tcs[1];
        o.tcl4 = tcs[2];
    }
}

// ---------------------------------------------------------------------------
// turvap: 9x9 implicit canopy / air / ground / snow system (canopy_exchange.py:470-811)
// Always double.  Unknowns: tu ts tl t12 t34 q12 q34 tg ti.
// ---------------------------------------------------------------------------

// Inputs of turvap that do not change across the three passes (stored in R;
// widened to double where the system is assembled).
template <typename R>
struct TvFixed {
    R xu, xs, xl, fi, chux, chsx, chlx, cog, coi, zirg, ziri;
    R wliqu, wliqs, wliql, wsnou, wsnos, wsnol;
    R rliqu, rliqs, rliql, fwetu, fwets, fwetl;
    R hvasug, hvasui, tsoi0, tsno0;
    R zwtot, swilt0, suction0, bex0;
    R fradu, frads, fradl, pfluxu, pfluxs, pfluxl;
    R solg, soli, firg, firi, firb;
    R lai1, lai0, lsl0, fu, fl;
};

template <typename R>
struct TvOut {
    double fsena, fsenu, fsens, fsenl, fseng, fseni;
    double fvapuw, fvaput, fvaps, fvaplw, fvaplt, fvapg, fvapi;
    double firg, firi, firb, ginvap, gsuvap, gtrans;
};

struct Sat64 { double q, dq; };

// Saturation humidity and its capped derivative at the blended temperature.
// The float kernels evaluate the Lowe polynomials in R (they carry R-precision
// inputs anyway) and widen the result; the float64 kernels stay in double.
template <typename R>
__device__ __forceinline__ Sat64 sat64(double t, double ps) {
    Sat64 s;
#if IBIS_FAST_SAT
    if constexpr (sizeof(R) == 4) {
        const float tf = (float)t, pf = (float)ps;
        const float e = esat(tf);
        const float q = qsat(e, pf);
        s.q = q;
        s.dq = fminf(dqsat(tf, q, e), q * 0.1f);
        return s;
    }
#endif
    double e = esat(t);
    s.q = qsat(e, ps);
    s.dq = fmin(dqsat(t, s.q, e), s.q * 0.1);
    return s;
}

template <typename R>
__device__ __forceinline__ void turvap(double (&W)[9], TvOut<R>& o, const double (&old)[5], const Trans<R>& T,
                                       double cp, double tfac, double wu, double ws, double wl, double wg,
                                       double wi, const TvFixed<R>& X, const Stom<R>& st, double ta, double qa,
                                       double ps, const Stat<R>& S, const DevParams<R>& P, double beta_power) {
    const double eps = (double)P.epsilon, dt = (double)P.dtime;
    const double tmelt = (double)P.tmelt, hvap = (double)P.hvap, hsub = (double)P.hsub;
    const double ch2o = (double)P.ch2o, cice = (double)P.cice, cvap = (double)P.cvap;
    const double tu = wu * W[0] + (1.0 - wu) * old[0];
    const double ts = ws * W[1] + (1.0 - ws) * old[1];
    const double tl = wl * W[2] + (1.0 - wl) * old[2];
    const double tg = wg * W[7] + (1.0 - wg) * old[3];
    const double ti = wi * W[8] + (1.0 - wi) * old[4];
    const double t34 = W[4], q12 = W[5], q34 = W[6];
    const Sat64 Su = sat64<R>(tu, ps), Ss = sat64<R>(ts, ps), Sl = sat64<R>(tl, ps), Sg = sat64<R>(tg, ps),
                Si = sat64<R>(ti, ps);
    const double qu = Su.q, dqu = Su.dq, qs = Ss.q, dqs = Ss.dq, ql = Sl.q, dql = Sl.dq;
    const double qg = Sg.q, dqg = Sg.dq, qi = Si.q, dqi = Si.dq;

    // soil-surface humidity factor (canopy_exchange.py:532-572)
    double hfac;
    if constexpr (sizeof(R) == 4) {
        // float kernels: the matric-potential factor in float (it scales qg only)
        const float psig = -P.grav * X.suction0 * powf(X.zwtot, -X.bex0);
        hfac = (double)expf(psig / (P.rvap * (float)tg));
    } else {
        const double psig = -(double)P.grav * (double)X.suction0 * pow((double)X.zwtot, -(double)X.bex0);
        hfac = exp(psig / ((double)P.rvap * tg));
    }
    const double hfac2 = dv<R>(q34, fmax(qg, eps));
    double betaw = clip(dv<R>((double)X.zwtot - (double)X.swilt0, fmax(1.0 - (double)X.swilt0, eps)), 0.0, 1.0);
    if (beta_power != 1.0) {
        if constexpr (sizeof(R) == 4) betaw = (double)powf((float)betaw, (float)beta_power);   // betaw in [0, 1]
        else betaw = pow(betaw, beta_power);
    }
    double qs1, dqs1;
    if constexpr (sizeof(R) == 4) {
        // float kernels: the canopy-air saturation terms in float, like the
        // five surface saturation terms above (they only weight betaw)
        const float t34f = (float)t34, e34f = esat(t34f);
        const float qs1f = qsat(e34f, (float)ps);
        qs1 = qs1f; dqs1 = dqsat(t34f, qs1f, e34f);
    } else {
        const double e34 = esat(t34);
        qs1 = qsat(e34, ps);
        dqs1 = dqsat(t34, qs1, e34);
    }
    const double xden = cp + dv<R>((double)P.zir * cube(t34), (double)T.sg);
    const double bfac = dv<R>(hvap * dqs1, xden);
    const double betas = dv<R>(betaw, 1.0 + bfac * (1.0 - betaw));
    double qgfac = (betas > 0.0) ? betas * hfac + (1.0 - betas) * hfac2 : hfac2;
    const double qeps = 1.0e-10;
    if (q34 > qg + qeps) qgfac = 1.0;
    const double fwux = (q12 > qu + qeps) ? 1.0 : X.fwetu;
    const double fwsx = (q12 > qs + qeps) ? 1.0 : X.fwets;
    const double fwlx = (q34 > ql + qeps) ? 1.0 : X.fwetl;

    // vapour conductances (canopy_exchange.py:587-618)
    const double su = T.su, ss = T.ss, sl = T.sl, sg = T.sg, si = T.si, cu = T.cu, cl = T.cl;
    const double tb = st.tcub, tc = st.tcuc;
    double fr[12];
#pragma unroll
    for (int j = 0; j < 12; ++j) fr[j] = (double)S(IBIS_STAT_FRAC, j);
    const double suw = fmin(fwux * su, dv<R>(0.8 * (X.wliqu + X.wsnou), fmax(dt * (qu - q12), eps)));
    const double sut = fmax(0.0, (1.0 - fwux) * 0.5 * (tb * fr[0] + tb * fr[1] + tb * fr[2] + tc * fr[3]
                                                      + tb * fr[4] + tc * fr[5] + tb * fr[6] + tb * fr[7]));
    const double hvu = hvap + cvap * (ta - tmelt) - ch2o * (tu - tmelt);
    const double hsu = hsub + cvap * (ta - tmelt) - cice * (tu - tmelt);
    const double suh = suw * (X.rliqu * hvu + (1.0 - X.rliqu) * hsu) + sut * hvu;
    const double ssw = fmin(fwsx * ss, dv<R>(0.8 * (X.wliqs + X.wsnos), fmax(dt * (qs - q12), eps)));
    const double ssh = ssw * (X.rliqs * (hvap + cvap * (ta - tmelt) - ch2o * (ts - tmelt))
                              + (1.0 - X.rliqs) * (hsub + cvap * (ta - tmelt) - cice * (ts - tmelt)));
    const double slw = fmin(fwlx * sl, dv<R>(0.8 * (X.wliql + X.wsnol), fmax(dt * (ql - q34), eps)));
    const double tls = st.tcls, tl3 = st.tcl3, tl4 = st.tcl4;
    const double slt0 = fmax(0.0, (1.0 - fwlx) * 0.5 * (tls * fr[8] + tls * fr[9] + tl4 * fr[10] + tl3 * fr[11]));
    const double slt = dv<R>(slt0 * (double)X.lai0, fmax((double)X.lsl0, eps));
    const double hvl = hvap + cvap * (ta - tmelt) - ch2o * (tl - tmelt);
    const double slh = slw * (X.rliql * hvl + (1.0 - X.rliql) * (hsub + cvap * (ta - tmelt) - cice * (tl - tmelt)))
                     + slt * hvl;

    // matrix and right-hand side (canopy_exchange.py:620-682)
    Sys9 M;
    sys9_zero(M);
    const double rdt = P.rdt64;
    const double fi = X.fi;
    double r2 = su * cp;
    M.a00 = X.chux * rdt + wu * r2 + wu * suh * dqu;
    M.a03 = -r2;
    M.a05 = -suh;
    M.b0 = old[0] * X.chux * rdt - (1.0 - wu) * r2 * tu - suh * (qu - wu * dqu * tu) + X.fradu - X.pfluxu;
    r2 = ss * cp;
    M.a11 = X.chsx * rdt + ws * r2 + ws * ssh * dqs;
    M.a13 = -r2;
    M.a15 = -ssh;
    M.b1 = old[1] * X.chsx * rdt - (1.0 - ws) * r2 * ts - ssh * (qs - ws * dqs * ts) + X.frads - X.pfluxs;
    r2 = sl * cp;
    M.a22 = X.chlx * rdt + wl * r2 + wl * slh * dql;
    M.a24 = -r2;
    M.a26 = -slh;
    M.b2 = old[2] * X.chlx * rdt - (1.0 - wl) * r2 * tl - slh * (ql - wl * dql * tl) + X.fradl - X.pfluxl;
    const double ru = X.xu * su, rs = X.xs * ss;
    M.a30 = -wu * ru;
    M.a31 = -ws * rs;
    M.a33 = cu + cl + ru + rs;
    M.a34 = -cl;
    M.b3 = cu * ta * tfac + (1.0 - wu) * ru * tu + (1.0 - ws) * rs * ts;
    const double rl = X.xl * sl, ri = fi * si;
    M.a42 = -wl * rl;
    M.a43 = -cl;
    M.a44 = cl + rl + (1.0 - fi) * sg + ri;
    M.a47 = -wg * (1.0 - fi) * sg;
    M.a48 = -wi * ri;
    M.b4 = (1.0 - wl) * rl * tl + (1.0 - wg) * (1.0 - fi) * sg * tg + (1.0 - wi) * ri * ti;
    const double ruq = X.xu * (suw + sut), rsq = X.xs * ssw;
    M.a50 = -wu * ruq * dqu;
    M.a51 = -ws * rsq * dqs;
    M.a55 = cu + cl + ruq + rsq;
    M.a56 = -cl;
    M.b5 = cu * qa + ruq * (qu - wu * dqu * tu) + rsq * (qs - ws * dqs * ts);
    const double rlq = X.xl * (slw + slt), rgq = (1.0 - fi) * sg;
    M.a62 = -wl * rlq * dql;
    M.a65 = -cl;
    M.a66 = cl + rlq + rgq + fi * si;
    M.a67 = -wg * rgq * qgfac * dqg;
    M.a68 = -wi * fi * si * dqi;
    M.b6 = rlq * (ql - wl * dql * tl) + rgq * qgfac * (qg - wg * dqg * tg) + fi * si * (qi - wi * dqi * ti);
    double r1 = sg * cp;
    r2 = sg * X.hvasug;
    M.a74 = -r1;
    M.a76 = -r2;
    M.a77 = r1 + r2 * qgfac * dqg + X.cog + X.zirg;
    M.b7 = -r2 * qgfac * (qg - dqg * tg) + X.cog * X.tsoi0 + X.solg + X.firg + X.zirg * old[3];
    r1 = si * cp;
    r2 = si * X.hvasui;
    M.a84 = -r1;
    M.a86 = -r2;
    M.a88 = r1 + r2 * dqi + X.coi + X.ziri;
    M.b8 = -r2 * (qi - dqi * ti) + X.coi * X.tsno0 + X.soli + X.firi + X.ziri * old[4];

    // bare cells: canopy rows pinned to the air (canopy_exchange.py:684-732)
    if ((X.xu + X.xs + X.xl) < eps) {
        M.a00 = 1.0; M.a03 = 0.0; M.a05 = 0.0;
        M.a11 = 1.0; M.a13 = 0.0; M.a15 = 0.0;
        M.a22 = 1.0; M.a24 = 0.0; M.a26 = 0.0;
        M.a30 = 0.0; M.a31 = 0.0; M.a33 = 1.0; M.a34 = 0.0;
        M.a42 = 0.0; M.a43 = 0.0; M.a44 = 1.0; M.a47 = 0.0; M.a48 = 0.0;
        M.a50 = 0.0; M.a51 = 0.0; M.a55 = 1.0; M.a56 = 0.0;
        M.a62 = 0.0; M.a65 = 0.0; M.a66 = 1.0; M.a67 = 0.0; M.a68 = 0.0;
        const double ttf = ta * tfac;
        M.b0 = ttf; M.b1 = ttf; M.b2 = ttf; M.b3 = ttf; M.b4 = ttf;
        M.b5 = qa;
        M.b6 = qa;
        M.b7 = M.b7 + ((X.fradu - X.pfluxu) * X.xu + (X.frads - X.pfluxs) * X.xs + (X.fradl - X.pfluxl) * X.xl);
    }

    double v[9];
    sys9_solve(M, v);
#pragma unroll
    for (int i = 0; i < 9; ++i) W[i] = v[i];
    const double nu = v[0], ns = v[1], nl = v[2], n12 = v[3], n34 = v[4], nq12 = v[5], nq34 = v[6];
    const double ng = v[7], ni = v[8];

    // flux diagnostics (canopy_exchange.py:746-795)
    o.fsena = cp * cu * (ta * tfac - n12);
    o.fsenu = cp * su * (wu * nu + (1.0 - wu) * tu - n12);
    o.fsens = cp * ss * (ws * ns + (1.0 - ws) * ts - n12);
    o.fsenl = cp * sl * (wl * nl + (1.0 - wl) * tl - n12);
    o.fseng = cp * sg * (wg * ng + (1.0 - wg) * tg - n34);
    o.fseni = cp * si * (wi * ni + (1.0 - wi) * ti - n34);
    const double quav = qu + wu * dqu * (nu - tu);
    o.fvapuw = suw * (quav - nq12);
    o.fvaput = fmax(0.0, sut * (quav - nq12));
    o.fvaps = ssw * (qs + ws * dqs * (ns - ts) - nq12);
    const double qlav = ql + wl * dql * (nl - tl);
    o.fvaplw = slw * (qlav - nq34);
    o.fvaplt = fmax(0.0, slt0 * (qlav - nq34));
    o.fvapg = sg * (qgfac * (qg + wg * dqg * (ng - tg)) - nq34);
    o.fvapi = si * (qi + wi * dqi * (ni - ti) - nq34);
    o.firg = X.firg - wg * X.zirg * (ng - old[3]);
    o.firi = X.firi - wi * X.ziri * (ni - old[4]);
    o.firb = X.firb + (1.0 - fi) * wg * X.zirg * (ng - old[3]) + fi * wi * X.ziri * (ni - old[4]);
    o.ginvap = o.fvapuw * X.xu + o.fvaps * X.xs + o.fvaplw * X.xl;
    o.gsuvap = o.fvapg * (1.0 - fi) + o.fvapi * fi;
    o.gtrans = o.fvaput * 2.0 * X.lai1 * X.fu + o.fvaplt * 2.0 * X.lai0 * X.fl * (1.0 - fi);
}

}  // namespace ibis
