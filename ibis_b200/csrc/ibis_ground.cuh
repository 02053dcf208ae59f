// Snow, soil (+ thermal-only bedrock) column solves, fire counters and wetland CH4.
// Reference: python-port/ibis/physics/snow_physics.py, soil_physics.py,
// bedrock.py, fire.py (per-step part) and bgc/methane.py.
#pragma once
#include "ibis_column.cuh"

// 1: the FP32 kernels solve soil water in float for the hour's increments
// (soil_water_increments); 0: in double on absolute contents (soil_water).
#ifndef IBIS_SOILW_INCREMENTS
#define IBIS_SOILW_INCREMENTS 1
#endif

namespace ibis {

// Thomas algorithm (solvers.py:17-83) on N unknowns held in registers.
template <typename T, int N>
__device__ __forceinline__ void thomas(const T (&lo)[N], const T (&di)[N], const T (&up)[N], const T (&r)[N],
                                       T (&x)[N]) {
    T gam[N];
    T alp = rcp(di[0]);
    gam[0] = up[0] * alp;
    x[0] = r[0] * alp;
#pragma unroll
    for (int k = 1; k < N - 1; ++k) {
        alp = rcp(di[k] - lo[k] * gam[k - 1]);
        gam[k] = up[k] * alp;
        x[k] = (r[k] - lo[k] * x[k - 1]) * alp;
    }
    x[N - 1] = (r[N - 1] - lo[N - 1] * x[N - 2]) / (di[N - 1] - lo[N - 1] * gam[N - 2]);
#pragma unroll
    for (int k = N - 2; k >= 0; --k) x[k] = x[k] - gam[k] * x[k + 1];
}

// ---------------------------------------------------------------------------
// snowheat (snow_physics.py:109-229): snow layers + one buried-vegetation node
// ---------------------------------------------------------------------------
template <typename R>
__device__ __forceinline__ void snow_heat(R (&tsno)[NS], R& tlsub, R& sflo_bot, R fhtop, R xl, R fi,
                                          const R (&hsno)[NS], R hsoi0, R consoi0, R tsoi0, const DevParams<R>& P) {
    const R conbur = R(2.0), hfake = R(0.01);
    R con[NS + 2];
    const R rs = R(0.5) / P.consno;
    con[0] = R(0.0);
#pragma unroll
    for (int k = 1; k < NS; ++k) con[k] = R(1.0) / (mx(hsno[k - 1], hfake) * rs + mx(hsno[k], hfake) * rs);
    con[NS] = R(1.0) / (mx(hsno[NS - 1], hfake) * rs + R(0.5) * xl / conbur);
    con[NS + 1] = R(1.0) / (xl * (R(0.5) / conbur) + R(0.5) * hsoi0 / mx(consoi0, R(1e-12)));
    R lo[NS + 1], di[NS + 1], up[NS + 1], r[NS + 1], tn[NS + 1];
    const R rdt = P.dtime / (P.rhos * P.cice);
#pragma unroll
    for (int k = 0; k < NS; ++k) {
        R dt = rdt / mx(hsno[k], hfake);
        lo[k] = -dt * con[k];
        di[k] = R(1.0) + dt * (con[k] + con[k + 1]);
        up[k] = -dt * con[k + 1];
        r[k] = tsno[k];
        if (k == 0) r[k] = r[k] + dt * fhtop;
    }
    R dti = xl * P.chl / P.dtime;
    lo[NS] = -con[NS];
    di[NS] = dti + (con[NS] + con[NS + 1]);
    up[NS] = R(0.0);
    r[NS] = dti * tlsub + con[NS + 1] * tsoi0;
    thomas(lo, di, up, r, tn);
    R s = fhtop;
    const R rh = P.rhos * P.cice / P.dtime;
#pragma unroll
    for (int k = 0; k < NS; ++k) s = s - rh * hsno[k] * (tn[k] - tsno[k]);
    sflo_bot = s - xl * (P.chl / P.dtime) * (tn[NS] - tlsub);
    if (fi > R(0.0)) {
#pragma unroll
        for (int k = 0; k < NS; ++k) tsno[k] = tn[k];
        tlsub = tn[NS];
    }
}

// vadapt (snow_physics.py:27-106)
template <typename R>
__device__ __forceinline__ void readapt_layers(R (&h)[NS], R (&t)[NS], R htop, R eps) {
    R zold[NS + 1];
    zold[0] = R(0.0);
#pragma unroll
    for (int k = 0; k < NS; ++k) zold[k + 1] = zold[k] + h[k];
    R ht = zold[NS];
    if (!(ht > eps)) return;
    bool thick = ht >= R(NS) * htop;
    R h1 = thick ? (ht - htop) / R(NS - 1) : mx(ht / R(NS), eps);
    R hn[NS];
#pragma unroll
    for (int k = 0; k < NS; ++k) hn[k] = h1;
    hn[0] = thick ? htop : h1;
    R znew[NS + 1];
    znew[0] = R(0.0);
#pragma unroll
    for (int k = 0; k < NS; ++k) znew[k + 1] = znew[k] + hn[k];
    R tn[NS];
#pragma unroll
    for (int k = 0; k < NS; ++k) {
        R acc = R(0.0);
#pragma unroll
        for (int ko = 0; ko < NS; ++ko) {
            R ov = mx(mn(zold[ko + 1], znew[k + 1]) - mx(zold[ko], znew[k]), R(0.0));
            acc = acc + t[ko] * ov;
        }
        tn[k] = acc / mx(hn[k], eps);
    }
#pragma unroll
    for (int k = 0; k < NS; ++k) { h[k] = hn[k]; t[k] = tn[k]; }
}

// ---------------------------------------------------------------------------
// soilh2o (soil_physics.py:196-373), always double
// ---------------------------------------------------------------------------
template <typename R>
__device__ __forceinline__ void soil_water(double (&w)[NL], double& wpud, double (&wflo)[NL + 1],
                                           const double (&wisoi)[NL], const double (&poros)[NL],
                                           const double (&pflo)[NL], const Stat<R>& S, double fwtop, double fwpud,
                                           const DevParams<R>& P) {
    const double dmin = 1e-9;
    const double dtime = (double)P.dtime, rhow = (double)P.rhow, eps = (double)P.epsilon;
    const bool consistent = (P.flags & IBIS_FLAG_H2O_CONSISTENT) != 0;
    double e[NL + 1], f[NL + 1], g[NL + 1];
    e[0] = f[0] = g[0] = 0.0;
    f[NL] = g[NL] = 0.0;
    double hyd_prev = (double)S(IBIS_STAT_HYDRAUL, 0);
    double suc_prev = (double)S(IBIS_STAT_SUCTION, 0);
    double bex_prev = (double)S(IBIS_STAT_BEX, 0);
#pragma unroll
    for (int k = 1; k < NL; ++k) {
        const double hyd = (double)S(IBIS_STAT_HYDRAUL, k);
        const double suc = (double)S(IBIS_STAT_SUCTION, k);
        const double bex = (double)S(IBIS_STAT_BEX, k);
        const double wp = P.sw_wp[k], wm = P.sw_wm[k];
        double a = wm * hyd_prev + wp * hyd;
        double b = wm * hyd_prev * suc_prev * bex_prev + wp * hyd * suc * bex;
        double zb = wm * bex_prev + wp * bex;
        int nb = (int)floor(zb + 0.5);
        int m = 2 * nb + 3;
        int nn = nb + 2;
        double ws = consistent ? wp * w[k - 1] + wm * w[k] : wm * w[k - 1] + wp * w[k];
        double wa = fmin(ws, 1.0);
        const double pw1 = ipow(wa, nn - 1);
        double bwn1 = b * pw1;
        double bwn = bwn1 * wa;
        if (bwn < dmin) bwn1 = 0.0;
        bwn = fmax(bwn, dmin);
        double dw, wam1;
        if constexpr (sizeof(R) == 4) {
            dw = (w[k] - w[k - 1]) * P.sw_rhm[k];
            wam1 = pw1 * pw1;                           // wa**(m-1) = (wa**(nn-1))**2
        } else {
            dw = (w[k] - w[k - 1]) / P.sw_hm[k];
            wam1 = ipow(wa, m - 1);
        }
        double ek = (-1.0 + (double)m) * a * (wam1 * wa) + ((0.0 * bwn) - (double)nn * bwn1 * wa) * dw;
        double fk = (double)(-m) * a * wam1 + (double)nn * bwn1 * dw;
        double zi = fmax(0.0, 1.0 - fmax(wisoi[k - 1], wisoi[k]));
        zi = zi * zi;
        e[k] = zi * ek;
        f[k] = zi * fk;
        g[k] = zi * bwn;
        hyd_prev = hyd; suc_prev = suc; bex_prev = bex;
    }
    {
        double wab = fmin(w[NL - 1], 1.0);
        int mb = 2 * (int)floor(bex_prev + 0.5) + 3;
        double zi = fmax(0.0, 1.0 - wisoi[NL - 1]);
        e[NL] = (zi * zi) * (-hyd_prev * ipow(wab, mb) * (double)P.bperm);
    }
    double lo[NL], di[NL], up[NL], r[NL], wn[NL];
#pragma unroll
    for (int k = 0; k < NL; ++k) {
        const double h = (double)P.hsoi[k];
        const double dt = dv<R>(dtime, fmax(pflo[k] * h, 1e-30));
        double d1, d2, d3;
        double rk = w[k] + dt * (e[k + 1] - e[k]);
        if constexpr (sizeof(R) == 4) {
            // the layer geometry as precomputed multipliers
            const double rhb = P.sw_rhb[k];
            d1 = dt * (f[k] * P.sw_c1[k] - g[k] * rhb);
            if (k == 0) rk = rk + dt * (fwtop + fwpud) * P.rrhow64;
            if (k < NL - 1) {
                const double rhp = P.sw_rhp[k];
                d2 = 1.0 + dt * (-f[k + 1] * P.sw_c3[k] + f[k] * P.sw_c5[k] + g[k + 1] * rhp + g[k] * rhb);
                d3 = dt * (-f[k + 1] * P.sw_c6[k] - g[k + 1] * rhp);
            } else {
                d2 = 1.0 + dt * (-f[k + 1] + f[k] * P.sw_c5[k] + g[k] * rhb);
                d3 = 0.0;
            }
        } else {
            const double hm = P.sw_hb[k];
            const int km1 = k > 0 ? k - 1 : 0;
            d1 = dt * (f[k] * 0.5 * h / hm - g[k] / hm);
            if (k == 0) rk = rk + dt * (fwtop + fwpud) / rhow;
            if (k < NL - 1) {
                const double hp = P.sw_hp[k];
                d2 = 1.0 + dt * (-f[k + 1] * 0.5 * (double)P.hsoi[k + 1] / hp + f[k] * 0.5 * (double)P.hsoi[km1] / hm
                                 + g[k + 1] / hp + g[k] / hm);
                d3 = dt * (-f[k + 1] * 0.5 * h / hp - g[k + 1] / hp);
            } else {
                d2 = 1.0 + dt * (-f[k + 1] + f[k] * 0.5 * (double)P.hsoi[km1] / hm + g[k] / hm);
                d3 = 0.0;
            }
        }
        if (k == 0) d1 = 0.0;
        lo[k] = d1; di[k] = d2; up[k] = d3; r[k] = rk;
    }
    thomas(lo, di, up, r, wn);
    wflo[NL] = -rhow * e[NL];
    double fsq = 0.0;
#pragma unroll
    for (int k = NL - 1; k >= 0; --k) {
        double zz = rhow * poros[k] * fmax(eps, 1.0 - wisoi[k]) * (double)P.hsoi[k];
        double wk = wn[k] + dv<R>(dtime * fsq, zz);
        double fsn = dv<R>(fmax(wk - 1.0, 0.0) * zz, dtime);
        wk = fmin(wk, 1.0);
        wflo[k] = wflo[k + 1] + dv<R>((wk - w[k]) * zz, dtime);
        wn[k] = wk;
        fsq = fsn;
    }
    wpud = fmax(wpud + (fsq - fwpud) * dtime, 0.0);
    wflo[0] = wflo[0] + fsq - fwpud;
#pragma unroll
    for (int k = 0; k < NL; ++k) w[k] = wn[k];
}

// The FP32 kernels' soilh2o (soil_physics.py:196-373): the same implicit system
// in float, solved for the hour's increments delta = w_new - w.  Its
// right-hand side holds the flux divergence and the implicit terms applied to
// the current profile, so float32 rounds relative to the hour's change where a
// layer changes slowly, and relative to w where the implicit terms dominate
// (wet, conductive layers), as the float32 state's own storage does.  The
// saturation bound and the upward excess flux work on the increments too.
template <typename R>
__device__ __forceinline__ void soil_water_increments(float (&w)[NL], float& wpud, float (&wflo)[NL + 1],
                                                      const float (&wisoi)[NL], const float (&poros)[NL],
                                                      const float (&pflo)[NL], const Stat<R>& S, float fwtop,
                                                      float fwpud, const DevParams<R>& P) {
    const float dmin = 1e-9f;
    const float dtime = P.dtime, rhow = P.rhow, eps = P.epsilon;
    const bool consistent = (P.flags & IBIS_FLAG_H2O_CONSISTENT) != 0;
    float e[NL + 1], f[NL + 1], g[NL + 1];
    e[0] = f[0] = g[0] = 0.0f;
    f[NL] = g[NL] = 0.0f;
    float hyd_prev = S(IBIS_STAT_HYDRAUL, 0);
    float suc_prev = S(IBIS_STAT_SUCTION, 0);
    float bex_prev = S(IBIS_STAT_BEX, 0);
#pragma unroll
    for (int k = 1; k < NL; ++k) {
        const float hyd = S(IBIS_STAT_HYDRAUL, k);
        const float suc = S(IBIS_STAT_SUCTION, k);
        const float bex = S(IBIS_STAT_BEX, k);
        const float wp = P.sw32_wp[k], wm = P.sw32_wm[k];
        const float a = wm * hyd_prev + wp * hyd;
        const float b = wm * hyd_prev * suc_prev * bex_prev + wp * hyd * suc * bex;
        const float zb = wm * bex_prev + wp * bex;
        const int nb = (int)floorf(zb + 0.5f);
        const int m = 2 * nb + 3;
        const int nn = nb + 2;
        const float ws = consistent ? wp * w[k - 1] + wm * w[k] : wm * w[k - 1] + wp * w[k];
        const float wa = fminf(ws, 1.0f);
        const float pw1 = ipow(wa, nn - 1);
        float bwn1 = b * pw1;
        float bwn = bwn1 * wa;
        if (bwn < dmin) bwn1 = 0.0f;
        bwn = fmaxf(bwn, dmin);
        const float dw = (w[k] - w[k - 1]) * P.sw32_rhm[k];
        const float wam1 = pw1 * pw1;                   // wa**(m-1) = (wa**(nn-1))**2
        const float ek = (float)(m - 1) * a * (wam1 * wa) - (float)nn * bwn1 * wa * dw;
        const float fk = (float)(-m) * a * wam1 + (float)nn * bwn1 * dw;
        float zi = fmaxf(0.0f, 1.0f - fmaxf(wisoi[k - 1], wisoi[k]));
        zi = zi * zi;
        e[k] = zi * ek;
        f[k] = zi * fk;
        g[k] = zi * bwn;
        hyd_prev = hyd; suc_prev = suc; bex_prev = bex;
    }
    {
        const float wab = fminf(w[NL - 1], 1.0f);
        const int mb = 2 * (int)floorf(bex_prev + 0.5f) + 3;
        const float zi = fmaxf(0.0f, 1.0f - wisoi[NL - 1]);
        e[NL] = (zi * zi) * (-hyd_prev * ipow(wab, mb) * P.bperm);
    }
    float lo[NL], di[NL], up[NL], r[NL], dl[NL];
#pragma unroll
    for (int k = 0; k < NL; ++k) {
        const float dt = dtime / fmaxf(pflo[k] * P.hsoi[k], 1e-30f);
        const float rhb = P.sw32_rhb[k];
        float d1 = dt * (f[k] * P.sw32_c1[k] - g[k] * rhb);
        float d2m, d3;                                  // d2m: the diagonal less its 1
        if (k < NL - 1) {
            const float rhp = P.sw32_rhp[k];
            d2m = dt * (-f[k + 1] * P.sw32_c3[k] + f[k] * P.sw32_c5[k] + g[k + 1] * rhp + g[k] * rhb);
            d3 = dt * (-f[k + 1] * P.sw32_c6[k] - g[k + 1] * rhp);
        } else {
            d2m = dt * (-f[k + 1] + f[k] * P.sw32_c5[k] + g[k] * rhb);
            d3 = 0.0f;
        }
        float rk = dt * (e[k + 1] - e[k]) - d2m * w[k];
        if (k == 0) {
            d1 = 0.0f;
            rk = rk + dt * (fwtop + fwpud) / rhow;
        } else {
            rk = rk - d1 * w[k - 1];
        }
        if (k < NL - 1) rk = rk - d3 * w[k + 1];
        lo[k] = d1; di[k] = 1.0f + d2m; up[k] = d3; r[k] = rk;
    }
    thomas(lo, di, up, r, dl);
    wflo[NL] = -rhow * e[NL];
    float fsq = 0.0f;
#pragma unroll
    for (int k = NL - 1; k >= 0; --k) {
        const float zz = rhow * poros[k] * fmaxf(eps, 1.0f - wisoi[k]) * P.hsoi[k];
        float dwk = dl[k] + dtime * fsq / zz;           // w_new - w before the saturation bound
        const float over = (w[k] - 1.0f) + dwk;         // w_new - 1
        const float fsn = fmaxf(over, 0.0f) * zz / dtime;
        if (over > 0.0f) dwk = 1.0f - w[k];
        wflo[k] = wflo[k + 1] + dwk * zz / dtime;
        w[k] = over > 0.0f ? 1.0f : w[k] + dwk;
        fsq = fsn;
    }
    wpud = fmaxf(wpud + (fsq - fwpud) * dtime, 0.0f);
    wflo[0] = wflo[0] + fsq - fwpud;
}

// ---------------------------------------------------------------------------
// soilheat / soilheat_with_bedrock (soil_physics.py:385-490, bedrock.py:88-153)
// NT = 6 (no bedrock) or 9; the first NL layers carry water.
// ---------------------------------------------------------------------------
// The soil heat solve of the FP32 kernels in increment form: the same system
// for delta = T_new - t, whose right-hand side holds only small terms -- the
// heat-capacity change times t, the transpired water's heat, the flux
// divergence, and the conduction of the current temperature differences -- so
// float32 rounds relative to the hour's change, not to the temperature.
template <int NT>
__device__ __forceinline__ void soil_heat_increments(float (&t)[NT], float (&hflo)[NL + 1], const float (&dtp)[NL],
                                                     const float (&owsoi)[NL], const float (&wsoi)[NL],
                                                     const float (&wisoi)[NL], const float (&poros)[NL],
                                                     const float (&consoi)[NL], const float (&csoi)[NL],
                                                     const float (&rhosoi)[NL], float c0pud0, float c1pud0,
                                                     float fhtop, const float (&wflo)[NL + 1],
                                                     const DevParams<float>& P) {
    float h[NT], con[NT + 1], whf[NT + 1], c0[NT], c1[NT], dc[NT], ts[NT];
#pragma unroll
    for (int k = 0; k < NT; ++k) {
        h[k] = k < NL ? P.hsoi[k] : P.hsoi_bed[k - NL];
        ts[k] = k < NL ? t[k] + dtp[k] : t[k];      // the starting temperatures, for the advected heat
    }
    auto cons = [&](int k) -> float { return k < NL ? consoi[k] : P.consoi_bed; };
    con[0] = 0.0f;
    con[NT] = 0.0f;
    whf[0] = wflo[0] * P.ch2o * ts[0];
#pragma unroll
    for (int k = 1; k < NT; ++k) {
        con[k] = 1.0f / (0.5f * (h[k - 1] / fmaxf(cons(k - 1), 1e-12f) + h[k] / fmaxf(cons(k), 1e-12f)));
        if (k < NL) whf[k] = wflo[k] * P.ch2o * ((h[k] * ts[k - 1] + h[k - 1] * ts[k]) / (h[k - 1] + h[k]));
    }
    const float drain = wflo[NL] * P.ch2o * ts[NL - 1];
#pragma unroll
    for (int k = NL; k <= NT; ++k) whf[k] = drain;
#pragma unroll
    for (int k = 0; k < NT; ++k) {
        if (k < NL) {
            const float r1 = (1.0f - poros[k]) * csoi[k] * rhosoi[k];
            const float r2 = poros[k] * (1.0f - wisoi[k]) * P.ch2o * P.rhow;
            const float r3 = poros[k] * wisoi[k] * P.cice * P.rhow;
            c0[k] = (k == 0 ? c0pud0 : 0.0f) + (r1 + r2 * owsoi[k] + r3) * h[k];
            c1[k] = (k == 0 ? c1pud0 : 0.0f) + (r1 + r2 * wsoi[k] + r3) * h[k];
            dc[k] = (k == 0 ? c0pud0 - c1pud0 : 0.0f) + r2 * (owsoi[k] - wsoi[k]) * h[k];   // c0 - c1
        } else {
            c0[k] = c1[k] = P.csoi_bed * P.rhosoi_bed * h[k];
            dc[k] = 0.0f;
        }
    }
    float lo[NT], di[NT], up[NT], r[NT], dl[NT];
#pragma unroll
    for (int k = 0; k < NT; ++k) {
        const float rw = P.dtime / c1[k];
        lo[k] = -rw * con[k];
        di[k] = 1.0f + rw * (con[k] + con[k + 1]);
        up[k] = -rw * con[k + 1];
        // (c0/c1) ts + rw (F - conduction of t) - t, term by term
        float cond = con[k] * (t[k] - (k > 0 ? t[k - 1] : t[k]));
        if (k + 1 < NT) cond = cond + con[k + 1] * (t[k] - t[k + 1]);
        float flux = whf[k] - whf[k + 1] + (k == 0 ? fhtop : 0.0f);
        r[k] = (dc[k] / c1[k]) * t[k] + (c0[k] / c1[k]) * (k < NL ? dtp[k] : 0.0f) + rw * (flux - cond);
    }
    thomas(lo, di, up, r, dl);
    float s = fhtop;
    hflo[0] = s;
#pragma unroll
    for (int k = 0; k < NT; ++k) {
        // (c1 T_new - c0 ts) / dt with T_new = t + delta and ts = t + dtp
        s = s - (c1[k] * dl[k] - dc[k] * t[k] - c0[k] * (k < NL ? dtp[k] : 0.0f)) / P.dtime;
        if (k < NL) hflo[k + 1] = s;
    }
#pragma unroll
    for (int k = 0; k < NT; ++k) t[k] = t[k] + dl[k];
}

// soilheat (soil_physics.py:385-490) or soilheat_with_bedrock (bedrock.py:88-153).
// The FP64 kernels perform the reference's operations on absolute temperatures.
// The FP32 kernels solve for the increments (soil_heat_increments above): on
// absolute temperatures (~280 K, one ulp 3e-5 K) float32 rounds each hour by a
// sizeable part of a deep layer's change (~1e-4 K), and the residue repeats
// while a layer changes slowly -- over a year it cooled the deep column of every
// cell by 0.03-0.09 K against the float64 kernels, and with it the runoff, ET
// and CH4 sums drifted by up to 4e-4.
//
// The layers' starting temperatures are t[k] + dtp[k] (dtp: the heat of the
// transpired water, loops.py:1008-1025), kept apart because in float32 an
// hourly increment below half an ulp of the temperature would be dropped.
template <typename R, int NT>
__device__ __forceinline__ void soil_heat(R (&t)[NT], R (&hflo)[NL + 1], const R (&dtp)[NL], const R (&owsoi)[NL],
                                          const R (&wsoi)[NL], const R (&wisoi)[NL], const R (&poros)[NL],
                                          const R (&consoi)[NL], const R (&csoi)[NL], const R (&rhosoi)[NL],
                                          R c0pud0, R c1pud0, R fhtop, const R (&wflo)[NL + 1],
                                          const DevParams<R>& P) {
    if constexpr (sizeof(R) == 4) {
        soil_heat_increments<NT>(t, hflo, dtp, owsoi, wsoi, wisoi, poros, consoi, csoi, rhosoi, c0pud0, c1pud0, fhtop,
                                 wflo, P);
        return;
    }
    using D = double;
    D h[NT], con[NT + 1], whf[NT + 1], c0[NT], c1[NT], td[NT];
#pragma unroll
    for (int k = 0; k < NT; ++k) {
        h[k] = k < NL ? (D)P.hsoi[k] : (D)P.hsoi_bed[k - NL];
        td[k] = k < NL ? (D)t[k] + (D)dtp[k] : (D)t[k];
    }
    const D ch2o = (D)P.ch2o, dtime = (D)P.dtime;
    auto cons = [&](int k) -> D { return k < NL ? (D)consoi[k] : (D)P.consoi_bed; };
    con[0] = 0.0;
    con[NT] = 0.0;
    whf[0] = (D)wflo[0] * ch2o * td[0];
#pragma unroll
    for (int k = 1; k < NT; ++k) {
        con[k] = dv<R>(1.0, 0.5 * (dv<R>(h[k - 1], fmax(cons(k - 1), 1e-12)) + dv<R>(h[k], fmax(cons(k), 1e-12))));
        if (k < NL) {
            D tav = dv<R>(h[k] * td[k - 1] + h[k - 1] * td[k], h[k - 1] + h[k]);
            whf[k] = (D)wflo[k] * ch2o * tav;
        }
    }
    D drain = (D)wflo[NL] * ch2o * td[NL - 1];
#pragma unroll
    for (int k = NL; k <= NT; ++k) whf[k] = drain;
#pragma unroll
    for (int k = 0; k < NT; ++k) {
        if (k < NL) {
            const D por = (D)poros[k];
            D r1 = (1.0 - por) * (D)csoi[k] * (D)rhosoi[k];
            D r2 = por * (1.0 - (D)wisoi[k]) * ch2o * (D)P.rhow;
            D r3 = por * (D)wisoi[k] * (D)P.cice * (D)P.rhow;
            D pud0 = k == 0 ? (D)c0pud0 : 0.0;
            D pud1 = k == 0 ? (D)c1pud0 : 0.0;
            c0[k] = pud0 + (r1 + r2 * (D)owsoi[k] + r3) * h[k];
            c1[k] = pud1 + (r1 + r2 * (D)wsoi[k] + r3) * h[k];
        } else {
            // bedrock: zero porosity and water, so (1-0) csoi rho plus 0 * 0 terms (bedrock.py:132-150)
            D r1 = (1.0 - 0.0) * (D)P.csoi_bed * (D)P.rhosoi_bed;
            D v = 0.0 + (r1 + 0.0 * 0.0 + 0.0) * h[k];
            c0[k] = v;
            c1[k] = v;
        }
    }
    D lo[NT], di[NT], up[NT], r[NT], tn[NT];
#pragma unroll
    for (int k = 0; k < NT; ++k) {
        D rw = dv<R>(dtime, c1[k]);
        lo[k] = -rw * con[k];
        di[k] = 1.0 + rw * (con[k] + con[k + 1]);
        up[k] = -rw * con[k + 1];
        r[k] = dv<R>(c0[k], c1[k]) * td[k] + rw * (whf[k] - whf[k + 1]);
        if (k == 0) r[k] = r[k] + dv<R>(dtime, c1[k]) * (D)fhtop;
    }
    thomas(lo, di, up, r, tn);
    D s = (D)fhtop;
    hflo[0] = (R)s;
#pragma unroll
    for (int k = 0; k < NT; ++k) {
        s = s - dv<R>(c1[k] * tn[k] - c0[k] * td[k], dtime);
        if (k < NL) hflo[k + 1] = (R)s;
    }
#pragma unroll
    for (int k = 0; k < NT; ++k) t[k] = (R)tn[k];
}

// wadjust (soil_physics.py:147-189); returns the mass adjustment rate
template <typename R>
__device__ __forceinline__ R water_bounds(R (&w)[NL], R (&i)[NL], const R (&poros)[NL], const DevParams<R>& P) {
    const R eps = P.epsilon;
    R tot = R(0.0);
#pragma unroll
    for (int k = 0; k < NL; ++k) {
        R z0 = P.hsoi[k] * poros[k] * P.rhow * ((R(1.0) - i[k]) * w[k] + i[k]);
        R ww = w[k] < eps ? R(0.0) : w[k];
        R ii = i[k] < eps ? R(0.0) : i[k];
        ww = mn(R(1.0), ww);
        ii = mn(R(1.0), ii);
        if (ii >= R(1.0) - eps) ww = R(0.0);
        R z1 = P.hsoi[k] * poros[k] * P.rhow * ((R(1.0) - ii) * ww + ii);
        tot = tot + (z1 - z0);
        w[k] = ww;
        i[k] = ii;
    }
    return tot / P.dtime;
}

// freeze_thaw (soil_physics.py:497-564)
template <typename R>
__device__ __forceinline__ void phase_change(R (&t)[NL], R (&w)[NL], R (&i)[NL], R (&pflo)[NL], const R (&poros)[NL],
                                             const R (&csoi)[NL], const R (&rhosoi)[NL], R c1pud0,
                                             const DevParams<R>& P) {
    const R eps = P.epsilon;
#pragma unroll
    for (int k = 0; k < NL; ++k) {
        R zp = mx(poros[k], eps);
        R c1 = k == 0 ? c1pud0 : R(0.0);
        R rw = c1 / (P.rhow * P.hsoi[k]) + (R(1.0) - zp) * csoi[k] * rhosoi[k] / P.rhow;
        R chav = rw + zp * (R(1.0) - i[k]) * w[k] * P.ch2o + zp * i[k] * P.cice;
        R zw = mn(R(1.0), w[k]);
        R dh = chav * (P.tmelt - t[k]);
        R dw = mn(zp * (R(1.0) - i[k]) * zw, mx(R(0.0), dh / P.hfus));
        R ik = i[k] + dw / zp;
        R wk = w[k] - (dw / zp) * (R(1.0) - zw) / mx(eps, R(1.0) - ik);
        chav = rw + zp * (R(1.0) - ik) * wk * P.ch2o + zp * ik * P.cice;
        R tk = P.tmelt - (dh - P.hfus * dw) / chav;
        dh = chav * (tk - P.tmelt);
        dw = mn(zp * ik, mx(R(0.0), dh / P.hfus));
        ik = ik - dw / zp;
        wk = wk + (dw / zp) * (R(1.0) - wk) / mx(eps, R(1.0) - ik);
        chav = rw + zp * (R(1.0) - ik) * wk * P.ch2o + zp * ik * P.cice;
        t[k] = P.tmelt + (dh - P.hfus * dw) / chav;
        w[k] = wk;
        i[k] = ik;
        pflo[k] = poros[k] * mx(eps, R(1.0) - ik);
    }
}

// puddle_freeze_thaw (soil_physics.py:567-615)
template <typename R>
__device__ __forceinline__ void puddle_phase(R& t0, R& wpud, R& wipud, R poros0, R w0, R i0, R csoi0, R rho0,
                                             const DevParams<R>& P) {
    R rw = ((R(1.0) - poros0) * csoi0 * rho0 + poros0 * (R(1.0) - i0) * w0 * P.ch2o * P.rhow
            + poros0 * i0 * P.cice * P.rhow) * P.hsoi[0];
    R chav = P.ch2o * wpud + P.cice * wipud + rw;
    R dh = chav * (P.tmelt - t0);
    R dw = mn(wpud, mx(R(0.0), dh / P.hfus));
    wipud = wipud + dw;
    wpud = wpud - dw;
    chav = P.ch2o * wpud + P.cice * wipud + rw;
    t0 = P.tmelt - (dh - P.hfus * dw) / chav;
    dh = chav * (t0 - P.tmelt);
    dw = mn(wipud, mx(R(0.0), dh / P.hfus));
    wipud = wipud - dw;
    wpud = wpud + dw;
    chav = P.ch2o * wpud + P.cice * wipud + rw;
    t0 = P.tmelt + (dh - P.hfus * dw) / chav;
    wpud = mx(wpud, R(0.0));
    wipud = mx(wipud, R(0.0));
}

// fire counters (fire.py:88-140, 340-366, 470-514, 583-604)
template <typename R>
__device__ __forceinline__ void fire_counters(Col<R>& c, R swilt0, const Forc<R>& F, const DevParams<R>& P) {
    R nyt = c.nytimes + R(1.0);
    R water = c.wisoi[0] + (R(1.0) - c.wisoi[0]) * c.wsoi[0];
    R frac = (water - swilt0) / (R(1.0) - swilt0);
    R fd = mn(R(1.0), mx(R(0.0), R(-2.0) * (frac - R(0.5))));
    R nn = mx(nyt, R(1.0));
    c.firefac = ((nn - R(1.0)) * c.firefac + fd) / nn;
    c.nytimes = nyt;
    R hit = fd > P.d_crit ? R(1.0) : R(0.0);
    c.nfirestep = c.nfirestep + hit;
    c.sdry = c.sdry + fd * hit;
    R eact = F.qa * F.ps / (R(0.622) + R(0.378) * F.qa);
    R vpd = mx(esat(F.ta) - eact, R(0.0)) / R(1000.0);
    R fl = clip(vpd / P.vpd_ref, R(0.0), R(1.0));
    hit = fl > P.d_crit_vpd ? R(1.0) : R(0.0);
    c.nfirestep_vpd = c.nfirestep_vpd + hit;
    c.sdry_vpd = c.sdry_vpd + fl * hit;
}

// Methane parameters of one cell: the parameter source's (one set per launch,
// or per run), or under IBIS_FLAG_CH4_BANDS the set of the cell's band
// (`band` = the STAT ch4_band value: 0 tropical, 1 temperate, 2 boreal), as
// biome_methane_params gives every cell its band's values (methane.py:521-563).
template <typename R>
struct Ch4Par {
    R sat_crit, z_max, r_ch4, q10p, t_ref, z_wt_max, z_tau, tau_oxid, wtot;
    R wtop[NL];
};

// entry b (0, 1 or 2) of a 3-entry table by selects, so no index into the
// parameter record depends on data
template <typename R>
__device__ __forceinline__ R pick3(const R (&a)[3], int b) { return b == 2 ? a[2] : (b == 1 ? a[1] : a[0]); }

template <typename R, typename Q>
__device__ __forceinline__ Ch4Par<R> ch4_params(R band, const DevParams<R>& P, const Q& q) {
    Ch4Par<R> m;
    if (P.flags & IBIS_FLAG_CH4_BANDS) {
        const int b = band >= R(1.5) ? 2 : (band >= R(0.5) ? 1 : 0);   // NaN: the first band
        m.sat_crit = pick3(P.ch4b_sat_crit, b);
        m.z_max = pick3(P.ch4b_z_max, b);
        m.r_ch4 = pick3(P.ch4b_r_ch4, b);
        m.q10p = pick3(P.ch4b_q10p, b);
        m.t_ref = pick3(P.ch4b_t_ref, b);
        m.z_wt_max = pick3(P.ch4b_z_wt_max, b);
        m.z_tau = pick3(P.ch4b_z_tau, b);
        m.tau_oxid = pick3(P.ch4b_tau_oxid, b);
        m.wtot = pick3(P.ch4b_wtot, b);
#pragma unroll
        for (int k = 0; k < NL; ++k)
            m.wtop[k] = b == 2 ? P.ch4b_wtop[2][k] : (b == 1 ? P.ch4b_wtop[1][k] : P.ch4b_wtop[0][k]);
    } else {
        m.sat_crit = P.sat_crit;
        m.z_max = P.z_max;
        m.r_ch4 = q.r_ch4();
        m.q10p = q.q10p();
        m.t_ref = P.t_ref;
        m.z_wt_max = q.z_wt_max();
        m.z_tau = q.z_tau();
        m.tau_oxid = q.tau_oxid();
        m.wtot = P.ch4_wtot;
#pragma unroll
        for (int k = 0; k < NL; ++k) m.wtop[k] = P.ch4_wtop[k];
    }
    return m;
}

// wetland_water_table (methane.py:233-276): the water table inside the
// inundated fraction, m; a finite observed depth `zwt_obs` replaces it, clipped
// to [0, z_max] (methane.py:366-367).
template <typename R>
__device__ __forceinline__ R wetland_water_table(const R (&w)[NL], const R (&i)[NL], const Ch4Par<R>& m, R zwt_obs) {
    R acc = R(0.0);
#pragma unroll
    for (int k = 0; k < NL; ++k) {
        R th = clip(w[k] * (R(1.0) - i[k]) + i[k], R(0.0), R(1.0));
        acc = acc + th * m.wtop[k];
    }
    R ttop = acc / m.wtot;
    R wet = clip(ttop / mx(m.sat_crit, R(1e-6)), R(0.0), R(1.0));
    R zwt = m.z_wt_max * (R(1.0) - wet);
    return isfinite(zwt_obs) ? clip(zwt_obs, R(0.0), m.z_max) : zwt;
}

// methane_flux (methane.py:233-383), kgC m-2 d-1; zwt_obs NaN: the model's water table
template <typename R>
__device__ __forceinline__ R methane(R f_inund, R rh, const R (&t)[NL], const R (&w)[NL], const R (&i)[NL],
                                     R zwt_obs, const Ch4Par<R>& m, const DevParams<R>& P) {
    R zwt = wetland_water_table(w, i, m, zwt_obs);
    R tt = R(0.0), tw = R(0.0);
#pragma unroll
    for (int k = 0; k < NL; ++k) {
        R below = P.hsoi_bot[k] - mx(zwt, P.hsoi_top[k]);
        R an = clip(below / P.hsoi[k], R(0.0), R(1.0)) * P.hsoi[k];
        R th = t[k] >= R(273.15) ? an : R(0.0);
        tt = tt + th;
        tw = tw + th * t[k];
    }
    R tth = tt > R(1e-12) ? tw / mx(tt, R(1e-12)) : t[0];
    R zp = mx(zwt, R(0.0));
    R rha = mx(rh, R(0.0)) * ex(-zp / mx(m.z_tau, R(1e-6)));
    R q10 = pw(m.q10p, (tth - m.t_ref) / R(10.0));
    R prod = mx(rha, R(0.0)) * m.r_ch4 * q10 * (tth >= R(273.15) ? R(1.0) : R(0.0));
    R area = clip(mx(f_inund, R(0.0)), R(0.0), R(1.0));
    return area * prod * ex(-zp / mx(m.tau_oxid, R(1e-6)));
}

}  // namespace ibis
