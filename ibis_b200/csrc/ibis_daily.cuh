// The daily cadence of the day loop, once per cell and day, around the day's
// 24 hourly steps (python-port/ibis/timestepping/loops_gswp3.py:382-608):
//   day_begin: phenology from the standing 10-day means and the last hour's
//              soil-water stress (physics/phenology.py:89-287), then the daily
//              sums zeroed;
//   day_end:   10-day means and annual sums, the Lloyd-Taylor x WFPS
//              decomposition factors, one day of soil C/N
//              (physics/biogeochem.py:23-243) and the respiration sums.
// With the day parameters' module switches on, day_begin also advances the
// seasonal states (loops_gswp3.py:418-437) and day_end the growing-season
// stress sums (loops_gswp3.py:585-596).  Crop and slot types are off (the
// reference's defaults).  Buffers are the step's planes in R (float or
// double); every operation runs in double.  Constants the reference forms in
// float32 are rounded to float32 here too.
#pragma once
#include "ibis_params.cuh"

namespace ibis {

template <typename R>
struct Planes {
    R* __restrict__ base;
    int ld;
    __device__ __forceinline__ double get(int p) const { return (double)base[(size_t)p * ld]; }
    __device__ __forceinline__ void set(int p, double v) const { base[(size_t)p * ld] = (R)v; }
};

// An accumulator: its plane minus its Kahan compensation plane (zero when the
// step sums without compensation).
template <typename R>
__device__ __forceinline__ double acc_value(const Planes<R>& A, int p) {
    return A.get(p) - A.get(p + IBIS_ACC_COUNT);
}

template <typename R>
__device__ __forceinline__ void acc_zero(const Planes<R>& A, int p) {
    A.set(p, 0.0);
    A.set(p + IBIS_ACC_COUNT, 0.0);
}

// Astronomical day length in hours (state/seasonal.py:56-61): solar
// declination 23.44 deg x sin(2 pi (doy - 81) / 365), the sunrise hour angle,
// clipped for polar day and night.
__device__ __forceinline__ double daylength_hours(double lat, double doy) {
    const double pi = 3.141592653589793;
    const double decl = 0.40910518 * sin(2.0 * pi * (doy - 81.0) / 365.0);
    const double x = fmin(fmax(-tan(lat) * tan(decl), -1.0), 1.0);
    return 24.0 / pi * acos(x);
}

// The seasonal states, once a day before phenology (loops_gswp3.py:418-437):
// acclimation S += (T - S) / tau; the senescence sums of cold degree-days below
// Tb while the day length is decreasing and below Pstart, reset otherwise.
// Returns through sen_u / sen_l whether photoperiod-gated senescence starts.
template <typename R>
__device__ __forceinline__ void seasonal_states(const Planes<R>& D, double td, const IbisDayParams& dp, bool& sen_u,
                                                bool& sen_l) {
    const double tc = td - 273.16, lat = D.get(IBIS_DAYST_LATITUDE);
    const double dl = daylength_hours(lat, dp.jday);
    const bool dec = dl < daylength_hours(lat, dp.jday - 1.0);
    const double x = D.get(IBIS_DAYST_ACCLIM_X);
    const double su = (dec && dl < dp.sen_pstart_u) ? D.get(IBIS_DAYST_SSEN_U) + fmax(dp.sen_tb_u - tc, 0.0) : 0.0;
    const double sl = (dec && dl < dp.sen_pstart_l) ? D.get(IBIS_DAYST_SSEN_L) + fmax(dp.sen_tb_l - tc, 0.0) : 0.0;
    D.set(IBIS_DAYST_ACCLIM_X, x + (tc - x) / dp.acclim_tau);
    D.set(IBIS_DAYST_SSEN_U, su);
    D.set(IBIS_DAYST_SSEN_L, sl);
    sen_u = dp.sen_photoperiod_u != 0.0 && su >= dp.sen_ycrit_u;
    sen_l = dp.sen_photoperiod_l != 0.0 && sl >= dp.sen_ycrit_l;
}

// pheno (phenology.py:89-287); sen_u / sen_l: photoperiod-gated senescence
// (phenology.py:148-150, 170-172)
template <typename R>
__device__ __forceinline__ void phenology(const Planes<R>& S, const Planes<R>& D, double td, double stresstu,
                                          double stresstl, const IbisDayParams& dp, double epsilon, bool sen_u,
                                          bool sen_l) {
    const double tmelt = 273.16, ddfac = 1.0 / dp.ddays;
    const double a10td = D.get(IBIS_DAYST_A10TD);
    const double tthr_u = fmax(fmax(0.0 + tmelt, D.get(IBIS_DAYST_TC) + dp.tthresh_u_offset + tmelt),
                               dp.tthresh_u_abs + tmelt);
    const double gthr_u = dp.gthresh_u_c + tmelt;
    const double agddu = (a10td < gthr_u || sen_u) ? 0.0 : D.get(IBIS_DAYST_AGDDU) + td - gthr_u;
    const double tempu = (a10td < tthr_u || sen_u) ? fmax(0.0, D.get(IBIS_DAYST_TEMPU) - ddfac)
                                                   : fmin(1.0, fmax(0.0, agddu - dp.gdd_thresh_u) / dp.gdd_ramp_u);
    const double tthr_l = dp.tthresh_l_c + tmelt, gthr_l = dp.gthresh_l_c + tmelt;
    const double agddl = (a10td < gthr_l || sen_l) ? 0.0 : D.get(IBIS_DAYST_AGDDL) + td - gthr_l;
    const double templ = (a10td < tthr_l || sen_l) ? fmax(0.0, D.get(IBIS_DAYST_TEMPL) - ddfac)
                                                   : fmin(1.0, fmax(0.0, agddl - dp.gdd_thresh_l) / dp.gdd_ramp_l);
    auto drop = [&](int plane, int anc, double s) {
        const double old = D.get(plane);
        const bool dry = D.get(anc) < dp.drop_thresh || s < dp.drop_stress_thresh;
        return dry ? fmax(dp.drop_floor, old - ddfac) : fmin(1.0, old + ddfac);
    };
    const double dropu = drop(IBIS_DAYST_DROPU, IBIS_DAYST_A10ANCUB, stresstu);
    const double dropls = drop(IBIS_DAYST_DROPLS, IBIS_DAYST_A10ANCLS, stresstl);
    const double dropl4 = drop(IBIS_DAYST_DROPL4, IBIS_DAYST_A10ANCL4, stresstl);
    const double dropl3 = drop(IBIS_DAYST_DROPL3, IBIS_DAYST_A10ANCL3, stresstl);
    double plai[12];
#pragma unroll
    for (int j = 0; j < 12; ++j) plai[j] = D.get(IBIS_DAYST_PLAI + j);
    const double avglaiu = plai[0] + plai[1] * dropu + plai[2] + plai[3] + plai[4] * tempu + plai[5]
                         + plai[6] * tempu + plai[7] * tempu;
    const double au = fmax(avglaiu, epsilon);
    S.set(IBIS_STAT_FRAC + 0, plai[0] / au);
    S.set(IBIS_STAT_FRAC + 1, plai[1] * dropu / au);
    S.set(IBIS_STAT_FRAC + 2, plai[2] / au);
    S.set(IBIS_STAT_FRAC + 3, plai[3] / au);
    S.set(IBIS_STAT_FRAC + 4, plai[4] * tempu / au);
    S.set(IBIS_STAT_FRAC + 5, plai[5] / au);
    S.set(IBIS_STAT_FRAC + 6, plai[6] * tempu / au);
    S.set(IBIS_STAT_FRAC + 7, plai[7] * tempu / au);
    const double m9 = fmin(templ, dropls), m10 = fmin(templ, dropl4), m11 = fmin(templ, dropl3);
    const double avglail = plai[8] + plai[9] * m9 + plai[10] * m10 + plai[11] * m11;
    const double al = fmax(avglail, epsilon);
    S.set(IBIS_STAT_FRAC + 8, plai[8] / al);
    S.set(IBIS_STAT_FRAC + 9, plai[9] * m9 / al);
    S.set(IBIS_STAT_FRAC + 10, plai[10] * m10 / al);
    S.set(IBIS_STAT_FRAC + 11, plai[11] * m11 / al);
    const double lai_lower = fmin(avglail / fmax(S.get(IBIS_STAT_FL), epsilon), 12.0);
    const double lai_upper = fmin(avglaiu / fmax(S.get(IBIS_STAT_FU), epsilon), 12.0);
    S.set(IBIS_STAT_LAI + 0, lai_lower);
    S.set(IBIS_STAT_LAI + 1, lai_upper);
    const double zbot1 = S.get(IBIS_STAT_ZBOT + 1);
    S.set(IBIS_STAT_ZBOT + 0, 0.05);
    S.set(IBIS_STAT_ZTOP + 0, fmin(fmax(0.25, lai_lower * 0.25), zbot1 - 0.5));
    D.set(IBIS_DAYST_TEMPU, tempu); D.set(IBIS_DAYST_TEMPL, templ);
    D.set(IBIS_DAYST_AGDDU, agddu); D.set(IBIS_DAYST_AGDDL, agddl);
    D.set(IBIS_DAYST_DROPU, dropu); D.set(IBIS_DAYST_DROPLS, dropls);
    D.set(IBIS_DAYST_DROPL3, dropl3); D.set(IBIS_DAYST_DROPL4, dropl4);
}

// Lloyd-Taylor temperature factor and WFPS moisture factor (loops_gswp3.py:509-520),
// with the float32 constants of the reference rounded as it rounds them.
__device__ __forceinline__ double decomp_temp(double t, double tconst) {
    const double tzero = (double)227.13f;
    const double safe = fmax(t, (double)(227.13f + 10.0f));
    const double inv_b = (double)(1.0f / (288.16f - 227.13f));
    return fmin(exp(tconst * (inv_b - 1.0 / (safe - tzero))), 10.0);
}

__device__ __forceinline__ double decomp_moist(double w, double i, double wshift) {
    const double wfps = (1.0 - i) * w * 100.0 - wshift;
    const double wet = (double)0.000371f * wfps * wfps - (double)0.0748f * wfps + (double)4.13f;
    const double dry = exp((wfps - 60.0) * (wfps - 60.0) / -800.0);
    return wfps >= 60.0 ? wet : dry;
}

__device__ __forceinline__ double clip_d(double x, double lo, double hi) { return fmin(fmax(x, lo), hi); }

// soilbgc (biogeochem.py:23-243), one call per day; returns tco2mic.
template <typename R>
__device__ __forceinline__ double soil_bgc(const Planes<R>& D, const Planes<R>& S, const double* hsoi,
                                           const IbisDayParams& b, double ndaypy) {
    const double* cnr = b.cnr;
    const double totts = 1.0 / ndaypy;
    auto split = [&](double cn, int last, double& fm, double& fs, double& fl) {
        fl = b.bgc_fmax * cn * cn / (b.rconst + cn * cn);
        fs = (1.0 / cn - fl / cnr[4] - (1.0 - fl) / cnr[6]) / (1.0 / cnr[last] - 1.0 / cnr[6]);
        fm = 1.0 - fl - fs;
    };
    double fraclm, fracls, fracll, fracrm, fracrs, fracrl, fracwm, fracws, fracwl;
    split(b.cnleaf, 5, fraclm, fracls, fracll);
    split(b.cnroot, 5, fracrm, fracrs, fracrl);
    split(b.cnwood, 7, fracwm, fracws, fracwl);
    const double rdepth = 1.0 / (hsoi[0] + hsoi[1] + hsoi[2] + hsoi[3]);
    double texsum = 0.0;
#pragma unroll
    for (int k = 0; k < 4; ++k) texsum += 0.01 * S.get(IBIS_STAT_SAND + k) * hsoi[k];
    const double texfact = texsum * rdepth;
    const double fbpom = 0.50;
    const double falll = D.get(IBIS_DAYST_FALLL), fallr = D.get(IBIS_DAYST_FALLR), fallw = D.get(IBIS_DAYST_FALLW);
    const double totcin = (falll + fallr + fallw) * totts;
    double clitlm = D.get(IBIS_DAYST_CLITLM), clitls = D.get(IBIS_DAYST_CLITLS), clitll = D.get(IBIS_DAYST_CLITLL);
    double clitrm = D.get(IBIS_DAYST_CLITRM), clitrs = D.get(IBIS_DAYST_CLITRS), clitrl = D.get(IBIS_DAYST_CLITRL);
    double clitwm = D.get(IBIS_DAYST_CLITWM), clitws = D.get(IBIS_DAYST_CLITWS), clitwl = D.get(IBIS_DAYST_CLITWL);
    const double slop = D.get(IBIS_DAYST_CSOISLOP), slon = D.get(IBIS_DAYST_CSOISLON), pas = D.get(IBIS_DAYST_CSOIPAS);
    const double cmic = D.get(IBIS_DAYST_TOTCMIC);
    const double totcbegin = clitlm + clitls + clitrm + clitrs + clitwm + clitws + slop + slon + pas + cmic + clitll
                           + clitrl + clitwl;
    const double cmicmx = b.fbsom * totcbegin;
    const double cmicp = fmin(cmic, cmicmx), cmicn = fmax(0.0, cmic - cmicmx);
    clitlm = clitlm + fraclm * falll * totts;
    clitls = clitls + fracls * falll * totts;
    clitll = clitll + fracll * falll * totts;
    clitrm = clitrm + fracrm * fallr * totts;
    clitrs = clitrs + fracrs * fallr * totts;
    clitrl = clitrl + fracrl * fallr * totts;
    clitwm = clitwm + fracwm * fallw * totts;
    clitws = clitws + fracws * fallw * totts;
    clitwl = clitwl + fracwl * fallw * totts;
    const double dl = D.get(IBIS_DAYST_DECOMPL), ds = D.get(IBIS_DAYST_DECOMPS);
    const double outcrs = fmin(ds * b.krs * clitrs, clitrs), outcws = fmin(dl * b.kws * clitws, clitws);
    const double outcls = fmin(dl * b.kls * clitls, clitls), outclm = fmin(dl * b.klm * clitlm, clitlm);
    const double outcrm = fmin(ds * b.krm * clitrm, clitrm), outcwm = fmin(dl * b.kwm * clitwm, clitwm);
    const double outcnb = fmin(ds * b.knb * slon, slon), outcpb = fmin(ds * b.kpb * slop, slop);
    const double outcsb = fmin(ds * b.ksb * pas, pas);
    const double outcbp = fmin(b.kbp * cmicp, cmicp) * b.effac, outcbn = fmin(b.kbn * cmicn, cmicn) * b.effac;
    const double dbdt = outcrs * b.yrs + outcws * b.yws + outcls * b.yls + outclm * b.ylm + outcrm * b.yrm
                      + outcwm * b.ywm + outcnb * b.ynb + outcpb * b.ypb + outcsb * b.ysb - outcbp - outcbn;
    const double outcll = fmin(dl * b.kll * clitll, clitll), outcrl = fmin(ds * b.krl * clitrl, clitrl);
    const double outcwl = fmin(dl * b.kwl * clitwl, clitwl), outcns = fmin(ds * b.kns * slon, slon);
    const double lig = b.lig_frac * (outcll * b.yll + outcrl * b.yrl + outcwl * b.ywl);
    double dcndt = lig + (1.0 - fbpom) * (b.ybn * outcbn + b.ybp * outcbp) - outcnb - outcns;
    const double outcps = fmin(ds * b.kps * slop, slop);
    double dcpdt = lig + fbpom * (b.ybn * outcbn + b.ybp * outcbp) - outcpb - outcps;
    const double fleach = 0.30e-03 / 18.0 * (0.01 + 0.04 * texfact);
    const double dcsdt = (b.yns * outcns + b.yps * outcps) - outcsb - fleach * pas;
    const double cleach = fleach * (pas + slop + slon);
    D.set(IBIS_DAYST_YNLEACH, D.get(IBIS_DAYST_YNLEACH) + fleach * pas / cnr[1] + fleach * slop / cnr[2]
                                  + fleach * slon / cnr[3]);
    dcndt = dcndt - fleach * slon;
    dcpdt = dcpdt - fleach * slop;
    D.set(IBIS_DAYST_YRLEACH, D.get(IBIS_DAYST_YRLEACH) + cleach);
    // net mineralisation (+) or immobilisation (-) of the nine microbial
    // fluxes, summed left to right in the reference's order
    double mins[9], imms[9];
    {
        const double ys[9] = {b.yrs, b.yls, b.yws, b.ywm, b.ylm, b.yrm, b.ynb, b.ypb, b.ysb};
        const double ct[9] = {cnr[5], cnr[5], cnr[7], cnr[7], cnr[6], cnr[6], cnr[3], cnr[2], cnr[1]};
        const double fl[9] = {outcrs, outcls, outcws, outcwm, outclm, outcrm, outcnb, outcpb, outcsb};
#pragma unroll
        for (int q = 0; q < 9; ++q) {
            const double net = (1.0 / ct[q] - ys[q] / cnr[0]) * fl[q];
            const bool up = ys[q] / cnr[0] > 1.0 / ct[q];
            mins[q] = up ? 0.0 : net;
            imms[q] = up ? net : 0.0;
        }
    }
    const double totimm = imms[0] + imms[1] + imms[2] + imms[3] + imms[4] + imms[5] + imms[6] + imms[7] + imms[8];
    const double totmin = mins[0] + mins[1] + mins[2] + mins[3] + mins[4] + mins[5] + mins[6] + mins[7] + mins[8];
    const double nrelps = outcps * (1.0 / cnr[2] - 1.0 / cnr[1]);
    const double nrelns = outcns * (1.0 / cnr[3] - 1.0 / cnr[1]);
    const double nrelbn = (1.0 - fbpom) * outcbn * (1.0 / cnr[0] - 1.0 / cnr[3])
                        + (1.0 - fbpom) * outcbp * (1.0 / cnr[0] - 1.0 / cnr[3]);
    const double nrelbp = fbpom * outcbp * (1.0 / cnr[0] - 1.0 / cnr[2]) + fbpom * outcbn * (1.0 / cnr[0] - 1.0 / cnr[2]);
    auto lr = [&](double o) {
        return b.lig_frac * o * (1.0 / cnr[4] - 1.0 / cnr[2]) + b.lig_frac * o * (1.0 / cnr[4] - 1.0 / cnr[3]);
    };
    const double totnrel = nrelps + nrelns + nrelbn + nrelbp + lr(outcll) + lr(outcrl) + lr(outcwl);
    const double netmin = totmin + totimm + totnrel;
    const double tnmin = fmax(0.0, netmin) / (86400.0 * 0.014);
    const double totcmic = fmax(0.0, cmic + dbdt);
    const double slon_n = fmax(0.0, slon + dcndt), slop_n = fmax(0.0, slop + dcpdt), pas_n = fmax(0.0, pas + dcsdt);
    clitlm = fmax(0.0, clitlm - outclm); clitls = fmax(0.0, clitls - outcls); clitll = fmax(0.0, clitll - outcll);
    clitrm = fmax(0.0, clitrm - outcrm); clitrs = fmax(0.0, clitrs - outcrs); clitrl = fmax(0.0, clitrl - outcrl);
    clitwm = fmax(0.0, clitwm - outcwm); clitws = fmax(0.0, clitws - outcws); clitwl = fmax(0.0, clitwl - outcwl);
    const double totlit = clitlm + clitls + clitll + clitrm + clitrs + clitrl + clitwm + clitws + clitwl;
    const double totalit = clitlm + clitls + clitwm + clitll + clitws + clitwl;
    const double totrlit = clitrm + clitrs + clitrl;
    const double totcsoi = pas_n + slop_n + totcmic + slon_n;
    D.set(IBIS_DAYST_CLITLM, clitlm); D.set(IBIS_DAYST_CLITLS, clitls); D.set(IBIS_DAYST_CLITLL, clitll);
    D.set(IBIS_DAYST_CLITRM, clitrm); D.set(IBIS_DAYST_CLITRS, clitrs); D.set(IBIS_DAYST_CLITRL, clitrl);
    D.set(IBIS_DAYST_CLITWM, clitwm); D.set(IBIS_DAYST_CLITWS, clitws); D.set(IBIS_DAYST_CLITWL, clitwl);
    D.set(IBIS_DAYST_CSOIPAS, pas_n); D.set(IBIS_DAYST_CSOISLON, slon_n); D.set(IBIS_DAYST_CSOISLOP, slop_n);
    D.set(IBIS_DAYST_TOTCMIC, totcmic);
    D.set(IBIS_DAYST_TOTLIT, totlit); D.set(IBIS_DAYST_TOTALIT, totalit); D.set(IBIS_DAYST_TOTRLIT, totrlit);
    D.set(IBIS_DAYST_TOTCSOI, totcsoi); D.set(IBIS_DAYST_TOTFALL, falll + fallr + fallw);
    D.set(IBIS_DAYST_TNMIN, tnmin);
    D.set(IBIS_DAYST_STOREDN, D.get(IBIS_DAYST_STOREDN) + tnmin);
    return (totcbegin + totcin - (totlit + totcsoi) - cleach) / (86400.0 * 0.012);
}

// Per-run constants of the day kernels.
struct DayConst {
    double hsoi[6];
    double ndaypy;
    double epsilon;
};

template <typename R>
__global__ void __launch_bounds__(128) day_begin_kernel(R* stat, R* dayst, R* acc, const R* td, int ncell, int ld,
                                                        const IbisDayParams dp, const DayConst c) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ncell) return;
    const Planes<R> S{stat + i, ld}, D{dayst + i, ld}, A{acc + i, ld};
    bool sen_u = false, sen_l = false;
    if (dp.seasonal_on != 0.0) {
        seasonal_states(D, (double)td[i], dp, sen_u, sen_l);
        // the day's hourly steps read the acclimation state from their STAT plane
        // (IBIS_FLAG_ACCLIM), as the reference's steps read state.seasonal.acclim_x
        S.set(IBIS_STAT_ACCLIM_X, D.get(IBIS_DAYST_ACCLIM_X));
    }
    phenology(S, D, (double)td[i], A.get(IBIS_ACC_STRESSTU_LAST), A.get(IBIS_ACC_STRESSTL_LAST), dp, c.epsilon, sen_u,
              sen_l);
    const int sums[7] = {IBIS_ACC_ADRAIN, IBIS_ACC_ADSNOW, IBIS_ACC_ADAET, IBIS_ACC_A10ANCUB, IBIS_ACC_A10ANCLS,
                         IBIS_ACC_A10ANCL3, IBIS_ACC_A10ANCL4};
#pragma unroll
    for (int q = 0; q < 7; ++q) acc_zero(A, sums[q]);
}

template <typename R>
__global__ void __launch_bounds__(128) day_end_kernel(const R* prog, R* stat, R* dayst, const R* acc, const R* td,
                                                      int ncell, int ld, const IbisDayParams dp, const DayConst c) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ncell) return;
    const Planes<R> S{stat + i, ld}, D{dayst + i, ld};
    const Planes<R> A{const_cast<R*>(acc) + i, ld}, G{const_cast<R*>(prog) + i, ld};
    const double zweight = exp(-1.0 / 10.0), alpha10 = 1.0 - zweight, day_sec = 86400.0;
    D.set(IBIS_DAYST_A10TD, zweight * D.get(IBIS_DAYST_A10TD) + alpha10 * (double)td[i]);
    const int means[4] = {IBIS_DAYST_A10ANCUB, IBIS_DAYST_A10ANCLS, IBIS_DAYST_A10ANCL3, IBIS_DAYST_A10ANCL4};
    const int sums[4] = {IBIS_ACC_A10ANCUB, IBIS_ACC_A10ANCLS, IBIS_ACC_A10ANCL3, IBIS_ACC_A10ANCL4};
#pragma unroll
    for (int q = 0; q < 4; ++q)
        D.set(means[q], zweight * D.get(means[q]) + alpha10 * (acc_value(A, sums[q]) / day_sec));
    D.set(IBIS_DAYST_AYPRCP, D.get(IBIS_DAYST_AYPRCP) + acc_value(A, IBIS_ACC_ADRAIN) + acc_value(A, IBIS_ACC_ADSNOW));
    D.set(IBIS_DAYST_AYAET, D.get(IBIS_DAYST_AYAET) + acc_value(A, IBIS_ACC_ADAET));
    // decomposition factors (loops_gswp3.py:494-562): top layer, and the
    // thickness-weighted mean of the top four
    const double* h = c.hsoi;
    const double tconst = (double)(float)dp.lt_e0, wshift = dp.wfps_opt - 60.0;
    const double lo = (double)0.001f, hi = (double)10.0f;
    D.set(IBIS_DAYST_DECOMPL, clip_d(decomp_temp(G.get(IBIS_PROG_TSOI), tconst)
                                     * decomp_moist(G.get(IBIS_PROG_WSOI), G.get(IBIS_PROG_WISOI), wshift) * dp.k_scale,
                                     lo, hi));
    const double h4 = h[0] + h[1] + h[2] + h[3];
    auto avg = [&](int plane) {
        return (G.get(plane) * h[0] + G.get(plane + 1) * h[1] + G.get(plane + 2) * h[2] + G.get(plane + 3) * h[3]) / h4;
    };
    D.set(IBIS_DAYST_DECOMPS, clip_d(decomp_temp(avg(IBIS_PROG_TSOI), tconst)
                                     * decomp_moist(avg(IBIS_PROG_WSOI), avg(IBIS_PROG_WISOI), wshift) * dp.k_scale,
                                     lo, hi));
    const double tco2mic = soil_bgc(D, S, c.hsoi, dp, c.ndaypy);
    S.set(IBIS_STAT_TCO2MIC, tco2mic);
    // heterotrophic and root respiration sums (loops_gswp3.py:575-584)
    const double conv = (double)(float)(12.0e-3 * 86400.0);
    D.set(IBIS_DAYST_AYCO2MIC, D.get(IBIS_DAYST_AYCO2MIC) + tco2mic * conv);
    D.set(IBIS_DAYST_AYCO2ROOT, D.get(IBIS_DAYST_AYCO2ROOT) + D.get(IBIS_DAYST_TCO2ROOT) * conv);
    // growing-season soil-water stress sums from the day's last hour
    // (loops_gswp3.py:585-596): days warmer than tmelt + stress_accum_tmin
    if (dp.stress_on != 0.0) {
        const double grow = (double)td[i] > 273.16 + dp.stress_accum_tmin ? 1.0 : 0.0;
        D.set(IBIS_DAYST_AYSTRESSU, D.get(IBIS_DAYST_AYSTRESSU) + A.get(IBIS_ACC_STRESSTU_LAST) * grow);
        D.set(IBIS_DAYST_AYSTRESSL, D.get(IBIS_DAYST_AYSTRESSL) + A.get(IBIS_ACC_STRESSTL_LAST) * grow);
        D.set(IBIS_DAYST_STRESS_NDAY, D.get(IBIS_DAYST_STRESS_NDAY) + grow);
    }
}

}  // namespace ibis
