// Daily weather -> hourly forcing on the device.
//
// Device form of the reference's `compute_precip_timing` and `diurnal`
// (python-port/ibis/physics/weather.py:395-443, 483-601): the day's
// precipitation event from two variates, then per hour the solar geometry and
// direct/diffuse split (Friend transmissivity), the Campbell-Norman Fourier
// temperature cycle, humidity capped at 99 % saturation, EPIC wind from one
// variate, Idso longwave (or the observed daily value) and the rain/snow split
// of the event; optionally an observed hourly shortwave in place of the
// generator's (observed_shortwave, weather.py:458-481).  The reference draws its variates from jax.random; these are
// counter-based (the SplitMix64 finalizer of Steele, Lea and Flood 2014 over
// (seed, day, slot) and the cell), so any hour of any cell can be regenerated
// without state.  FP32 arithmetic, with the day's orbital terms in double.
#pragma once
#include <stdint.h>

#include "ibis_column.cuh"

namespace ibis {

__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// 24-bit variate k in [0, 2^24): the fraction k / 2^24 is exact in float.
__device__ __forceinline__ uint32_t draw24(uint32_t seed, uint32_t cell, uint32_t day, uint32_t slot) {
    const uint64_t c = ((uint64_t)seed << 32) | ((uint64_t)(day & 0xFFFFFFu) << 8) | (slot & 0xFFu);
    return (uint32_t)(mix64(mix64(c) ^ (uint64_t)cell) >> 40);
}

struct Event { float plens, startp, endp; };

// compute_precip_timing (weather.py:395-443).  The variates enter as 24-bit
// integers: floor(u * n) is formed exactly as (k * n) >> 24.
__device__ __forceinline__ Event precip_timing(uint32_t k_plen, uint32_t k_start, float precip, float dtime) {
    const int niter = (int)(86400.0f / dtime);
    const int plenmin = 1 + (int)((4.0f * 3600.0f - 1.0f) / dtime);
    const int plenmax = max((int)(24.0f * 3600.0f / dtime), plenmin);
    int plen = plenmin + (int)(((uint64_t)k_plen * (uint64_t)(plenmax - plenmin + 1)) >> 24);
    plen = min(max(plen, plenmin), plenmax);
    const int needed = (int)ceil((double)precip / 15.0);
    plen = min(max(max(plen, needed), plenmin), plenmax);
    const int max_start = max(0, niter - plen);
    const int start = min((int)(((uint64_t)k_start * (uint64_t)(max_start + 1)) >> 24), max_start);
    Event e;
    e.plens = dtime * (float)plen;
    e.startp = dtime * (float)start;
    e.endp = e.startp + e.plens;
    return e;
}

// Orbital terms of one day (weather.py:448-455, 521-535), in double.
struct DayGeom { float sindecl, cosdecl, sw; };

__device__ __forceinline__ DayGeom day_geometry(int jday) {
    const double pi = 3.14159265358979323846;
    const double orbit = 2.0 * pi * jday / 365.2425;
    const double decl = 0.006918 - 0.399912 * cos(orbit) + 0.070257 * sin(orbit) - 0.006758 * cos(2.0 * orbit)
                      + 0.000907 * sin(2.0 * orbit) - 0.002697 * cos(3.0 * orbit) + 0.001480 * sin(3.0 * orbit);
    DayGeom g;
    g.sindecl = (float)sin(decl);
    g.cosdecl = (float)cos(decl);
    g.sw = (float)(1370.0 * (1.000110 + 0.034221 * cos(orbit) + 0.001280 * sin(orbit) + 0.000719 * cos(2.0 * orbit)
                             + 0.000077 * sin(2.0 * orbit)));
    return g;
}

struct DailyRec { float tmax, tmin, cloud, precip, psurf, qd, ud, fira; };

// The hour starting `time` seconds after midnight (weather.py:503-601).
__device__ __forceinline__ Forc<float> diurnal_hour(const DailyRec& d, const DayGeom& g, float sinlat, float coslat,
                                                    float time, const Event& ev, uint32_t k_wind, float dtime,
                                                    bool observed_fira) {
    const float pi = 3.14159265f;
    const float rtime = time / 3600.0f;
    const float angle = 2.0f * pi * (rtime - 12.0f) / 24.0f;
    Forc<float> F;
    F.cosz = fmaxf(0.0f, sinlat * g.sindecl + coslat * g.cosdecl * cosf(angle));
    const float trans = 0.251f + 0.509f * (1.0f - d.cloud);
    const float fdiff = trans > 0.75f ? 0.166f
                      : 1.0045f + 0.0435f * trans - 3.5227f * trans * trans + 2.6313f * trans * trans * trans;
    const float base = g.sw * F.cosz * trans;
    F.sd[0] = base * 0.46f * (1.0f - fdiff);
    F.sd[1] = base * 0.54f * (1.0f - fdiff);
    F.si[0] = base * 0.46f * fdiff;
    F.si[1] = base * 0.54f * fdiff;
    const float gamma = 0.44f - 0.46f * sinf(pi / 12.0f * rtime + 0.9f) + 0.11f * sinf(2.0f * pi / 12.0f * rtime + 0.9f);
    F.ta = d.tmax * gamma + d.tmin * (1.0f - gamma);
    F.ps = d.psurf;
    const float qmin = fminf(d.qd, 0.99f * qsat(esat(d.tmin), d.psurf));
    const float qmax = (d.qd - 0.56f * qmin) / 0.44f;
    const float qsa = 0.99f * qsat(esat(F.ta), d.psurf);
    F.qa = fminf(qsa, qmax * gamma + qmin * (1.0f - gamma));
    const float u = fmaxf((float)k_wind * (1.0f / 16777216.0f), 1e-10f);
    F.ua = fminf(fmaxf(1.13989f * d.ud * powf(-logf(u), 0.30f), 2.5f), 10.0f);
    if (observed_fira) {
        F.fira = d.fira;
    } else {
        const float emb = 0.01f * (d.psurf * F.qa / (0.622f + F.qa));
        const float ea = 0.70f + 5.95e-5f * emb * expf(1500.0f / F.ta);
        const float t4 = F.ta * F.ta * F.ta * F.ta * 5.67e-8f;
        F.fira = (1.0f - d.cloud) * ea * t4 + d.cloud * 0.950f * t4;
    }
    const bool in_event = time >= ev.startp && time < ev.endp;
    const bool warm = (F.ta - 273.15f) > 2.5f;
    const float rate = d.precip / fmaxf(ev.plens, dtime);
    F.rain = in_event && warm ? rate : 0.0f;
    F.snow = in_event && !warm ? rate : 0.0f;
    return F;
}

// observed_shortwave (weather.py:458-481): an observed hourly total `sw_obs`
// split into direct and diffuse by the hourly clearness-index relation of
// Spitters et al. (1986), all diffuse with the sun down, then into the two
// bands; `s0` is the day's effective solar constant.
__device__ __forceinline__ void observed_shortwave(float sw_obs, float s0, Forc<float>& F) {
    const float cz = F.cosz;
    const float kt = fminf(fmaxf(sw_obs / fmaxf(s0 * cz, 1.0f), 0.0f), 1.0f);
    const float r = 0.847f - 1.61f * cz + 1.04f * cz * cz;
    const float kk = (1.47f - r) / 1.66f;
    float fd = kt <= 0.22f ? 1.0f
             : kt <= 0.35f ? 1.0f - 6.4f * (kt - 0.22f) * (kt - 0.22f)
             : kt <= kk    ? 1.47f - 1.66f * kt
                           : r;
    fd = cz <= 0.0f ? 1.0f : fminf(fmaxf(fd, 0.0f), 1.0f);
    const float sw = fmaxf(sw_obs, 0.0f);
    F.sd[0] = sw * 0.46f * (1.0f - fd);
    F.sd[1] = sw * 0.54f * (1.0f - fd);
    F.si[0] = sw * 0.46f * fd;
    F.si[1] = sw * 0.54f * fd;
}

__device__ __forceinline__ void store_forc(const Forc<float>& F, float* __restrict__ f, int ld) {
    auto s = [&](int plane, float v) { f[(size_t)plane * ld] = v; };
    s(IBIS_FORC_TA, F.ta); s(IBIS_FORC_QA, F.qa); s(IBIS_FORC_UA, F.ua); s(IBIS_FORC_PSURF, F.ps);
    s(IBIS_FORC_COSZEN, F.cosz);
    s(IBIS_FORC_SOLAD, F.sd[0]); s(IBIS_FORC_SOLAD + 1, F.sd[1]);
    s(IBIS_FORC_SOLAI, F.si[0]); s(IBIS_FORC_SOLAI + 1, F.si[1]);
    s(IBIS_FORC_FIRA, F.fira); s(IBIS_FORC_RAINA, F.rain); s(IBIS_FORC_SNOWA, F.snow);
}

__device__ __forceinline__ DailyRec load_daily(const float* __restrict__ p, int ld) {
    auto g = [&](int plane) { return __ldg(p + (size_t)plane * ld); };
    DailyRec d;
    d.tmax = g(IBIS_DAILY_TMAX); d.tmin = g(IBIS_DAILY_TMIN); d.cloud = g(IBIS_DAILY_CLOUD);
    d.precip = g(IBIS_DAILY_PRECIP); d.psurf = g(IBIS_DAILY_PSURF); d.qd = g(IBIS_DAILY_QD); d.ud = g(IBIS_DAILY_UD);
    d.fira = g(IBIS_DAILY_FIRA);
    return d;
}

}  // namespace ibis
