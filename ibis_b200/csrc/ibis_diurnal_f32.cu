// Device forcing generator: daily weather planes -> hourly forcing planes.
#include <errno.h>
#include <stdio.h>

#include "../../include/ibis_b200.h"
#include "ibis_diurnal.cuh"

namespace ibis {

// One thread per cell walks its days and hours; the writes of a warp to one
// forcing plane are 32 consecutive floats.
__global__ void __launch_bounds__(128) diurnal_kernel(const float* __restrict__ daily, const float* __restrict__ lat,
                                                      const float* __restrict__ sw_obs,
                                                      const unsigned char* __restrict__ use,
                                                      float* __restrict__ forc, int ncell, int ld, int nday, int nh,
                                                      int jday0, int day0, float dtime, uint32_t seed, bool obs,
                                                      int cell0) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ncell) return;
    const uint32_t key = (uint32_t)(i + cell0);   // the cell in the caller's numbering keys its variates
    const double xlat = (double)__ldg(lat + i) * (3.14159265358979323846 / 180.0);
    const float sinlat = (float)sin(xlat), coslat = (float)cos(xlat);
#pragma unroll 1
    for (int d = 0; d < nday; ++d) {
        const int jday = (jday0 - 1 + d) % 365 + 1;
        const DayGeom g = day_geometry(jday);
        const DailyRec rec = load_daily(daily + (size_t)d * IBIS_DAILY_COUNT * ld + i, ld);
        const uint32_t day = (uint32_t)(day0 + d);
        const Event ev = precip_timing(draw24(seed, key, day, 0), draw24(seed, key, day, 1), rec.precip, dtime);
        const bool use_sw = sw_obs && use[(size_t)d * ld + i];
#pragma unroll 1
        for (int h = 0; h < nh; ++h) {
            Forc<float> F = diurnal_hour(rec, g, sinlat, coslat, (float)h * dtime, ev, draw24(seed, key, day, 2 + h),
                                         dtime, obs);
            if (use_sw) observed_shortwave(__ldg(sw_obs + (size_t)(d * nh + h) * ld + i), g.sw, F);
            store_forc(F, forc + (size_t)(d * nh + h) * IBIS_FORC_COUNT * ld + i, ld);
        }
    }
}

// The forcing generator on `ncell` cells whose first is cell `cell0` of the
// caller's numbering (the variates are keyed by that number).
int diurnal(const float* daily, const float* lat, const float* sw_obs, const unsigned char* use, float* forc,
            int ncell, int ld, int nday, int jday0, int day0, float dtime, unsigned int seed, unsigned int flags,
            void* stream, const char* what, int cell0) {
    if (!daily || !lat || !forc || (sw_obs && !use)) return -EINVAL;
    if (ncell < 0 || nday < 0 || ld < ncell || ld % 32 || day0 < 0 || jday0 < 1 || jday0 > 366) return -EINVAL;
    if (!(dtime > 0.0f)) return -EINVAL;
    const int nh = (int)(86400.0f / dtime);
    if (nh < 1 || nh > 254 || (float)nh * dtime != 86400.0f) return -EINVAL;
    if (flags & ~IBIS_DIURNAL_OBSERVED_FIRA) return -EINVAL;
    if (ncell == 0 || nday == 0) return 0;
    const int block = 128, grid = (ncell + block - 1) / block;
    ibis::diurnal_kernel<<<grid, block, 0, (cudaStream_t)stream>>>(daily, lat, sw_obs, use, forc, ncell, ld, nday, nh,
                                                                   jday0, day0, dtime, (uint32_t)seed,
                                                                   (flags & IBIS_DIURNAL_OBSERVED_FIRA) != 0, cell0);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        fprintf(stderr, "%s: launch failed: %s\n", what, cudaGetErrorString(e));
        return -(int)e - 1000;
    }
    return 0;
}

}  // namespace ibis

extern "C" int ibis_diurnal_f32(const float* daily, const float* lat, float* forc, int ncell, int ld, int nday,
                                int jday0, int day0, float dtime, unsigned int seed, unsigned int flags,
                                void* stream) {
    return ibis::diurnal(daily, lat, nullptr, nullptr, forc, ncell, ld, nday, jday0, day0, dtime, seed, flags, stream,
                         "ibis_diurnal_f32", 0);
}

extern "C" int ibis_diurnal_sw_f32(const float* daily, const float* lat, const float* sw_obs,
                                   const unsigned char* use, float* forc, int ncell, int ld, int nday, int jday0,
                                   int day0, float dtime, unsigned int seed, unsigned int flags, void* stream) {
    if (!sw_obs) return -EINVAL;
    return ibis::diurnal(daily, lat, sw_obs, use, forc, ncell, ld, nday, jday0, day0, dtime, seed, flags, stream,
                         "ibis_diurnal_sw_f32", 0);
}
