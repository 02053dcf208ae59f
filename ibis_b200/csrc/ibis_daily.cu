// Daily cadence of the day loop: day_begin / day_end kernels, float and double planes.
#include <errno.h>
#include <stdio.h>

#include "../../include/ibis_b200.h"
#include "ibis_daily.cuh"

namespace {

bool valid(const void* a, const void* b, const void* c, const void* d, int ncell, int ld, const IbisParams* P,
           const IbisDayParams* dp) {
    if (!a || !b || !c || !d || !P || !dp) return false;
    if (ncell < 0 || ld < ncell || ld % 32) return false;
    if (!(P->ndaypy > 0.0) || !(dp->ddays > 0.0) || !(dp->gdd_ramp_u > 0.0) || !(dp->gdd_ramp_l > 0.0)) return false;
    // the module switches are 0 or 1; the seasonal states need a time constant and a day of year
    for (const double sw : {dp->seasonal_on, dp->stress_on, dp->sen_photoperiod_u, dp->sen_photoperiod_l})
        if (sw != 0.0 && sw != 1.0) return false;
    if (dp->seasonal_on != 0.0 && (!(dp->acclim_tau > 0.0) || !(dp->jday >= 1.0 && dp->jday <= 366.0))) return false;
    double h4 = 0.0;
    for (int k = 0; k < 4; ++k) {
        if (!(P->hsoi[k] > 0.0)) return false;
        h4 += P->hsoi[k];
    }
    return h4 > 0.0;
}

ibis::DayConst day_const(const IbisParams* P) {
    ibis::DayConst c;
    for (int k = 0; k < 6; ++k) c.hsoi[k] = P->hsoi[k];
    c.ndaypy = P->ndaypy;
    c.epsilon = P->epsilon;
    return c;
}

int launched(const char* what) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        fprintf(stderr, "%s: launch failed: %s\n", what, cudaGetErrorString(e));
        return -(int)e - 1000;
    }
    return 0;
}

template <typename R>
int day_begin(R* stat, R* dayst, R* acc, const R* td, int ncell, int ld, const IbisParams* P,
              const IbisDayParams* dp, void* stream, const char* what) {
    if (!valid(stat, dayst, acc, td, ncell, ld, P, dp)) return -EINVAL;
    if (ncell == 0) return 0;
    const int block = 128, grid = (ncell + block - 1) / block;
    ibis::day_begin_kernel<R><<<grid, block, 0, (cudaStream_t)stream>>>(stat, dayst, acc, td, ncell, ld, *dp,
                                                                        day_const(P));
    return launched(what);
}

template <typename R>
int day_end(const R* prog, R* stat, R* dayst, const R* acc, const R* td, int ncell, int ld, const IbisParams* P,
            const IbisDayParams* dp, void* stream, const char* what) {
    if (!prog || !valid(stat, dayst, acc, td, ncell, ld, P, dp)) return -EINVAL;
    if (ncell == 0) return 0;
    const int block = 128, grid = (ncell + block - 1) / block;
    ibis::day_end_kernel<R><<<grid, block, 0, (cudaStream_t)stream>>>(prog, stat, dayst, acc, td, ncell, ld, *dp,
                                                                      day_const(P));
    return launched(what);
}

}  // namespace

extern "C" int ibis_day_begin_f32(float* stat, float* dayst, float* acc, const float* td, int ncell, int ld,
                                  const IbisParams* params, const IbisDayParams* dayparams, void* stream) {
    return day_begin(stat, dayst, acc, td, ncell, ld, params, dayparams, stream, "ibis_day_begin_f32");
}

extern "C" int ibis_day_begin_f64(double* stat, double* dayst, double* acc, const double* td, int ncell, int ld,
                                  const IbisParams* params, const IbisDayParams* dayparams, void* stream) {
    return day_begin(stat, dayst, acc, td, ncell, ld, params, dayparams, stream, "ibis_day_begin_f64");
}

extern "C" int ibis_day_end_f32(const float* prog, float* stat, float* dayst, const float* acc, const float* td,
                                int ncell, int ld, const IbisParams* params, const IbisDayParams* dayparams,
                                void* stream) {
    return day_end(prog, stat, dayst, acc, td, ncell, ld, params, dayparams, stream, "ibis_day_end_f32");
}

extern "C" int ibis_day_end_f64(const double* prog, double* stat, double* dayst, const double* acc,
                                const double* td, int ncell, int ld, const IbisParams* params,
                                const IbisDayParams* dayparams, void* stream) {
    return day_end(prog, stat, dayst, acc, td, ncell, ld, params, dayparams, stream, "ibis_day_end_f64");
}
