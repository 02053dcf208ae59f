// Monthly wetland methane: month_begin / month_end kernels, float and double planes.
#include <errno.h>
#include <stdio.h>

#include "../../include/ibis_b200.h"
#include "ibis_kernels.cuh"
#include "ibis_month.cuh"

namespace {

int launched(const char* what) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        fprintf(stderr, "%s: launch failed: %s\n", what, cudaGetErrorString(e));
        return -(int)e - 1000;
    }
    return 0;
}

template <typename R>
int month_begin(R* acc, R* wet, const R* dayst, int ncell, int ld, unsigned flags, void* stream, const char* what) {
    if (!acc || !wet) return -EINVAL;
    if (ncell < 0 || ld < ncell || ld % 32 || (flags & ~IBIS_MONTH_NEW_YEAR)) return -EINVAL;
    if (ncell == 0) return 0;
    const int block = 128, grid = (ncell + block - 1) / block;
    ibis::month_begin_kernel<R><<<grid, block, 0, (cudaStream_t)stream>>>(acc, wet, dayst, ncell, ld,
                                                                          (flags & IBIS_MONTH_NEW_YEAR) != 0);
    return launched(what);
}

template <typename R>
int month_end(const R* prog, const R* stat, const R* acc, R* wet, R* dayst, const R* scale, int ncell, int ld,
              int ndays, const IbisParams* hp, unsigned flags, void* stream, const char* what) {
    if (!prog || !stat || !wet || !hp) return -EINVAL;
    if (ncell < 0 || ld < ncell || ld % 32 || ndays < 1) return -EINVAL;
    if (flags & ~(IBIS_MONTH_FROM_MEAN | IBIS_MONTH_PARTITION)) return -EINVAL;
    if ((flags & IBIS_MONTH_FROM_MEAN) && !acc) return -EINVAL;
    if ((flags & IBIS_MONTH_PARTITION) && !dayst) return -EINVAL;
    if (hp->flags & ~(unsigned)IBIS_FLAG_ZWT_OBS & ~(IBIS_FLAG_BEDROCK | IBIS_FLAG_H2O_CONSISTENT |
                                                   IBIS_FLAG_SUNSHADE_U | IBIS_FLAG_SUNSHADE_L | IBIS_FLAG_ACC |
                                                   IBIS_FLAG_CH4 | IBIS_FLAG_SOIL_MEANS | IBIS_FLAG_DIAG |
                                                   IBIS_FLAG_KAHAN | IBIS_FLAG_ETPARTS | IBIS_FLAG_NEEPARTS |
                                                   IBIS_FLAGS_X3 | IBIS_FLAG_CH4_BANDS))
        return -EINVAL;
    if (!(hp->dtime > 0.0)) return -EINVAL;
    if (ncell == 0) return 0;
    const ibis::DevParams<R> P = ibis::make_dev_params<R>(*hp);
    const int block = 128, grid = (ncell + block - 1) / block;
    ibis::month_end_kernel<R><<<grid, block, 0, (cudaStream_t)stream>>>(
        prog, stat, acc, wet, dayst, scale, ncell, ld, ndays, P, (flags & IBIS_MONTH_FROM_MEAN) != 0,
        (flags & IBIS_MONTH_PARTITION) != 0);
    return launched(what);
}

}  // namespace

extern "C" int ibis_month_begin_f32(float* acc, float* wet, const float* dayst, int ncell, int ld, unsigned int flags,
                                    void* stream) {
    return month_begin(acc, wet, dayst, ncell, ld, flags, stream, "ibis_month_begin_f32");
}

extern "C" int ibis_month_begin_f64(double* acc, double* wet, const double* dayst, int ncell, int ld,
                                    unsigned int flags, void* stream) {
    return month_begin(acc, wet, dayst, ncell, ld, flags, stream, "ibis_month_begin_f64");
}

extern "C" int ibis_month_end_f32(const float* prog, const float* stat, const float* acc, float* wet, float* dayst,
                                  const float* scale, int ncell, int ld, int ndays, const IbisParams* params,
                                  unsigned int flags, void* stream) {
    return month_end(prog, stat, acc, wet, dayst, scale, ncell, ld, ndays, params, flags, stream,
                     "ibis_month_end_f32");
}

extern "C" int ibis_month_end_f64(const double* prog, const double* stat, const double* acc, double* wet,
                                  double* dayst, const double* scale, int ncell, int ld, int ndays,
                                  const IbisParams* params, unsigned int flags, void* stream) {
    return month_end(prog, stat, acc, wet, dayst, scale, ncell, ld, ndays, params, flags, stream,
                     "ibis_month_end_f64");
}
