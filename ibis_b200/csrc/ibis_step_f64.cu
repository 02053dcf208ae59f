// Float64 kernels of the hourly step: every operation in double, compiled
// without fused multiply-add contraction so the rounding sequence follows the
// reference's float64 run as closely as the device allows.
#include "../../include/ibis_b200.h"
#include "ibis_kernels.cuh"

extern "C" int ibis_step_f64(double* prog, const double* stat, const double* forc, double* diag, double* acc,
                             int ncell, int ld, int nstep, const IbisParams* params, int* status, void* stream) {
    return ibis::hourly_step<double>(prog, stat, forc, diag, acc, ncell, ld, nstep, params, status, stream, nullptr,
                                     ibis::kDefaultFused);
}
