// FP32 production kernels of the hourly step (FP64 islands in the canopy and
// soil-water solves) and their C-ABI entry point.
#include "../../include/ibis_b200.h"
#include "ibis_kernels.cuh"

extern "C" int ibis_step_f32(float* prog, const float* stat, const float* forc, float* diag, float* acc, int ncell,
                             int ld, int nstep, const IbisParams* params, int* status, void* stream) {
    return ibis::hourly_step<float>(prog, stat, forc, diag, acc, ncell, ld, nstep, params, status, stream);
}

extern "C" int ibis_step_split_f32(float* prog, const float* stat, const float* forc, float* diag, float* acc,
                                   float* scratch, int ncell, int ld, int nstep, const IbisParams* params,
                                   int* status, void* stream) {
    if (!scratch) return -EINVAL;
    return ibis::hourly_step<float>(prog, stat, forc, diag, acc, ncell, ld, nstep, params, status, stream, scratch);
}

extern "C" int ibis_mid_planes(void) { return ibis::kMidCount; }
