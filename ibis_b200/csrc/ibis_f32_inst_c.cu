// Explicit instantiations of the FP32 step kernels (part c); see ibis_step_f32.cu.
#include "../../include/ibis_b200.h"
#include "ibis_kernels.cuh"

namespace ibis {
#define IBIS_INST(NT, SU, SL, CFG) template cudaError_t run_config<float, NT, SU, SL, CFG>(IBIS_RUN_ARGS(float));
IBIS_F77_CONFIGS(IBIS_INST, 6)
#undef IBIS_INST
}  // namespace ibis
