// Explicit instantiations of the FP32 step kernels (part d); see ibis_step_f32.cu.
#include "../../include/ibis_b200.h"
#include "ibis_kernels.cuh"

namespace ibis {
#define IBIS_INST(NT, SU, SL, CFG) template cudaError_t run_config<float, NT, SU, SL, CFG>(IBIS_RUN_ARGS(float));
IBIS_SUN_CONFIGS(IBIS_INST, 6)
IBIS_SUN_CONFIGS(IBIS_INST, 9)
#undef IBIS_INST
}  // namespace ibis
