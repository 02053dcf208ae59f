// Explicit instantiations of the FP32 step kernels (part e: the staged fused
// configuration with bedrock); see ibis_step_f32.cu.
#include "../../include/ibis_b200.h"
#include "ibis_kernels.cuh"

namespace ibis {
#define IBIS_INST(NT, SU, SL, CFG) template cudaError_t run_config<float, NT, SU, SL, CFG>(IBIS_RUN_ARGS(float));
IBIS_INST(9, false, false, 11)
#undef IBIS_INST
}  // namespace ibis
