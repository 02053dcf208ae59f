// Explicit instantiations of the FP32 step kernels (part a); see ibis_step_f32.cu.
#include "../../include/ibis_b200.h"
#include "ibis_kernels.cuh"

namespace ibis {
#define IBIS_INST(NT, SU, SL, CFG) template cudaError_t run_config<float, NT, SU, SL, CFG>(IBIS_RUN_ARGS(float));
IBIS_INST(9, false, false, 0) IBIS_INST(9, false, false, 1) IBIS_INST(9, false, false, 2)
IBIS_INST(9, false, false, 3) IBIS_INST(9, false, false, 4)
#undef IBIS_INST
}  // namespace ibis
