// Explicit instantiations of the FP32 step kernels (part b); see ibis_step_f32.cu.
#include "../../include/ibis_b200.h"
#include "ibis_kernels.cuh"

namespace ibis {
#define IBIS_INST(NT, SU, SL, CFG) template cudaError_t run_config<float, NT, SU, SL, CFG>(IBIS_RUN_ARGS(float));
IBIS_INST(9, false, false, 5) IBIS_INST(9, false, false, 6) IBIS_INST(9, false, false, 7)
IBIS_INST(9, false, false, 8) IBIS_INST(9, false, false, 9) IBIS_INST(9, false, false, 10)
#undef IBIS_INST
}  // namespace ibis
