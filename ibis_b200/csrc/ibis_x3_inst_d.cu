// Explicit instantiations of the FP32 step kernels with the IBIS 3.0 extensions (part d);
// see ibis_step_f32.cu.
#include "../../include/ibis_b200.h"
#include "ibis_kernels.cuh"

namespace ibis {
#define IBIS_INST(NT, SU, SL, CFG) \
    template cudaError_t run_config<float, NT, SU, SL, CFG, true>(IBIS_RUN_ARGS(float));
IBIS_INST(6, false, false, 8)
IBIS_INST(6, true, true, 0)
IBIS_INST(6, true, true, 6)
IBIS_INST(6, true, true, 8)
#undef IBIS_INST
}  // namespace ibis
