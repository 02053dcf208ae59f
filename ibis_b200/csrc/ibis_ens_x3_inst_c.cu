// Explicit instantiations of the ensemble kernels with the IBIS 3.0 extensions
// (one launch per hour, 9 temperature nodes per column); see ibis_ensemble_f32.cu.
#include "../../include/ibis_b200.h"
#include "ibis_ensemble.cuh"

namespace ibis {
#define IBIS_INST(NT, SU, SL) \
    template cudaError_t launch_ensemble_hours<NT, SU, SL, true>(const EnsArgs&, const DevParams<float>&, int*, int, \
                                                                 cudaStream_t);
IBIS_ENS_VARIANTS(IBIS_INST, 9)
#undef IBIS_INST
}  // namespace ibis
