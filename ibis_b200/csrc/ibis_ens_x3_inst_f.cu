// Explicit instantiations of the ensemble kernels with the IBIS 3.0 extensions
// (persistent form over day records, 6 temperature nodes per column); see ibis_ensemble_f32.cu.
#include "../../include/ibis_b200.h"
#include "ibis_ensemble.cuh"

namespace ibis {
#define IBIS_INST(NT, SU, SL) \
    template cudaError_t launch_ensemble<NT, SU, SL, true, true>(const EnsArgs&, const DevParams<float>&, int, int, \
                                                              cudaStream_t);                                    \
    template int ensemble_occupancy<NT, SU, SL, true, true>(int);
IBIS_ENS_VARIANTS(IBIS_INST, 6)
#undef IBIS_INST
}  // namespace ibis
