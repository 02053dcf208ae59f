// C-ABI entry points of the calibration-ensemble kernels (ibis_ensemble.cuh).
// The kernel instantiations live in ibis_ens_inst_*.cu so they compile in
// parallel.
#include <stdint.h>

#include "../../include/ibis_b200.h"
#include "ibis_ensemble.cuh"

namespace ibis {
#define IBIS_ENS_EXTERN(NT, SU, SL)                                                                          \
    extern template cudaError_t launch_ensemble<NT, SU, SL>(const EnsArgs&, const DevParams<float>&, int, int, \
                                                            cudaStream_t);                                     \
    extern template int ensemble_occupancy<NT, SU, SL>(int);                                                  \
    extern template cudaError_t launch_ensemble_hours<NT, SU, SL>(const EnsArgs&, const DevParams<float>&, int*, \
                                                                  int, cudaStream_t);
IBIS_ENS_VARIANTS(IBIS_ENS_EXTERN, 9)
IBIS_ENS_VARIANTS(IBIS_ENS_EXTERN, 6)
#undef IBIS_ENS_EXTERN
#define IBIS_ENS_DAILY_EXTERN(NT, SU, SL)                                                                    \
    extern template cudaError_t launch_ensemble<NT, SU, SL, true>(const EnsArgs&, const DevParams<float>&, int, \
                                                                  int, cudaStream_t);                          \
    extern template int ensemble_occupancy<NT, SU, SL, true>(int);
IBIS_ENS_VARIANTS(IBIS_ENS_DAILY_EXTERN, 9)
IBIS_ENS_VARIANTS(IBIS_ENS_DAILY_EXTERN, 6)
#undef IBIS_ENS_DAILY_EXTERN
#define IBIS_ENS_X3_EXTERN(NT, SU, SL)                                                                       \
    extern template cudaError_t launch_ensemble<NT, SU, SL, false, true>(const EnsArgs&, const DevParams<float>&, \
                                                                         int, int, cudaStream_t);               \
    extern template int ensemble_occupancy<NT, SU, SL, false, true>(int);                                       \
    extern template cudaError_t launch_ensemble<NT, SU, SL, true, true>(const EnsArgs&, const DevParams<float>&,  \
                                                                        int, int, cudaStream_t);                \
    extern template int ensemble_occupancy<NT, SU, SL, true, true>(int);                                        \
    extern template cudaError_t launch_ensemble_hours<NT, SU, SL, true>(const EnsArgs&, const DevParams<float>&,  \
                                                                        int*, int, cudaStream_t);
IBIS_ENS_VARIANTS(IBIS_ENS_X3_EXTERN, 9)
IBIS_ENS_VARIANTS(IBIS_ENS_X3_EXTERN, 6)
#undef IBIS_ENS_X3_EXTERN

namespace {

constexpr unsigned kEnsFlags = IBIS_FLAG_BEDROCK | IBIS_FLAG_H2O_CONSISTENT | IBIS_FLAG_SUNSHADE_U |
                               IBIS_FLAG_SUNSHADE_L | IBIS_FLAG_ACC | IBIS_FLAG_CH4 | IBIS_FLAG_SOIL_MEANS |
                               IBIS_FLAG_KAHAN | IBIS_FLAG_ZWT_OBS | IBIS_FLAG_ETPARTS | IBIS_FLAG_NEEPARTS |
                               IBIS_FLAGS_X3;

// Validate an ensemble description; fills `a`.  Returns 0, or -EINVAL.
int ens_args(const IbisEnsemble* e, const IbisParams* hp, EnsArgs& a) {
    if (!e || !hp) return -EINVAL;
    if (e->nrun < 0 || e->nsite < 0 || e->forc_len < 0 || (e->order && (e->norder < 0 || e->norder > e->nrun)))
        return -EINVAL;
    if (e->nrun == 0) return 0;
    if (!e->prog || !e->stat || !e->forc || !e->run_params || !e->run_site || !e->run_forc || !e->run_nstep)
        return -EINVAL;
    if (e->nsite < 1 || e->ld_run < e->nrun || e->ld_run % 32 || e->ld_site < e->nsite || e->ld_site % 32)
        return -EINVAL;
    if ((uintptr_t)e->forc % 16) return -EINVAL;
    if (hp->flags & ~kEnsFlags) return -EINVAL;
    const bool accum = hp->flags & (IBIS_FLAG_ACC | IBIS_FLAG_CH4 | IBIS_FLAG_SOIL_MEANS);
    if (accum && !e->acc) return -EINVAL;
    if (e->yearly && (!e->acc || !(hp->flags & IBIS_FLAG_ACC) || e->year_steps <= 0 || e->nyear < 0))
        return -EINVAL;
    if (!(hp->dtime > 0.0)) return -EINVAL;
    a.prog = e->prog;
    a.acc = accum ? e->acc : nullptr;
    a.stat = e->stat;
    a.forc = e->forc;
    a.run_params = e->run_params;
    a.run_site = e->run_site;
    a.run_forc = e->run_forc;
    a.run_nstep = e->run_nstep;
    a.run_pos = e->run_pos;
    a.order = e->order;
    a.yearly = e->yearly;
    a.forc_len = e->forc_len;
    a.nrun = e->nrun;
    a.ld_run = e->ld_run;
    a.nsite = e->nsite;
    a.ld_site = e->ld_site;
    a.nyear = e->nyear;
    a.year_steps = e->year_steps > 0 ? e->year_steps : 1;
    a.nwork = e->order ? e->norder : e->nrun;
    a.queue = e->queue;
    a.status = e->status;
    return 0;
}

int launch_error(cudaError_t err, const char* what) {
    if (err == cudaSuccess) return 0;
    fprintf(stderr, "ibis_b200: %s failed: %s\n", what, cudaGetErrorString(err));
    return -(int)err - 1000;
}

// Expands CALL(NT, SU, SL, X3) for the model variant the flags select: any
// IBIS_FLAGS_X3 flag selects the kernels with the IBIS 3.0 extensions.
#define IBIS_BY_CANOPY(flags, CALL, X3)                                                              \
    (((flags) & IBIS_FLAG_BEDROCK)                                                                  \
         ? (((flags) & IBIS_FLAG_SUNSHADE_U)                                                        \
                ? (((flags) & IBIS_FLAG_SUNSHADE_L) ? CALL(9, true, true, X3) : CALL(9, true, false, X3))  \
                : (((flags) & IBIS_FLAG_SUNSHADE_L) ? CALL(9, false, true, X3) : CALL(9, false, false, X3))) \
         : (((flags) & IBIS_FLAG_SUNSHADE_U)                                                        \
                ? (((flags) & IBIS_FLAG_SUNSHADE_L) ? CALL(6, true, true, X3) : CALL(6, true, false, X3))  \
                : (((flags) & IBIS_FLAG_SUNSHADE_L) ? CALL(6, false, true, X3) : CALL(6, false, false, X3))))
#define IBIS_BY_VARIANT(flags, CALL) \
    (((flags) & IBIS_FLAGS_X3) ? IBIS_BY_CANOPY(flags, CALL, true) : IBIS_BY_CANOPY(flags, CALL, false))

}  // namespace
}  // namespace ibis

using namespace ibis;

extern "C" int ibis_ensemble_occupancy(const IbisParams* params, int block) {
    if (!params || block < 32 || block > 256 || block % 32) return 0;
#define IBIS_OCC(NT, SU, SL, X3) ensemble_occupancy<NT, SU, SL, false, X3>(block)
    return IBIS_BY_VARIANT(params->flags, IBIS_OCC);
#undef IBIS_OCC
}

namespace {

// The persistent launch of ibis_ensemble_f32 / ibis_ensemble_daily_f32 on a
// validated description.
template <bool DAILY>
int ensemble_launch(const IbisEnsemble* ens, EnsArgs& a, const IbisParams* params, int block, void* stream) {
    if (!ens->queue) return -EINVAL;
    if (block != 0 && (block < 32 || block > 256 || block % 32)) return -EINVAL;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0)
        return -ENODEV;
    if (a.nwork == 0) return 0;
    const int nitem = (a.nwork + 31) / 32;
    if (block == 0) {
        const int w = (nitem + sms - 1) / sms;          // warps per SM that cover every item in one pass
        block = 32 * (w < 1 ? 1 : (w > 8 ? 8 : w));
    }
#define IBIS_OCC(NT, SU, SL, X3) ensemble_occupancy<NT, SU, SL, DAILY, X3>(block)
    const int occ = IBIS_BY_VARIANT(params->flags, IBIS_OCC);
#undef IBIS_OCC
    if (occ <= 0) return -EINVAL;
    const int per_block = block / 32;
    int grid = sms * occ;
    const int need = (nitem + per_block - 1) / per_block;
    if (need < grid) grid = need;
    const DevParams<float> P = make_dev_params<float>(*params);
    cudaStream_t s = (cudaStream_t)stream;
    const int rc = launch_error(cudaMemsetAsync(ens->queue, 0, sizeof(int), s), "ensemble queue reset");
    if (rc) return rc;
#define IBIS_RUN(NT, SU, SL, X3) launch_ensemble<NT, SU, SL, DAILY, X3>(a, P, block, grid, s)
    const cudaError_t err = IBIS_BY_VARIANT(params->flags, IBIS_RUN);
#undef IBIS_RUN
    return launch_error(err, "ensemble launch");
}

}  // namespace

extern "C" int ibis_ensemble_f32(const IbisEnsemble* ens, const IbisParams* params, int block, void* stream) {
    EnsArgs a{};
    int rc = ens_args(ens, params, a);
    if (rc || ens->nrun == 0) return rc;
    return ensemble_launch<false>(ens, a, params, block, stream);
}

extern "C" int ibis_ensemble_daily_f32(const IbisEnsemble* ens, const IbisEnsembleDaily* daily,
                                       const IbisParams* params, int block, void* stream) {
    if (!ens || !daily || !params) return -EINVAL;
    if (!daily->records || !daily->site_lat || daily->len < 0 || ((uintptr_t)daily->records % 16) ||
        (daily->flags & ~IBIS_DIURNAL_OBSERVED_FIRA))
        return -EINVAL;
    if (!(params->dtime > 0.0)) return -EINVAL;
    const int nh = (int)(86400.0 / params->dtime);
    if (nh < 1 || nh > 254 || (double)nh * params->dtime != 86400.0) return -EINVAL;
    IbisEnsemble hourly = *ens;          // the hourly-record checks do not apply: no hourly records
    alignas(16) static const float kNoRecords[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    hourly.forc = kNoRecords;
    hourly.forc_len = 0;
    EnsArgs a{};
    int rc = ens_args(&hourly, params, a);
    if (rc || ens->nrun == 0) return rc;
    a.forc = nullptr;
    a.daily = daily->records;
    a.site_lat = daily->site_lat;
    a.daily_len = daily->len;
    a.seed = daily->seed;
    a.obs_fira = (daily->flags & IBIS_DIURNAL_OBSERVED_FIRA) != 0;
    a.nh = nh;
    a.dtime = (float)params->dtime;
    return ensemble_launch<true>(ens, a, params, block, stream);
}

extern "C" int ibis_ensemble_hours_f32(const IbisEnsemble* ens, const IbisParams* params, int* hour, int nhour,
                                       void* stream) {
    EnsArgs a{};
    int rc = ens_args(ens, params, a);
    if (rc || ens->nrun == 0) return rc;
    if (!hour || nhour < 0) return -EINVAL;
    if (nhour == 0) return 0;
    const DevParams<float> P = make_dev_params<float>(*params);
    cudaStream_t s = (cudaStream_t)stream;
#define IBIS_RUN(NT, SU, SL, X3) launch_ensemble_hours<NT, SU, SL, X3>(a, P, hour, nhour, s)
    const cudaError_t err = IBIS_BY_VARIANT(params->flags, IBIS_RUN);
#undef IBIS_RUN
    return launch_error(err, "ensemble hourly launch");
}
