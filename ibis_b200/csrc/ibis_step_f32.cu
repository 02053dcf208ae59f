// FP32 production kernels of the hourly step (FP64 islands in the canopy and
// soil-water solves) and their C-ABI entry points.  The kernel instantiations
// live in ibis_f32_inst_*.cu so they compile in parallel.
#include <atomic>

#include "../../include/ibis_b200.h"
#include "ibis_kernels.cuh"

namespace ibis {
#define IBIS_EXTERN(NT, SU, SL, CFG) \
    extern template cudaError_t run_config<float, NT, SU, SL, CFG>(IBIS_RUN_ARGS(float));
IBIS_F77_CONFIGS(IBIS_EXTERN, 6)
IBIS_F77_CONFIGS(IBIS_EXTERN, 9)
IBIS_SUN_CONFIGS(IBIS_EXTERN, 6)
IBIS_SUN_CONFIGS(IBIS_EXTERN, 9)
#undef IBIS_EXTERN
#define IBIS_EXTERN_X3(NT, SU, SL, CFG) \
    extern template cudaError_t run_config<float, NT, SU, SL, CFG, true>(IBIS_RUN_ARGS(float));
IBIS_X3_CONFIGS(IBIS_EXTERN_X3, 6)
IBIS_X3_CONFIGS(IBIS_EXTERN_X3, 9)
#undef IBIS_EXTERN_X3
}  // namespace ibis

extern "C" int ibis_step_f32(float* prog, const float* stat, const float* forc, float* diag, float* acc, int ncell,
                             int ld, int nstep, const IbisParams* params, int* status, void* stream) {
    // launches of several hours take the fastest fused configuration at full
    // size (block 224, accumulators on chip); shorter ones the default
    const int cfg = nstep >= ibis::kAccSmemMinSteps ? ibis::kLongFused : ibis::kDefaultFused;
    return ibis::hourly_step<float>(prog, stat, forc, diag, acc, ncell, ld, nstep, params, status, stream, nullptr,
                                    cfg);
}

extern "C" int ibis_step_split_f32(float* prog, const float* stat, const float* forc, float* diag, float* acc,
                                   float* scratch, int ncell, int ld, int nstep, const IbisParams* params,
                                   int* status, void* stream) {
    if (!scratch) return -EINVAL;
    return ibis::hourly_step<float>(prog, stat, forc, diag, acc, ncell, ld, nstep, params, status, stream, scratch,
                                    ibis::kDefaultSplit);
}

extern "C" int ibis_step_config_f32(float* prog, const float* stat, const float* forc, float* diag, float* acc,
                                    float* scratch, int ncell, int ld, int nstep, const IbisParams* params,
                                    int* status, void* stream, int config) {
    return ibis::hourly_step<float>(prog, stat, forc, diag, acc, ncell, ld, nstep, params, status, stream, scratch,
                                    config);
}

extern "C" int ibis_mid_planes(void) { return ibis::kMidCount; }

extern "C" int ibis_num_configs(void) { return ibis::kNumConfigs; }

extern "C" int ibis_config_info(int config, int* form, int* block, int* min_blocks, int* block2, int* min_blocks2) {
    if (config < 0 || config >= ibis::kNumConfigs) return -EINVAL;
    const ibis::LaunchConfig& c = ibis::kConfigs[config];
    if (form) *form = c.form;
    if (block) *block = c.block;
    if (min_blocks) *min_blocks = c.minb;
    if (block2) *block2 = c.block2;
    if (min_blocks2) *min_blocks2 = c.minb2;
    return 0;
}

// ---------------------------------------------------------------------------
// Two-kernel step without any allocation by the caller or the library.
//
// Some callers cannot call cudaMalloc at the point where they run the step: an
// XLA custom-call handler must not allocate behind XLA's allocator, and serving
// loops that reserve all device memory up front have nothing left to hand out.
// For them the hand-off planes of the two-kernel form live in a fixed device
// array owned by this library, sized for kNoAllocMaxLd cells.
// ---------------------------------------------------------------------------
namespace {
constexpr int kNoAllocMaxLd = 32768;   // largest leading dimension (cells, padded to 32) accepted
constexpr int kMaxDevices = 64;
// kMidCount planes x kNoAllocMaxLd floats = 3.5 MiB, resident on every GPU that loads the library.
static __device__ __align__(256) float g_noalloc_mid[ibis::kMidCount * kNoAllocMaxLd];
// The array's device address per device, looked up on the first call there.
// Host threads may race on a slot; every writer stores the same address, and
// the atomics make the race well defined.  Not refreshed after cudaDeviceReset.
std::atomic<float*> g_noalloc_ptr[kMaxDevices];
}  // namespace

extern "C" int ibis_step_split_noalloc_f32(float* prog, const float* stat, const float* forc, float* diag,
                                           float* acc, int ncell, int ld, int nstep, const IbisParams* params,
                                           int* status, void* stream) {
    if (ld > kNoAllocMaxLd) {
        fprintf(stderr, "ibis_step_split_noalloc_f32: ld=%d exceeds the built-in scratch (%d cells)\n", ld,
                kNoAllocMaxLd);
        return -EINVAL;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return -ENODEV;
    float* mid = g_noalloc_ptr[dev].load(std::memory_order_relaxed);
    if (!mid) {
        // once per device, with that device current: the device address of the array
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_mid);
        if (e != cudaSuccess || !p) {
            fprintf(stderr, "ibis_step_split_noalloc_f32: cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
            return -(int)e - 1000;
        }
        mid = static_cast<float*>(p);
        g_noalloc_ptr[dev].store(mid, std::memory_order_relaxed);
    }
    return ibis::hourly_step<float>(prog, stat, forc, diag, acc, ncell, ld, nstep, params, status, stream, mid,
                                    ibis::kDefaultSplit);
}
