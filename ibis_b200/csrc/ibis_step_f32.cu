// FP32 production kernels of the hourly step (FP64 islands in the canopy and
// soil-water solves) and their C-ABI entry points.  The kernel instantiations
// live in ibis_f32_inst_*.cu so they compile in parallel.
#include <atomic>
#include <mutex>

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
// the forcing generator of ibis_diurnal_f32.cu on a range of cells
int diurnal(const float* daily, const float* lat, const float* sw_obs, const unsigned char* use, float* forc,
            int ncell, int ld, int nday, int jday0, int day0, float dtime, unsigned int seed, unsigned int flags,
            void* stream, const char* what, int cell0);
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

// ---------------------------------------------------------------------------
// The step from host buffers.  A batch of several waves is cut into groups of
// columns: each group's forcing is copied in on one copy stream, its hours run
// on one of a few compute streams, and its state is copied out on a second
// copy stream, so the copies of one group overlap the steps of the others and
// the groups' kernels fill the SMs together (no group waits for another
// group's slowest column).  A batch of about a wave or less has no later
// waves to hide copies behind: its hours are cut into chunks instead, the
// copy of each chunk overlapping the steps of the chunk before.
// ---------------------------------------------------------------------------
namespace {
constexpr int kHostStreams = 16;    // compute streams the groups take in turn
constexpr int kHostMaxGroups = 64;
constexpr int kHostMaxPieces = 256; // (group, chunk of hours) pairs of one call
// groups when the caller leaves the size to ibis_step_host_f32: at 95,333
// cells x 24 hours, each group's day in two chunks, a day from host to host
// takes 3.17 ms in 16 groups, 3.19 in 12, 3.20 in 24 and 3.26 in 20 (median of
// 4 interleaved rounds; the same day with its forcing already on the device:
// 2.99 ms)
constexpr int kHostAutoGroups = 16;
// the same for ibis_day_host_f32 (forcing generated per group from daily weather)
constexpr int kDayHostAutoGroups = 20;
// batches of more than this many waves of the launch configuration are cut
// into groups, smaller ones into chunks of hours.  A day from host to host,
// groups / chunks: 1 wave (33,152 cells) 2.30 / 1.71 ms; 1.25 waves 2.37 /
// 2.68 ms; 1.5 waves 2.54 / 2.77 ms; 2 waves 2.88 / 3.00 ms.
constexpr double kHostGroupWaves = 1.15;

struct HostPipe {
    bool ready = false;
    cudaStream_t h2d = nullptr, d2h = nullptr, comp[kHostStreams] = {};
    cudaEvent_t start = nullptr, out_done = nullptr;
    cudaEvent_t landed[kHostMaxPieces] = {}, stepped[kHostMaxGroups] = {};
};
std::mutex g_host_mu;
HostPipe g_host[kMaxDevices];

cudaError_t host_pipe_init(HostPipe& h) {
    if (h.ready) return cudaSuccess;
    cudaError_t e = cudaStreamCreateWithFlags(&h.h2d, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h.d2h, cudaStreamNonBlocking);
    for (int k = 0; k < kHostStreams && e == cudaSuccess; ++k)
        e = cudaStreamCreateWithFlags(&h.comp[k], cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h.start, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&h.out_done, cudaEventDisableTiming);
    for (int g = 0; g < kHostMaxPieces && e == cudaSuccess; ++g)
        e = cudaEventCreateWithFlags(&h.landed[g], cudaEventDisableTiming);
    for (int g = 0; g < kHostMaxGroups && e == cudaSuccess; ++g)
        e = cudaEventCreateWithFlags(&h.stepped[g], cudaEventDisableTiming);
    h.ready = e == cudaSuccess;
    return e;
}

int host_error(cudaError_t e, const char* what, const char* entry = "ibis_step_host_f32") {
    fprintf(stderr, "%s: %s failed: %s\n", entry, what, cudaGetErrorString(e));
    return -(int)e - 1000;
}

// Hours of each chunk: `chunk` hours each; -c: c hours, then the rest; with
// chunk 0 and several groups (`whole`), a third of the hours, then the rest
// (every group's first third is copied before any group's remainder, so the
// first wave starts after a third of its copy; measured at 49,728 - 95,333
// cells x 24 hours, [8, 16] beat one chunk by 5-11 % and [4, 20], [12, 12],
// [16, 8] and 2 x 12 or 4 x 6 equal chunks by up to 14 %); with chunk 0 and one
// group, 4 hours growing by 1.75 per chunk, the last taking a remainder under
// half its size (a copy of each chunk then stays within the steps of the chunk
// before, and few launches keep their tails few).
int chunk_schedule(int nstep, int chunk, bool whole, int* out, int cap) {
    int n = 0, h = 0;
    double c = 4.0;
    while (h < nstep) {
        int m;
        if (chunk > 0) m = chunk;
        else if (chunk < 0) m = n == 0 ? -chunk : nstep - h;   // -c: c hours, then the rest
        else if (whole) m = n == 0 ? (nstep + 2) / 3 : nstep - h;
        else {
            m = (int)c;
            const int rem = nstep - h;
            if (m > rem || rem - m < m / 2.0) m = rem;
            c *= 1.75;
        }
        if (m > nstep - h) m = nstep - h;
        if (n == cap) return -1;
        out[n++] = m;
        h += m;
    }
    return n;
}
}  // namespace

extern "C" int ibis_step_host_f32(float* prog, const float* stat, const float* host_forc, float* forc, float* diag,
                                  float* acc, float* host_prog, int ncell, int ld, int nstep,
                                  const IbisParams* params, int* status, int group, int chunk, int config,
                                  void* stream) {
    if (!prog || !stat || !host_forc || !forc || !params) return -EINVAL;
    if (ncell < 0 || nstep < 0 || ld < ncell || ld % 32 || group < 0 || group % 32 || chunk < -(1 << 20))
        return -EINVAL;
    if (config < -1 || config >= ibis::kNumConfigs || (config >= 0 && ibis::kConfigs[config].form == 1))
        return -EINVAL;
    if (ncell == 0) return 0;
    const int cfg = config >= 0 ? config : (nstep >= ibis::kAccSmemMinSteps ? ibis::kLongFused : ibis::kDefaultFused);
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return -ENODEV;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) return -ENODEV;
    if (group == 0) {
        // whole blocks per group: a partial block in every group would add
        // blocks to the batch, and a batch of whole waves would spill into one more
        const int block = ibis::kConfigs[cfg].block;
        const double wave = (double)sms * block * ibis::kConfigs[cfg].minb;
        group = ncell > kHostGroupWaves * wave
                    ? ((ncell + kHostAutoGroups - 1) / kHostAutoGroups + block - 1) / block * block
                    : (ncell + 31) / 32 * 32;
    }
    const int min_group = ((ncell + kHostMaxGroups - 1) / kHostMaxGroups + 31) / 32 * 32;
    if (group < min_group) group = min_group;
    const int ngroup = (ncell + group - 1) / group;
    int sched[kHostMaxPieces];
    const int nchunk = chunk_schedule(nstep, chunk, ngroup > 1, sched, kHostMaxPieces);
    if (nchunk < 0 || (long long)ngroup * nchunk > kHostMaxPieces) {
        fprintf(stderr, "ibis_step_host_f32: %d groups x %d chunks exceed %d pieces\n", ngroup, nchunk,
                kHostMaxPieces);
        return -EINVAL;
    }
    std::lock_guard<std::mutex> lock(g_host_mu);   // one caller at a time uses the device's streams and events
    HostPipe& h = g_host[dev];
    cudaError_t e = host_pipe_init(h);
    if (e != cudaSuccess) return host_error(e, "stream setup");
    cudaStream_t user = (cudaStream_t)stream;
    // everything queued on the caller's stream before this call comes first
    if ((e = cudaEventRecord(h.start, user)) != cudaSuccess) return host_error(e, "event record");
    e = cudaStreamWaitEvent(h.h2d, h.start, 0);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(h.d2h, h.start, 0);
    for (int k = 0; k < kHostStreams && k < ngroup && e == cudaSuccess; ++k)
        e = cudaStreamWaitEvent(h.comp[k], h.start, 0);
    if (e != cudaSuccess) return host_error(e, "stream wait");
    const size_t pitch = (size_t)ld * sizeof(float);
    const size_t fstride = (size_t)IBIS_FORC_COUNT * ld;
    int rc = 0, queued = 0;                         // groups whose work is on the library's streams
    const char* what = nullptr;
    // chunk-major: every group's first chunk is copied before any group's
    // second, so the first wave's blocks start while the rest still copies;
    // after a group's last chunk its stream position is recorded at once (a
    // later group may share the stream) and its state copied out
    for (int k = 0, h0 = 0; k < nchunk && !rc && !what; h0 += sched[k], ++k) {
        const int m = sched[k];
        for (int g = 0; g < ngroup && !rc && !what; ++g) {
            const int c0 = g * group, n = ncell - c0 < group ? ncell - c0 : group;
            cudaStream_t cs = h.comp[g % kHostStreams];
            cudaEvent_t landed = h.landed[g * nchunk + k];
            e = cudaMemcpy2DAsync(forc + h0 * fstride + c0, pitch, host_forc + h0 * fstride + c0, pitch,
                                  (size_t)n * sizeof(float), (size_t)m * IBIS_FORC_COUNT, cudaMemcpyHostToDevice,
                                  h.h2d);
            if (e == cudaSuccess) e = cudaEventRecord(landed, h.h2d);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(cs, landed, 0);
            if (e != cudaSuccess) { what = "forcing copy"; break; }
            rc = ibis::hourly_step<float>(prog + c0, stat + c0, forc + h0 * fstride + c0, diag ? diag + c0 : nullptr,
                                          acc ? acc + c0 : nullptr, n, ld, m, params, status, cs, nullptr, cfg, c0);
            if (k + 1 < nchunk && !rc) continue;
            // the group's stream position (on failure too, so the join below covers it)
            const cudaError_t r = cudaEventRecord(h.stepped[g], cs);
            if (r != cudaSuccess) { what = "event record"; e = r; break; }
            queued = g + 1;
            if (rc) break;
            if (!host_prog) continue;
            e = cudaStreamWaitEvent(h.d2h, h.stepped[g], 0);
            if (e == cudaSuccess)
                e = cudaMemcpy2DAsync(host_prog + c0, pitch, prog + c0, pitch, (size_t)n * sizeof(float),
                                      IBIS_PROG_COUNT, cudaMemcpyDeviceToHost, h.d2h);
            if (e != cudaSuccess) what = "state copy";
        }
    }
    if (nchunk == 0) {                              // no hours: the state as it stands
        for (int g = 0; g < ngroup && !what; ++g) {
            const int c0 = g * group, n = ncell - c0 < group ? ncell - c0 : group;
            if ((e = cudaEventRecord(h.stepped[g], h.comp[g % kHostStreams])) != cudaSuccess) {
                what = "event record";
                break;
            }
            queued = g + 1;
            if (!host_prog) continue;
            e = cudaStreamWaitEvent(h.d2h, h.stepped[g], 0);
            if (e == cudaSuccess)
                e = cudaMemcpy2DAsync(host_prog + c0, pitch, prog + c0, pitch, (size_t)n * sizeof(float),
                                      IBIS_PROG_COUNT, cudaMemcpyDeviceToHost, h.d2h);
            if (e != cudaSuccess) what = "state copy";
        }
    }
    // the caller's stream continues after every queued group's hours and copies,
    // on failure too, so that nothing of this call is still running when the
    // caller's stream reaches its next work
    cudaError_t j = cudaSuccess;
    for (int g = 0; g < queued && j == cudaSuccess; ++g) j = cudaStreamWaitEvent(user, h.stepped[g], 0);
    if (j == cudaSuccess) j = cudaEventRecord(h.out_done, h.d2h);
    if (j == cudaSuccess) j = cudaStreamWaitEvent(user, h.out_done, 0);
    if (what) return host_error(e, what);
    if (rc) return rc;
    if (j != cudaSuccess) return host_error(j, "stream join");
    return 0;
}

// ---------------------------------------------------------------------------
// Days from host daily weather: per group of columns, the group's days of
// weather copied in (tens of bytes per cell-day), its hourly forcing generated
// on the device, its hours stepped and its state copied out, the groups on the
// library's streams so one group's generation and copies overlap the others'
// hours.
// ---------------------------------------------------------------------------
extern "C" int ibis_day_host_f32(float* prog, const float* stat, const float* host_daily, float* daily,
                                 const float* lat, float* forc, float* diag, float* acc, float* host_prog, int ncell,
                                 int ld, int nday, int jday0, int day0, unsigned int seed, unsigned int dflags,
                                 const IbisParams* params, int* status, int group, int config, void* stream) {
    if (!prog || !stat || !host_daily || !daily || !lat || !forc || !params) return -EINVAL;
    if (ncell < 0 || nday < 0 || ld < ncell || ld % 32 || group < 0 || group % 32) return -EINVAL;
    if (config < -1 || config >= ibis::kNumConfigs || (config >= 0 && ibis::kConfigs[config].form == 1))
        return -EINVAL;
    if (day0 < 0 || jday0 < 1 || jday0 > 366 || (dflags & ~IBIS_DIURNAL_OBSERVED_FIRA)) return -EINVAL;
    if (!(params->dtime > 0.0)) return -EINVAL;
    const int nh = (int)(86400.0 / params->dtime);
    if (nh < 1 || nh > 254 || (double)nh * params->dtime != 86400.0) return -EINVAL;
    if (ncell == 0) return 0;
    const int nstep = nday * nh;
    const int cfg = config >= 0 ? config : (nstep >= ibis::kAccSmemMinSteps ? ibis::kLongFused : ibis::kDefaultFused);
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return -ENODEV;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) return -ENODEV;
    if (group == 0) {
        const int block = ibis::kConfigs[cfg].block;
        const double wave = (double)sms * block * ibis::kConfigs[cfg].minb;
        group = ncell > kHostGroupWaves * wave
                    ? ((ncell + kDayHostAutoGroups - 1) / kDayHostAutoGroups + block - 1) / block * block
                    : (ncell + 31) / 32 * 32;
    }
    const int min_group = ((ncell + kHostMaxGroups - 1) / kHostMaxGroups + 31) / 32 * 32;
    if (group < min_group) group = min_group;
    const int ngroup = (ncell + group - 1) / group;
    std::lock_guard<std::mutex> lock(g_host_mu);
    HostPipe& h = g_host[dev];
    cudaError_t e = host_pipe_init(h);
    if (e != cudaSuccess) return host_error(e, "stream setup", "ibis_day_host_f32");
    cudaStream_t user = (cudaStream_t)stream;
    if ((e = cudaEventRecord(h.start, user)) != cudaSuccess) return host_error(e, "event record", "ibis_day_host_f32");
    e = cudaStreamWaitEvent(h.h2d, h.start, 0);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(h.d2h, h.start, 0);
    for (int k = 0; k < kHostStreams && k < ngroup && e == cudaSuccess; ++k)
        e = cudaStreamWaitEvent(h.comp[k], h.start, 0);
    if (e != cudaSuccess) return host_error(e, "stream wait", "ibis_day_host_f32");
    const size_t pitch = (size_t)ld * sizeof(float);
    int rc = 0, queued = 0;
    const char* what = nullptr;
    for (int g = 0; g < ngroup && !rc && !what; ++g) {
        const int c0 = g * group, n = ncell - c0 < group ? ncell - c0 : group;
        cudaStream_t cs = h.comp[g % kHostStreams];
        if (nday > 0) {
            e = cudaMemcpy2DAsync(daily + c0, pitch, host_daily + c0, pitch, (size_t)n * sizeof(float),
                                  (size_t)nday * IBIS_DAILY_COUNT, cudaMemcpyHostToDevice, h.h2d);
            if (e == cudaSuccess) e = cudaEventRecord(h.landed[g], h.h2d);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(cs, h.landed[g], 0);
            if (e != cudaSuccess) { what = "weather copy"; break; }
            rc = ibis::diurnal(daily + c0, lat + c0, nullptr, nullptr, forc + c0, n, ld, nday, jday0, day0,
                               (float)params->dtime, seed, dflags, cs, "ibis_day_host_f32", c0);
            if (!rc)
                rc = ibis::hourly_step<float>(prog + c0, stat + c0, forc + c0, diag ? diag + c0 : nullptr,
                                              acc ? acc + c0 : nullptr, n, ld, nstep, params, status, cs, nullptr,
                                              cfg, c0);
        }
        const cudaError_t r = cudaEventRecord(h.stepped[g], cs);
        if (r != cudaSuccess) { what = "event record"; e = r; break; }
        queued = g + 1;
        if (rc || !host_prog) continue;
        e = cudaStreamWaitEvent(h.d2h, h.stepped[g], 0);
        if (e == cudaSuccess)
            e = cudaMemcpy2DAsync(host_prog + c0, pitch, prog + c0, pitch, (size_t)n * sizeof(float), IBIS_PROG_COUNT,
                                  cudaMemcpyDeviceToHost, h.d2h);
        if (e != cudaSuccess) what = "state copy";
    }
    cudaError_t j = cudaSuccess;
    for (int g = 0; g < queued && j == cudaSuccess; ++g) j = cudaStreamWaitEvent(user, h.stepped[g], 0);
    if (j == cudaSuccess) j = cudaEventRecord(h.out_done, h.d2h);
    if (j == cudaSuccess) j = cudaStreamWaitEvent(user, h.out_done, 0);
    if (what) return host_error(e, what, "ibis_day_host_f32");
    if (rc) return rc;
    if (j != cudaSuccess) return host_error(j, "stream join", "ibis_day_host_f32");
    return 0;
}
