// Kernels and host-side launch helpers of the hourly step (included by one
// translation unit per precision: ibis_step_f32.cu and ibis_step_f64.cu).
#pragma once
#include <errno.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include "ibis_step.cuh"

#ifndef IBIS_SMEM_STATE
#define IBIS_SMEM_STATE 1
#endif

namespace ibis {

// Launch configurations.  form 0: one fused kernel per launch (all hours in
// registers/shared memory); form 1: a surface kernel and a ground kernel per
// hour; form 2: the fused kernel with each hour's forcing brought into shared
// memory by bulk copies while the hour before it runs.  block/minb are the
// block size and the minimum resident blocks per SM promised to the compiler
// (__launch_bounds__), i.e. the register budget.
struct LaunchConfig {
    int form, block, minb, block2, minb2;
};
constexpr LaunchConfig kConfigs[] = {
    {0, 128, 2, 0, 0}, {0, 64, 4, 0, 0},  {0, 96, 2, 0, 0},    {0, 128, 3, 0, 0},
    {0, 160, 1, 0, 0}, {0, 192, 1, 0, 0}, {0, 224, 1, 0, 0},   {0, 256, 1, 0, 0},
    {1, 128, 2, 128, 3}, {1, 256, 1, 256, 2}, {1, 128, 3, 128, 4}, {2, 224, 1, 0, 0}};
constexpr int kNumConfigs = sizeof(kConfigs) / sizeof(kConfigs[0]);
constexpr int kDefaultFused = 0;
constexpr int kLongFused = 6;      // ibis_step_f32's choice for launches of kAccSmemMinSteps hours or more
constexpr int kDefaultSplit = 8;

// FP32 kernels keep each column's prognostic state in shared memory (array of
// structures: the 71-word stride is odd, so a warp's accesses to one field fall
// in 32 different banks); that frees registers for the step's temporaries.
template <typename R>
struct StateInSmem {
    static constexpr bool value = IBIS_SMEM_STATE && sizeof(R) == 4;
};

template <typename R>
__device__ __forceinline__ void load_col(Col<R>& c, const R* __restrict__ p, int ld) {
    auto g = [&](int plane) { return p[(size_t)plane * ld]; };
#pragma unroll
    for (int k = 0; k < NL; ++k) {
        c.tsoi[k] = g(IBIS_PROG_TSOI + k);
        c.wsoi[k] = g(IBIS_PROG_WSOI + k);
        c.wisoi[k] = g(IBIS_PROG_WISOI + k);
    }
    c.tg = g(IBIS_PROG_TG); c.wpud = g(IBIS_PROG_WPUD); c.wipud = g(IBIS_PROG_WIPUD);
#pragma unroll
    for (int k = 0; k < NB; ++k) c.tsoi_deep[k] = g(IBIS_PROG_TSOI_DEEP + k);
    c.fi = g(IBIS_PROG_FI);
#pragma unroll
    for (int k = 0; k < NS; ++k) { c.tsno[k] = g(IBIS_PROG_TSNO + k); c.hsno[k] = g(IBIS_PROG_HSNO + k); }
    c.ti = g(IBIS_PROG_TI); c.tlsub = g(IBIS_PROG_TLSUB);
    c.tu = g(IBIS_PROG_TU); c.ts = g(IBIS_PROG_TS); c.tl = g(IBIS_PROG_TL);
    c.t12 = g(IBIS_PROG_T12); c.t34 = g(IBIS_PROG_T34); c.q12 = g(IBIS_PROG_Q12); c.q34 = g(IBIS_PROG_Q34);
    c.wliqu = g(IBIS_PROG_WLIQU); c.wliqs = g(IBIS_PROG_WLIQS); c.wliql = g(IBIS_PROG_WLIQL);
    c.wsnou = g(IBIS_PROG_WSNOU); c.wsnos = g(IBIS_PROG_WSNOS); c.wsnol = g(IBIS_PROG_WSNOL);
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        c.ci_u[j] = g(IBIS_PROG_CI_UPPER + j); c.gs_u[j] = g(IBIS_PROG_GS_UPPER + j); c.cs_u[j] = g(IBIS_PROG_CS_UPPER + j);
    }
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        c.ci_l[j] = g(IBIS_PROG_CI_LOWER + j); c.gs_l[j] = g(IBIS_PROG_GS_LOWER + j); c.cs_l[j] = g(IBIS_PROG_CS_LOWER + j);
    }
    c.a10su = g(IBIS_PROG_A10SCALPARAMU); c.a10du = g(IBIS_PROG_A10DAYLIGHTU);
    c.a10sl = g(IBIS_PROG_A10SCALPARAML); c.a10dl = g(IBIS_PROG_A10DAYLIGHTL);
    c.firefac = g(IBIS_PROG_FIREFAC); c.nytimes = g(IBIS_PROG_NYTIMES); c.nfirestep = g(IBIS_PROG_NFIRESTEP);
    c.sdry = g(IBIS_PROG_SDRY); c.nfirestep_vpd = g(IBIS_PROG_NFIRESTEP_VPD); c.sdry_vpd = g(IBIS_PROG_SDRY_VPD);
}

template <typename R>
__device__ __forceinline__ R store_col(const Col<R>& c, R* __restrict__ p, int ld) {
    R sum = R(0.0);
    auto s = [&](int plane, R v) { p[(size_t)plane * ld] = v; sum = sum + v; };
#pragma unroll
    for (int k = 0; k < NL; ++k) {
        s(IBIS_PROG_TSOI + k, c.tsoi[k]); s(IBIS_PROG_WSOI + k, c.wsoi[k]); s(IBIS_PROG_WISOI + k, c.wisoi[k]);
    }
    s(IBIS_PROG_TG, c.tg); s(IBIS_PROG_WPUD, c.wpud); s(IBIS_PROG_WIPUD, c.wipud);
#pragma unroll
    for (int k = 0; k < NB; ++k) s(IBIS_PROG_TSOI_DEEP + k, c.tsoi_deep[k]);
    s(IBIS_PROG_FI, c.fi);
#pragma unroll
    for (int k = 0; k < NS; ++k) { s(IBIS_PROG_TSNO + k, c.tsno[k]); s(IBIS_PROG_HSNO + k, c.hsno[k]); }
    s(IBIS_PROG_TI, c.ti); s(IBIS_PROG_TLSUB, c.tlsub);
    s(IBIS_PROG_TU, c.tu); s(IBIS_PROG_TS, c.ts); s(IBIS_PROG_TL, c.tl);
    s(IBIS_PROG_T12, c.t12); s(IBIS_PROG_T34, c.t34); s(IBIS_PROG_Q12, c.q12); s(IBIS_PROG_Q34, c.q34);
    s(IBIS_PROG_WLIQU, c.wliqu); s(IBIS_PROG_WLIQS, c.wliqs); s(IBIS_PROG_WLIQL, c.wliql);
    s(IBIS_PROG_WSNOU, c.wsnou); s(IBIS_PROG_WSNOS, c.wsnos); s(IBIS_PROG_WSNOL, c.wsnol);
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        s(IBIS_PROG_CI_UPPER + j, c.ci_u[j]); s(IBIS_PROG_GS_UPPER + j, c.gs_u[j]); s(IBIS_PROG_CS_UPPER + j, c.cs_u[j]);
    }
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        s(IBIS_PROG_CI_LOWER + j, c.ci_l[j]); s(IBIS_PROG_GS_LOWER + j, c.gs_l[j]); s(IBIS_PROG_CS_LOWER + j, c.cs_l[j]);
    }
    s(IBIS_PROG_A10SCALPARAMU, c.a10su); s(IBIS_PROG_A10DAYLIGHTU, c.a10du);
    s(IBIS_PROG_A10SCALPARAML, c.a10sl); s(IBIS_PROG_A10DAYLIGHTL, c.a10dl);
    s(IBIS_PROG_FIREFAC, c.firefac); s(IBIS_PROG_NYTIMES, c.nytimes); s(IBIS_PROG_NFIRESTEP, c.nfirestep);
    s(IBIS_PROG_SDRY, c.sdry); s(IBIS_PROG_NFIRESTEP_VPD, c.nfirestep_vpd); s(IBIS_PROG_SDRY_VPD, c.sdry_vpd);
    return sum;
}

template <typename R>
__device__ __forceinline__ Forc<R> load_forc(const R* __restrict__ f, int ld) {
    Forc<R> F;
    auto g = [&](int plane) { return __ldg(f + (size_t)plane * ld); };
    F.ta = g(IBIS_FORC_TA); F.qa = g(IBIS_FORC_QA); F.ua = g(IBIS_FORC_UA); F.ps = g(IBIS_FORC_PSURF);
    F.cosz = g(IBIS_FORC_COSZEN);
    F.sd[0] = g(IBIS_FORC_SOLAD); F.sd[1] = g(IBIS_FORC_SOLAD + 1);
    F.si[0] = g(IBIS_FORC_SOLAI); F.si[1] = g(IBIS_FORC_SOLAI + 1);
    F.fira = g(IBIS_FORC_FIRA); F.rain = g(IBIS_FORC_RAINA); F.snow = g(IBIS_FORC_SNOWA);
    return F;
}

// Accumulators of the fused kernel kept in shared memory for the launch: plane p
// of thread t at sacc[p * BLOCK + t] (consecutive threads, consecutive banks)
// for the kAccOnChip planes every day loop keeps, then their compensation
// planes; the optional planes from kAccOnChip on stay in global memory.  Only
// the planes the flags write move: loaded before the first hour, stored after
// the last, so the hourly read-modify-writes stay on chip.
__device__ __forceinline__ bool acc_plane_used(int p, unsigned flags) {
    const int q = p < IBIS_ACC_COUNT ? p : p - IBIS_ACC_COUNT;
    const bool last_value = q == IBIS_ACC_STRESSTU_LAST || q == IBIS_ACC_STRESSTL_LAST;    // no Kahan terms
    if (p >= IBIS_ACC_COUNT && (!(flags & IBIS_FLAG_KAHAN) || last_value)) return false;
    if (q == IBIS_ACC_CH4) return (flags & IBIS_FLAG_CH4) != 0;
    if (q >= IBIS_ACC_TSOI_MEAN && q < IBIS_ACC_AFSENA) return (flags & IBIS_FLAG_SOIL_MEANS) != 0;
    if (q >= IBIS_ACC_ET_TRANS && q <= IBIS_ACC_ET_SNOWSUB)
        return (flags & IBIS_FLAG_ACC) && (flags & IBIS_FLAG_ETPARTS);
    if (q == IBIS_ACC_NEE_NIGHT || q == IBIS_ACC_NEE_DAY)
        return (flags & IBIS_FLAG_ACC) && (flags & IBIS_FLAG_NEEPARTS);
    return (flags & IBIS_FLAG_ACC) != 0;
}

// The planes move in batches of kAccMoveBatch: all loads of a batch are issued
// before its stores, so a thread has that many global loads in flight instead
// of waiting out one load latency per plane at the start of every launch.
constexpr int kAccMoveBatch = 16;

template <typename R, bool TO_SMEM>
__device__ __forceinline__ void acc_move(R* __restrict__ g, int ld, R* __restrict__ sacc, int sld, unsigned flags) {
    constexpr int kPlanes = 2 * kAccOnChip;
    auto global_plane = [](int p) { return p < kAccOnChip ? p : p - kAccOnChip + IBIS_ACC_COUNT; };
#pragma unroll 1
    for (int p0 = 0; p0 < kPlanes; p0 += kAccMoveBatch) {
        R v[kAccMoveBatch];
        bool use[kAccMoveBatch];
#pragma unroll
        for (int j = 0; j < kAccMoveBatch; ++j) {
            const int p = p0 + j;
            use[j] = p < kPlanes && acc_plane_used(global_plane(p), flags);
            if (TO_SMEM) v[j] = use[j] ? g[(size_t)global_plane(p) * ld] : R(0.0);
            else v[j] = use[j] ? sacc[p * sld] : R(0.0);
        }
#pragma unroll
        for (int j = 0; j < kAccMoveBatch; ++j) {
            const int p = p0 + j;
            if (!use[j]) continue;
            if (TO_SMEM) sacc[p * sld] = v[j];
            else g[(size_t)global_plane(p) * ld] = v[j];
        }
    }
}

// Whether a fused configuration keeps its accumulators in shared memory: the
// column state plus the on-chip accumulator planes of MINB resident blocks must fit
// the SM's 228 KB (1 KB reserved per block).  Launches of fewer than
// kAccSmemMinSteps hours keep them in global memory instead (ACCSM = false):
// the on-chip copy only pays back over several hours, and the larger
// shared-memory carveout leaves less L1 for the register spills.
template <typename R, int BLOCK, int MINB, bool ACCSM = true>
struct AccInSmem {
    static constexpr bool value =
        ACCSM && StateInSmem<R>::value &&
        ((sizeof(Col<R>) + 2 * kAccOnChip * sizeof(R)) * BLOCK + 1024) * MINB <= 228 * 1024;
};
constexpr int kAccSmemMinSteps = 4;

// The uniform parameter source of a kernel: with X3 the one that compiles in the
// IBIS 3.0 extensions of the step (any IBIS_FLAGS_X3 flag selects those kernels).
template <typename R, bool X3>
__device__ __forceinline__ auto uniform_source(const DevParams<R>& P) {
    if constexpr (X3) return UniformQ3<R>{{P}};
    else return UniformQ<R>{P};
}

// Status word written by the kernels: [0] bit 0 = a column left the step with a
// non-finite prognostic value; [1] = smallest such cell index (INT_MAX if none).
template <typename R, int NT, bool SU, bool SL, int BLOCK, int MINB, bool ACCSM, bool X3>
__global__ void __launch_bounds__(BLOCK, MINB) hourly_step_kernel(R* __restrict__ prog, const R* __restrict__ stat,
                                                             const R* __restrict__ forc, R* __restrict__ diag,
                                                             R* __restrict__ acc, int ncell, int ld, int nstep,
                                                             long long forc_stride, const DevParams<R> P,
                                                             int* __restrict__ status) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ncell) return;
    extern __shared__ unsigned char smem_raw[];
    Col<R> creg;
    Col<R>* cp;
    if constexpr (StateInSmem<R>::value) cp = reinterpret_cast<Col<R>*>(smem_raw) + threadIdx.x;
    else cp = &creg;
    Col<R>& c = *cp;
    load_col(c, prog + i, ld);
    Stat<R> S{stat + i, ld};
    Diag<R> D{diag ? diag + i : nullptr, ld};
    constexpr bool kAccSmem = AccInSmem<R, BLOCK, MINB, ACCSM>::value;
    // with the accumulators on chip the view always points at shared memory
    // (acc == nullptr comes with no accumulator flags, so nothing is added)
    R* const sacc = kAccSmem ? reinterpret_cast<R*>(smem_raw + BLOCK * sizeof(Col<R>)) + threadIdx.x : nullptr;
    const bool kahan = (P.flags & IBIS_FLAG_KAHAN) != 0;
    using AccT = Acc<R, kAccSmem ? BLOCK : 0>;
    AccT A = kAccSmem ? AccT{sacc, ld, kahan, true, acc ? acc + i : nullptr} : AccT{acc ? acc + i : nullptr, ld, kahan};
    if (kAccSmem && acc) acc_move<R, true>(acc + i, ld, sacc, BLOCK, P.flags);
#pragma unroll 1
    for (int s = 0; s < nstep; ++s) {
        Forc<R> F = load_forc(forc + (size_t)s * forc_stride + i, ld);
        A.last = (s + 1 == nstep);
        column_step<R, NT, SU, SL>(c, F, S, D, A, P, uniform_source<R, X3>(P));
    }
    if (kAccSmem && acc) acc_move<R, false>(acc + i, ld, sacc, BLOCK, P.flags);
    R sum = store_col(c, prog + i, ld);
    if (status && !finite(sum)) {
        atomicOr(status, 1);
        atomicMin(status + 1, i + P.cell0);
    }
}

// ---- Fused kernel with the forcing staged by the bulk-copy (TMA) engine (form 2)
//
// Each hour's forcing tile -- IBIS_FORC_COUNT planes x the block's cells, one
// untiled cp.async.bulk per plane -- lands in shared memory while the block
// computes the hour before it.  Thread 0 issues hour s+1 as soon as every live
// thread of the block has copied hour s out of the buffer (the "empty"
// mbarrier counts the live threads, the "full" mbarrier counts the bytes in);
// the copy then has the whole of hour s to land.  One buffer is enough: the
// threads read their 12 values at the top of the hour.  Every wait is bounded:
// a wait that gives up sets the block's abort word (no copy is issued after it
// and later waits return at once) and status[0] bit 2, and the block finishes
// its hours on whatever the buffer holds; thread 0 then waits, again bounded,
// for its last copy to land before it leaves.
constexpr int kStageWaitLimit = 1 << 22;

template <typename R, int BLOCK>
struct ForcStage {
    static_assert(BLOCK % 4 == 0, "a plane's tile must start on a 16-byte boundary");
    static constexpr size_t data = (size_t)IBIS_FORC_COUNT * BLOCK * sizeof(R);
    static constexpr size_t bytes = data + 32;  // + full, empty mbarriers, abort and last-issued words
};

__device__ __forceinline__ unsigned smem_addr(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* b, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(b)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(unsigned long long* b) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(b)) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long* b, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(b)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned long long* b, unsigned parity) {
    unsigned done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_addr(b)), "r"(parity)
        : "memory");
    return done != 0;
}

// Wait for the phase of `b` with the given parity to complete: true when it
// did, false when the block's abort word is set or kStageWaitLimit polls pass.
__device__ __forceinline__ bool stage_wait(unsigned long long* b, unsigned parity, volatile int* abort_word) {
    for (int k = 0; k < kStageWaitLimit; ++k) {
        if (mbar_try_wait(b, parity)) return true;
        if (*abort_word) return false;
    }
    return false;
}

// Issue hour `h`'s forcing tile into `buf`: plane p of the tile at buf[p * BLOCK].
// `bytes` per plane is the live cells rounded up to 4 (16 bytes), which stays
// inside a plane of ld >= ncell cells because ld and the tile start are
// multiples of 4 cells.
template <typename R, int BLOCK>
__device__ __forceinline__ void stage_issue(R* buf, const R* __restrict__ src, int ld, unsigned bytes,
                                            unsigned long long* full) {
    mbar_arrive_expect_tx(full, bytes * IBIS_FORC_COUNT);
#pragma unroll
    for (int p = 0; p < IBIS_FORC_COUNT; ++p)
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                         smem_addr(buf + p * BLOCK)),
                     "l"(src + (size_t)p * ld), "r"(bytes), "r"(smem_addr(full))
                     : "memory");
}

template <typename R>
__device__ __forceinline__ Forc<R> read_forc_tile(const R* t, int block) {
    Forc<R> F;
    auto g = [&](int plane) { return t[plane * block]; };
    F.ta = g(IBIS_FORC_TA); F.qa = g(IBIS_FORC_QA); F.ua = g(IBIS_FORC_UA); F.ps = g(IBIS_FORC_PSURF);
    F.cosz = g(IBIS_FORC_COSZEN);
    F.sd[0] = g(IBIS_FORC_SOLAD); F.sd[1] = g(IBIS_FORC_SOLAD + 1);
    F.si[0] = g(IBIS_FORC_SOLAI); F.si[1] = g(IBIS_FORC_SOLAI + 1);
    F.fira = g(IBIS_FORC_FIRA); F.rain = g(IBIS_FORC_RAINA); F.snow = g(IBIS_FORC_SNOWA);
    return F;
}

// The staged kernel's shared memory: column state, the on-chip accumulators,
// then the forcing tile and its barriers (16-byte aligned).
template <typename R, int BLOCK, int MINB>
struct StagedSmem {
    static constexpr size_t col = (size_t)BLOCK * sizeof(Col<R>);
    static constexpr size_t acc = (size_t)BLOCK * 2 * kAccOnChip * sizeof(R);
    static constexpr size_t stage_off = (col + acc + 15) / 16 * 16;
    static constexpr size_t total = stage_off + ForcStage<R, BLOCK>::bytes;
};

// Callers guarantee: `forc` 16-byte aligned, forc_stride and ld multiples of 4
// (launch_staged checks and otherwise runs the unstaged kernel).
// Give up on the staged forcing: no further copies, later waits return at once.
__device__ __forceinline__ void stage_give_up(volatile int* abort_word, int* status) {
    *abort_word = 1;
    if (status) atomicOr(status, 4);
}

template <typename R, int NT, bool SU, bool SL, int BLOCK, int MINB, bool X3>
__global__ void __launch_bounds__(BLOCK, MINB) hourly_step_staged_kernel(
    R* __restrict__ prog, const R* __restrict__ stat, const R* __restrict__ forc, R* __restrict__ diag,
    R* __restrict__ acc, int ncell, int ld, int nstep, long long forc_stride, const DevParams<R> P,
    int* __restrict__ status) {
    static_assert(sizeof(R) == 4 && StateInSmem<R>::value, "the staged form is the FP32 shared-memory kernel");
    static_assert(AccInSmem<R, BLOCK, MINB>::value, "the staged form keeps the accumulators on chip");
    using SM = StagedSmem<R, BLOCK, MINB>;
    static_assert((SM::total + 1024) * MINB <= 228 * 1024, "staged shared memory exceeds the SM");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    // fixed offsets from the shared-memory base, so none of them holds a register across the hour
    R* const tile = reinterpret_cast<R*>(smem_raw + SM::stage_off);
    unsigned long long* const full = reinterpret_cast<unsigned long long*>(smem_raw + SM::stage_off +
                                                                           ForcStage<R, BLOCK>::data);
    unsigned long long* const empty = full + 1;
    volatile int* const abort_word = reinterpret_cast<volatile int*>(full + 2);
    volatile int* const last_issued = abort_word + 1;
    const int i0 = blockIdx.x * BLOCK;
    if (threadIdx.x == 0) {
        const int nlive = ncell - i0 < BLOCK ? ncell - i0 : BLOCK;
        mbar_init(full, 1);
        mbar_init(empty, (unsigned)nlive);
        *abort_word = 0;
        *last_issued = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();  // every thread of the block reaches this before any leaves
    // bytes per plane: the block's live cells rounded up to 4 (16 bytes)
    auto plane_bytes = [&]() {
        const int nlive = ncell - i0 < BLOCK ? ncell - i0 : BLOCK;
        return (unsigned)((nlive + 3) & ~3) * (unsigned)sizeof(R);
    };
    if (threadIdx.x == 0 && nstep > 0) stage_issue<R, BLOCK>(tile, forc + i0, ld, plane_bytes(), full);
    const int i = i0 + threadIdx.x;
    if (i >= ncell) return;
    Col<R>& c = *(reinterpret_cast<Col<R>*>(smem_raw) + threadIdx.x);
    load_col(c, prog + i, ld);
    Stat<R> S{stat + i, ld};
    Diag<R> D{diag ? diag + i : nullptr, ld};
    R* const sacc = reinterpret_cast<R*>(smem_raw + SM::col) + threadIdx.x;
    const bool kahan = (P.flags & IBIS_FLAG_KAHAN) != 0;
    using AccT = Acc<R, BLOCK>;
    AccT A{sacc, ld, kahan, true, acc ? acc + i : nullptr};
    if (acc) acc_move<R, true>(acc + i, ld, sacc, BLOCK, P.flags);
#pragma unroll 1
    for (int s = 0; s < nstep; ++s) {
        const unsigned parity = (unsigned)(s & 1);
        if (!stage_wait(full, parity, abort_word)) stage_give_up(abort_word, status);
        Forc<R> F = read_forc_tile(tile + threadIdx.x, BLOCK);
        mbar_arrive(empty);
        if (threadIdx.x == 0 && s + 1 < nstep && !*abort_word) {
            if (stage_wait(empty, parity, abort_word)) {
                stage_issue<R, BLOCK>(tile, forc + (size_t)(s + 1) * forc_stride + i0, ld, plane_bytes(), full);
                *last_issued = s + 1;
            } else {
                stage_give_up(abort_word, status);
            }
        }
        A.last = (s + 1 == nstep);
        column_step<R, NT, SU, SL>(c, F, S, D, A, P, uniform_source<R, X3>(P));
    }
    if (acc) acc_move<R, false>(acc + i, ld, sacc, BLOCK, P.flags);
    R sum = store_col(c, prog + i, ld);
    if (threadIdx.x == 0 && *abort_word) {
        // after a give-up the last copy may still be landing: let it finish
        // (bounded) before the block's shared memory is released
        volatile int never = 0;
        stage_wait(full, (unsigned)(*last_issued & 1), &never);
    }
    if (status && !finite(sum)) {
        atomicOr(status, 1);
        atomicMin(status + 1, i + P.cell0);
    }
}

// Two-kernel form of one hour: the surface phase writes the hand-off values to
// `mid` (kMidCount planes), the ground phase reads them.  Both phases load the
// column from `prog` and write back what they change.
template <typename R, bool SU, bool SL, int BLOCK, int MINB, bool X3>
__global__ void __launch_bounds__(BLOCK, MINB) surface_kernel(R* __restrict__ prog, const R* __restrict__ stat,
                                                                    const R* __restrict__ forc, R* __restrict__ diag,
                                                                    R* __restrict__ mid, int ncell, int ld,
                                                                    const DevParams<R> P) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ncell) return;
    extern __shared__ unsigned char smem_raw[];
    Col<R> creg;
    Col<R>* cp;
    if constexpr (StateInSmem<R>::value) cp = reinterpret_cast<Col<R>*>(smem_raw) + threadIdx.x;
    else cp = &creg;
    Col<R>& c = *cp;
    load_col(c, prog + i, ld);
    Stat<R> S{stat + i, ld};
    Diag<R> D{diag ? diag + i : nullptr, ld};
    Forc<R> F = load_forc(forc + i, ld);
    Mid<R> M;
    surface_phase<R, SU, SL>(c, F, S, D, P, uniform_source<R, X3>(P), M);
    mid_store(M, mid + i, ld);
    store_col(c, prog + i, ld);
}

template <typename R, int NT, int BLOCK, int MINB, bool X3>
__global__ void __launch_bounds__(BLOCK, MINB) ground_kernel(R* __restrict__ prog, const R* __restrict__ stat,
                                                                   const R* __restrict__ forc, R* __restrict__ diag,
                                                                   R* __restrict__ acc, const R* __restrict__ mid,
                                                                   int ncell, int ld, const DevParams<R> P,
                                                                   int* __restrict__ status) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ncell) return;
    extern __shared__ unsigned char smem_raw[];
    Col<R> creg;
    Col<R>* cp;
    if constexpr (StateInSmem<R>::value) cp = reinterpret_cast<Col<R>*>(smem_raw) + threadIdx.x;
    else cp = &creg;
    Col<R>& c = *cp;
    load_col(c, prog + i, ld);
    Stat<R> S{stat + i, ld};
    Diag<R> D{diag ? diag + i : nullptr, ld};
    Acc<R> A{acc ? acc + i : nullptr, ld, (P.flags & IBIS_FLAG_KAHAN) != 0};
    Forc<R> F = load_forc(forc + i, ld);
    Mid<R> M;
    mid_load(M, mid + i, ld);
    ground_phase<R, NT>(c, F, S, D, A, P, uniform_source<R, X3>(P), M);
    R sum = store_col(c, prog + i, ld);
    if (status && !finite(sum)) {
        atomicOr(status, 1);
        atomicMin(status + 1, i + P.cell0);
    }
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

template <typename R>
static DevParams<R> make_dev_params(const IbisParams& h) {
    DevParams<R> d;
    memset(&d, 0, sizeof(d));
#define IBIS_S(name) d.name = (R)h.name;
#define IBIS_A(name, n) for (int q = 0; q < n; ++q) d.name[q] = (R)h.name[q];
    IBIS_PARAM_LIST(IBIS_S, IBIS_A)
#undef IBIS_S
#undef IBIS_A
    d.flags = h.flags;
    d.tfac = (R)(1.0 / pow(0.999, h.cappa));
    d.vonk2 = (R)pow(h.vonk, 2.0);
    d.cdmax = (R)(300.0 / (2.0 * h.dtime));
    d.zweight = (R)exp(-1.0 / (10.0 * 86400.0 / h.dtime));
    d.wliqmin = (R)(0.001 * (h.dtime / 3600.0) * (h.wliqumax / 0.2));
    d.wsnomin = (R)(0.001 * (h.dtime / 3600.0) * (h.wsnoumax / 2.0));
    d.znorm = (R)(1.0 - exp(h.stressfac));
    d.rdt = (R)(1.0 / h.dtime);
    d.zir = (R)(4.0 * 0.95 * h.stef);
    for (int k = 1; k < NL; ++k) {
        d.sw_hm[k] = 0.5 * (h.hsoi[k - 1] + h.hsoi[k]);
        d.sw_wp[k] = 0.5 * h.hsoi[k] / d.sw_hm[k];
        d.sw_wm[k] = 1.0 - d.sw_wp[k];
    }
    for (int k = 0; k < NL; ++k) {
        double hb = k == 0 ? 0.5 * h.hsoi[0] : 0.5 * h.hsoi[k - 1] + 0.5 * h.hsoi[k];
        d.sw_hb[k] = hb > 1e-30 ? hb : 1e-30;
        double hp = k < NL - 1 ? 0.5 * (h.hsoi[k] + h.hsoi[k + 1]) : 1.0;
        d.sw_hp[k] = hp > 1e-30 ? hp : 1e-30;
        const int km1 = k > 0 ? k - 1 : 0, kp1 = k < NL - 1 ? k + 1 : k;
        d.sw_rhm[k] = k > 0 ? 1.0 / d.sw_hm[k] : 0.0;
        d.sw_rhb[k] = 1.0 / d.sw_hb[k];
        d.sw_rhp[k] = 1.0 / d.sw_hp[k];
        d.sw_c1[k] = 0.5 * h.hsoi[k] / d.sw_hb[k];
        d.sw_c3[k] = 0.5 * h.hsoi[kp1] / d.sw_hp[k];
        d.sw_c5[k] = 0.5 * h.hsoi[km1] / d.sw_hb[k];
        d.sw_c6[k] = 0.5 * h.hsoi[k] / d.sw_hp[k];
    }
    d.rdt64 = 1.0 / h.dtime;
    d.rrhow64 = 1.0 / h.rhow;
    for (int k = 0; k < NL; ++k) {
        d.sw32_wp[k] = (float)d.sw_wp[k]; d.sw32_wm[k] = (float)d.sw_wm[k];
        d.sw32_rhm[k] = (float)d.sw_rhm[k]; d.sw32_rhb[k] = (float)d.sw_rhb[k]; d.sw32_rhp[k] = (float)d.sw_rhp[k];
        d.sw32_c1[k] = (float)d.sw_c1[k]; d.sw32_c3[k] = (float)d.sw_c3[k];
        d.sw32_c5[k] = (float)d.sw_c5[k]; d.sw32_c6[k] = (float)d.sw_c6[k];
    }
    // respiration tables formed in float32 as the reference does (loops_gswp3.py:185-190)
    const float per_s = (float)(h.ndaypy * 86400.0), mol = (float)(1000.0 / 12.0);
    for (int j = 0; j < 12; ++j) {
        d.rwood_s[j] = (R)(((float)h.rwood[j] / per_s) * mol);
        d.rroot_s[j] = (R)(((float)h.rroot[j] / per_s) * mol);
        d.keep[j] = (R)(1.0f - (float)h.rgrowth[j]);
    }
    // crop_vfac's increments (loops.py:218-231), float32 values as the reference forms them
    for (int j = 0; j < 12; ++j) d.crop_inc[j] = (R)0.0;
    if (h.crop_c4_share < 0.0) {
        d.crop_inc[10] = (R)(float)(h.crop_vmax_scale_c4 - 1.0);
        d.crop_inc[11] = (R)(float)(h.crop_vmax_scale_c3 - 1.0);
    } else {
        const double qc = h.crop_c4_share > 1.0 ? 1.0 : h.crop_c4_share;
        const double s_mix = (1.0 - qc) * h.crop_vmax_scale_c3 + qc * h.crop_vmax_scale_c4;
        d.crop_inc[10] = d.crop_inc[11] = (R)(float)(s_mix - 1.0);
    }
    d.ch4_w = (R)(float)(h.dtime / 86400.0);
    d.rh_conv = (R)(float)(12.0e-3 * 86400.0);
    double top = 0.0, tot = 0.0;
    for (int k = 0; k < NL; ++k) {
        double bot = top + h.hsoi[k];
        double w = h.z_wt_ref - top;
        w = w < 0.0 ? 0.0 : (w > h.hsoi[k] ? h.hsoi[k] : w);
        d.ch4_wtop[k] = (R)w;
        tot += w;
        d.hsoi_top[k] = (R)top;
        d.hsoi_bot[k] = (R)bot;
        top = bot;
    }
    d.ch4_wtot = (R)(tot > 1e-12 ? tot : 1e-12);
    for (int b = 0; b < 3; ++b) {
        double btop = 0.0, btot = 0.0;
        for (int k = 0; k < NL; ++k) {
            double w = h.ch4b_z_wt_ref[b] - btop;
            w = w < 0.0 ? 0.0 : (w > h.hsoi[k] ? h.hsoi[k] : w);
            d.ch4b_wtop[b][k] = (R)w;
            btot += w;
            btop += h.hsoi[k];
        }
        d.ch4b_wtot[b] = (R)(btot > 1e-12 ? btot : 1e-12);
    }
    return d;
}

// The SM's 256 KB unified array is split between shared memory and L1, and L1
// caches the register spills of these kernels.  Ask for the smallest
// shared-memory carveout that holds `smem` bytes for every block the register
// budget lets reside (228 KB of shared memory per SM on sm_100, 1 KB reserved
// per block), so the rest stays L1, and allow `smem_max` dynamic bytes.
template <typename K>
cudaError_t fit_smem(K k, int block, size_t smem, size_t smem_max) {
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, k);
    if (e != cudaSuccess) return e;
    const int regs = (fa.numRegs + 7) / 8 * 8;
    int blocks = regs > 0 ? 65536 / (block * regs) : 32;
    blocks = blocks < 1 ? 1 : (blocks > 32 ? 32 : blocks);
    const size_t per_sm = 228 * 1024;
    const size_t need = (smem + fa.sharedSizeBytes + 1024) * (size_t)blocks;
    int pct = (int)((need * 100 + per_sm - 1) / per_sm);
    pct = pct > 100 ? 100 : pct;
    if (smem_max > 48 * 1024) {
        e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_max);
        if (e != cudaSuccess) return e;
    }
    return cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, pct);
}

// fit_smem once per kernel instantiation and device (`done` is the caller's
// per-instantiation bit set; a repeated call is harmless).
template <typename K>
cudaError_t fit_smem_once(unsigned long long& done, K k, int block, size_t smem, size_t smem_max) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return fit_smem(k, block, smem, smem_max);
    const unsigned long long bit = 1ull << dev;
    if (done & bit) return cudaSuccess;
    cudaError_t e = fit_smem(k, block, smem, smem_max);
    if (e == cudaSuccess) done |= bit;
    return e;
}

template <typename R, int NT, bool SU, bool SL, int BLOCK, int MINB, bool ACCSM, bool X3>
cudaError_t launch_fused(R* prog, const R* stat, const R* forc, R* diag, R* acc, int ncell, int ld, int nstep,
                         long long fstride, const DevParams<R>& P, int* status, cudaStream_t s) {
    const int grid = (ncell + BLOCK - 1) / BLOCK;
    const size_t col_smem = StateInSmem<R>::value ? BLOCK * sizeof(Col<R>) : 0;
    const size_t acc_smem = AccInSmem<R, BLOCK, MINB, ACCSM>::value ? BLOCK * 2 * kAccOnChip * sizeof(R) : 0;
    const size_t smem = col_smem + acc_smem;
    auto k = hourly_step_kernel<R, NT, SU, SL, BLOCK, MINB, ACCSM, X3>;
    static unsigned long long fitted = 0;
    cudaError_t e = fit_smem_once(fitted, k, BLOCK, col_smem + acc_smem, col_smem + acc_smem);
    if (e != cudaSuccess) return e;
    k<<<grid, BLOCK, smem, s>>>(prog, stat, forc, diag, acc, ncell, ld, nstep, fstride, P, status);
    return cudaGetLastError();
}

// Form 2: the staged fused kernel.  A forcing buffer the bulk copies cannot
// address (start not 16-byte aligned, hour or plane stride not a multiple of 4
// cells) runs the unstaged kernel of the same block size instead: the results
// are the same, only the loads differ.
template <typename R, int NT, bool SU, bool SL, int BLOCK, int MINB, bool X3>
cudaError_t launch_staged(R* prog, const R* stat, const R* forc, R* diag, R* acc, int ncell, int ld, int nstep,
                          long long fstride, const DevParams<R>& P, int* status, cudaStream_t s) {
    if ((reinterpret_cast<uintptr_t>(forc) & 15) != 0 || (fstride & 3) != 0 || (ld & 3) != 0)
        return launch_fused<R, NT, SU, SL, BLOCK, MINB, true, X3>(prog, stat, forc, diag, acc, ncell, ld, nstep,
                                                                  fstride, P, status, s);
    using SM = StagedSmem<R, BLOCK, MINB>;
    const int grid = (ncell + BLOCK - 1) / BLOCK;
    auto k = hourly_step_staged_kernel<R, NT, SU, SL, BLOCK, MINB, X3>;
    static unsigned long long fitted = 0;
    cudaError_t e = fit_smem_once(fitted, k, BLOCK, SM::total, SM::total);
    if (e != cudaSuccess) return e;
    k<<<grid, BLOCK, SM::total, s>>>(prog, stat, forc, diag, acc, ncell, ld, nstep, fstride, P, status);
    return cudaGetLastError();
}

template <typename R, int NT, bool SU, bool SL, int B1, int M1, int B2, int M2, bool X3>
cudaError_t launch_split(R* prog, const R* stat, const R* forc, R* diag, R* acc, R* mid, int ncell, int ld,
                         int nstep, long long fstride, const DevParams<R>& P, int* status, cudaStream_t s) {
    const int g1 = (ncell + B1 - 1) / B1, g2 = (ncell + B2 - 1) / B2;
    const size_t sm1 = StateInSmem<R>::value ? B1 * sizeof(Col<R>) : 0;
    const size_t sm2 = StateInSmem<R>::value ? B2 * sizeof(Col<R>) : 0;
    auto k1 = surface_kernel<R, SU, SL, B1, M1, X3>;
    auto k2 = ground_kernel<R, NT, B2, M2, X3>;
    static unsigned long long fitted1 = 0, fitted2 = 0;
    cudaError_t e = fit_smem_once(fitted1, k1, B1, sm1, sm1);
    if (e == cudaSuccess) e = fit_smem_once(fitted2, k2, B2, sm2, sm2);
    if (e != cudaSuccess) return e;
    for (int h = 0; h < nstep; ++h) {
        const R* f = forc + (size_t)h * fstride;
        k1<<<g1, B1, sm1, s>>>(prog, stat, f, diag, mid, ncell, ld, P);
        k2<<<g2, B2, sm2, s>>>(prog, stat, f, diag, acc, mid, ncell, ld, P, status);
    }
    return cudaGetLastError();
}

template <typename R, int NT, bool SU, bool SL, int CFG, bool X3 = false>
cudaError_t run_config(R* prog, const R* stat, const R* forc, R* diag, R* acc, R* mid, int ncell, int ld, int nstep,
                       long long fs, const DevParams<R>& P, int* status, cudaStream_t s) {
    constexpr LaunchConfig C = kConfigs[CFG];
    if constexpr (C.form == 0) {
        // the default fused configuration (the plain entry points' and the
        // per-hour callers') also has a global-accumulator twin for short launches
        if constexpr (CFG == kDefaultFused && AccInSmem<R, C.block, C.minb>::value) {
            if (nstep < kAccSmemMinSteps)
                return launch_fused<R, NT, SU, SL, C.block, C.minb, false, X3>(prog, stat, forc, diag, acc, ncell,
                                                                               ld, nstep, fs, P, status, s);
        }
        return launch_fused<R, NT, SU, SL, C.block, C.minb, true, X3>(prog, stat, forc, diag, acc, ncell, ld, nstep,
                                                                      fs, P, status, s);
    } else if constexpr (C.form == 2) {
        return launch_staged<R, NT, SU, SL, C.block, C.minb, X3>(prog, stat, forc, diag, acc, ncell, ld, nstep, fs, P,
                                                                 status, s);
    } else {
        return launch_split<R, NT, SU, SL, C.block, C.minb, C.block2, C.minb2, X3>(prog, stat, forc, diag, acc, mid,
                                                                                  ncell, ld, nstep, fs, P, status, s);
    }
}

#define IBIS_RUN_ARGS(R) \
    R*, const R*, const R*, R*, R*, R*, int, int, int, long long, const DevParams<R>&, int*, cudaStream_t

// Every (variant, configuration) pair the FP32 library instantiates: the F77
// canopy (no sunlit/shaded split) in every configuration, the sunlit/shaded
// variants in the two default ones.  X(NT, SU, SL, CFG).
#define IBIS_F77_CONFIGS(X, NT)                                                                                \
    X(NT, false, false, 0) X(NT, false, false, 1) X(NT, false, false, 2) X(NT, false, false, 3)                \
    X(NT, false, false, 4) X(NT, false, false, 5) X(NT, false, false, 6) X(NT, false, false, 7)                \
    X(NT, false, false, 8) X(NT, false, false, 9) X(NT, false, false, 10) X(NT, false, false, 11)
#define IBIS_SUN_CONFIGS(X, NT)                                                                                \
    X(NT, true, false, 0) X(NT, false, true, 0) X(NT, true, true, 0)                                           \
    X(NT, true, false, 8) X(NT, false, true, 8) X(NT, true, true, 8)
// The IBIS 3.0 kernels (X3): every canopy variant in the two default
// configurations, and the long fused configuration for both canopies F77 or
// both sunlit/shaded.  X(NT, SU, SL, CFG).
#define IBIS_X3_CONFIGS(X, NT)                                                                                 \
    X(NT, false, false, 0) X(NT, false, false, 6) X(NT, false, false, 8)                                       \
    X(NT, true, true, 0) X(NT, true, true, 6) X(NT, true, true, 8)                                             \
    X(NT, true, false, 0) X(NT, true, false, 8) X(NT, false, true, 0) X(NT, false, true, 8)

template <typename R, int NT, bool SU, bool SL, bool X3>
cudaError_t dispatch_config(int cfg, R* prog, const R* stat, const R* forc, R* diag, R* acc, R* mid, int ncell,
                            int ld, int nstep, long long fs, const DevParams<R>& P, int* status, cudaStream_t s) {
#define IBIS_ARGS prog, stat, forc, diag, acc, mid, ncell, ld, nstep, fs, P, status, s
    if constexpr (sizeof(R) == 8) {
        // the float64 kernels always carry the IBIS 3.0 extensions: with their
        // switches off they perform the F77 step's operations
        return run_config<R, NT, SU, SL, kDefaultFused, true>(IBIS_ARGS);
    } else if constexpr (X3) {
        if (cfg == kLongFused && SU == SL) return run_config<R, NT, SU, SL, kLongFused, true>(IBIS_ARGS);
        if (kConfigs[cfg].form != 1) return run_config<R, NT, SU, SL, kDefaultFused, true>(IBIS_ARGS);
        return run_config<R, NT, SU, SL, kDefaultSplit, true>(IBIS_ARGS);
    } else if constexpr (SU || SL) {
        if (kConfigs[cfg].form != 1) return run_config<R, NT, SU, SL, kDefaultFused>(IBIS_ARGS);
        return run_config<R, NT, SU, SL, kDefaultSplit>(IBIS_ARGS);
    } else {
        switch (cfg) {
            case 1: return run_config<R, NT, SU, SL, 1>(IBIS_ARGS);
            case 2: return run_config<R, NT, SU, SL, 2>(IBIS_ARGS);
            case 3: return run_config<R, NT, SU, SL, 3>(IBIS_ARGS);
            case 4: return run_config<R, NT, SU, SL, 4>(IBIS_ARGS);
            case 5: return run_config<R, NT, SU, SL, 5>(IBIS_ARGS);
            case 6: return run_config<R, NT, SU, SL, 6>(IBIS_ARGS);
            case 7: return run_config<R, NT, SU, SL, 7>(IBIS_ARGS);
            case 8: return run_config<R, NT, SU, SL, 8>(IBIS_ARGS);
            case 9: return run_config<R, NT, SU, SL, 9>(IBIS_ARGS);
            case 10: return run_config<R, NT, SU, SL, 10>(IBIS_ARGS);
            case 11: return run_config<R, NT, SU, SL, 11>(IBIS_ARGS);
            default: return run_config<R, NT, SU, SL, 0>(IBIS_ARGS);
        }
    }
#undef IBIS_ARGS
}

template <typename R>
static int hourly_step(R* prog, const R* stat, const R* forc, R* diag, R* acc, int ncell, int ld, int nstep,
                       const IbisParams* hp, int* status, void* stream, R* mid, int cfg, int cell0 = 0) {
    if (!prog || !stat || !forc || !hp) return -EINVAL;
    if (cfg < 0 || cfg >= kNumConfigs) return -EINVAL;
    if (kConfigs[cfg].form == 1 && (!mid || sizeof(R) != 4)) return -EINVAL;
    if (ncell < 0 || nstep < 0 || ld < ncell || (ld % 32) != 0) return -EINVAL;
    if (ncell == 0 || nstep == 0) return 0;
    const unsigned known = IBIS_FLAG_BEDROCK | IBIS_FLAG_H2O_CONSISTENT | IBIS_FLAG_SUNSHADE_U | IBIS_FLAG_SUNSHADE_L |
                           IBIS_FLAG_ACC | IBIS_FLAG_CH4 | IBIS_FLAG_SOIL_MEANS | IBIS_FLAG_DIAG | IBIS_FLAG_KAHAN |
                           IBIS_FLAG_ZWT_OBS | IBIS_FLAG_ETPARTS | IBIS_FLAG_NEEPARTS | IBIS_FLAGS_X3 |
                           IBIS_FLAG_CH4_BANDS;
    if (hp->flags & ~known) return -EINVAL;
    if ((hp->flags & (IBIS_FLAG_ACC | IBIS_FLAG_CH4 | IBIS_FLAG_SOIL_MEANS)) && !acc) return -EINVAL;
    if ((hp->flags & IBIS_FLAG_DIAG) && !diag) return -EINVAL;
    if (!(hp->dtime > 0.0)) return -EINVAL;
    DevParams<R> P = make_dev_params<R>(*hp);
    P.cell0 = cell0;
    if (!(hp->flags & IBIS_FLAG_DIAG)) diag = nullptr;
    if (!(hp->flags & (IBIS_FLAG_ACC | IBIS_FLAG_CH4 | IBIS_FLAG_SOIL_MEANS))) acc = nullptr;
    const long long fstride = (long long)IBIS_FORC_COUNT * ld;
    cudaStream_t s = (cudaStream_t)stream;
    const bool bed = hp->flags & IBIS_FLAG_BEDROCK;
    const bool su = hp->flags & IBIS_FLAG_SUNSHADE_U;
    const bool sl = hp->flags & IBIS_FLAG_SUNSHADE_L;
    const bool x3 = (hp->flags & IBIS_FLAGS_X3) != 0;
    cudaError_t e;
#define IBIS_CASE(NT_, SU_, SL_)                                                                                     \
    e = x3 ? dispatch_config<R, NT_, SU_, SL_, true>(cfg, prog, stat, forc, diag, acc, mid, ncell, ld, nstep, fstride, \
                                                     P, status, s)                                                   \
           : dispatch_config<R, NT_, SU_, SL_, false>(cfg, prog, stat, forc, diag, acc, mid, ncell, ld, nstep,       \
                                                      fstride, P, status, s)
    if (bed) {
        if (su) { if (sl) IBIS_CASE(9, true, true); else IBIS_CASE(9, true, false); }
        else { if (sl) IBIS_CASE(9, false, true); else IBIS_CASE(9, false, false); }
    } else {
        if (su) { if (sl) IBIS_CASE(6, true, true); else IBIS_CASE(6, true, false); }
        else { if (sl) IBIS_CASE(6, false, true); else IBIS_CASE(6, false, false); }
    }
#undef IBIS_CASE
    if (e != cudaSuccess) {
        fprintf(stderr, "ibis_b200: kernel launch failed: %s\n", cudaGetErrorString(e));
        return -(int)e - 1000;
    }
    return 0;
}

}  // namespace ibis
