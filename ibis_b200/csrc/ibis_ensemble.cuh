// Calibration ensembles: many runs (site x parameter vector), each a record of
// hourly steps of its own length, in one persistent launch or in one launch per
// hour.
//
// The reference evaluates calibration candidates one site run at a time, in a
// pool of host worker processes (verify/calibration/site_fit.py:375-436), each
// run a scan of the day loop (loops_gswp3.py:115-331) with the candidate's
// parameters applied to SimParams (verify/calibration/fit_carbon.py:438).  Here
// every run is one thread: its prognostic state and calibrated parameters stay
// on chip for the whole record, the site's static inputs and forcing records
// are shared by all runs at that site, and warps draw 32-run work items from a
// device counter in the caller's order (longest records first).
#pragma once
#include "ibis_diurnal.cuh"
#include <type_traits>

#include "ibis_kernels.cuh"

namespace ibis {

// Device view of an IbisEnsemble (include/ibis_b200.h).
struct EnsArgs {
    float* prog;
    float* acc;
    const float* stat;
    const float* forc;
    const float* run_params;
    const int* run_site;
    const long long* run_forc;
    const int* run_nstep;
    const int* run_pos;
    const int* order;
    float* yearly;
    long long forc_len;
    int nrun, ld_run, nsite, ld_site, nyear, year_steps;
    int nwork;   // entries of order to run (nrun when order is NULL)
    int* queue;
    int* status;
    // daily-weather form (IbisEnsembleDaily): run_forc indexes day records
    const float* daily;     // [daily_len][kEnsDailyWords]; nullptr: hourly records in forc
    const float* site_lat;  // [nsite] degrees
    long long daily_len;
    uint32_t seed;
    bool obs_fira;
    int nh;                 // steps per day
    float dtime;
};

// A day record of the daily-weather form: the IBIS_DAILY_* words, the day of
// year, two words of padding (48 bytes, three 16-byte loads).
constexpr int kEnsDailyWords = 12;
constexpr int kEnsDailyJday = IBIS_DAILY_COUNT;

// A run whose descriptor points outside the buffers is flagged (status bit 1)
// and skipped, so no access leaves the caller's arrays.
__device__ __forceinline__ bool run_ok(const EnsArgs& e, int r, int site, int nstep, long long first, int pos) {
    const long long len = e.daily ? e.daily_len : e.forc_len;
    const long long need = e.daily ? ((long long)nstep + e.nh - 1) / e.nh : (long long)nstep;
    const bool ok = r >= 0 && r < e.nrun && site >= 0 && site < e.nsite && nstep >= 0 && first >= 0 &&
                    first + need <= len && pos >= 0;
    if (!ok && e.status) atomicOr(e.status, 2);
    return ok;
}

// Accumulator plane of IBIS_YEARLY entry k (the order of include/ibis_layout.h).
__host__ __device__ constexpr int yearly_plane(int k) {
    return k == IBIS_YEARLY_AYGPPTOT   ? IBIS_ACC_AYGPPTOT
           : k == IBIS_YEARLY_AYNPPTOT ? IBIS_ACC_AYNPPTOT
           : k == IBIS_YEARLY_ADAET    ? IBIS_ACC_ADAET
           : k == IBIS_YEARLY_AFSENA   ? IBIS_ACC_AFSENA
           : k == IBIS_YEARLY_AYTRUNOF ? IBIS_ACC_AYTRUNOF
           : k == IBIS_YEARLY_AYTDRAIN ? IBIS_ACC_AYTDRAIN
                                       : IBIS_ACC_CH4;
}

// One hour of a site's forcing record: IBIS_FORC_COUNT words (48 bytes, three
// 16-byte loads; every run at the site reads the same address).
__device__ __forceinline__ Forc<float> load_forc_record(const float* __restrict__ f) {
    const float4* p = reinterpret_cast<const float4*>(f);
    const float4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2);
    const float v[IBIS_FORC_COUNT] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, c.x, c.y, c.z, c.w};
    Forc<float> F;
    F.ta = v[IBIS_FORC_TA]; F.qa = v[IBIS_FORC_QA]; F.ua = v[IBIS_FORC_UA]; F.ps = v[IBIS_FORC_PSURF];
    F.cosz = v[IBIS_FORC_COSZEN];
    F.sd[0] = v[IBIS_FORC_SOLAD]; F.sd[1] = v[IBIS_FORC_SOLAD + 1];
    F.si[0] = v[IBIS_FORC_SOLAI]; F.si[1] = v[IBIS_FORC_SOLAI + 1];
    F.fira = v[IBIS_FORC_FIRA]; F.rain = v[IBIS_FORC_RAINA]; F.snow = v[IBIS_FORC_SNOWA];
    return F;
}

// What a run of the daily-weather form keeps of its current day (in shared
// memory): the day's weather, orbital terms and precipitation event, and the
// site's latitude terms.
struct DayCache {
    DailyRec rec;
    DayGeom g;
    Event ev;
    float sinlat, coslat;
};

// Day record `rec` of `site`: its weather and orbital terms, and the event the
// counter-based variates (seed, record, site) place (ibis_diurnal.cuh).
__device__ __forceinline__ void load_day(DayCache& dc, const EnsArgs& e, int site, long long rec) {
    const float4* p = reinterpret_cast<const float4*>(e.daily + (size_t)rec * kEnsDailyWords);
    const float4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2);
    const float v[kEnsDailyWords] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, c.x, c.y, c.z, c.w};
    dc.rec.tmax = v[IBIS_DAILY_TMAX]; dc.rec.tmin = v[IBIS_DAILY_TMIN]; dc.rec.cloud = v[IBIS_DAILY_CLOUD];
    dc.rec.precip = v[IBIS_DAILY_PRECIP]; dc.rec.psurf = v[IBIS_DAILY_PSURF]; dc.rec.qd = v[IBIS_DAILY_QD];
    dc.rec.ud = v[IBIS_DAILY_UD]; dc.rec.fira = v[IBIS_DAILY_FIRA];
    dc.g = day_geometry((int)v[kEnsDailyJday]);
    const uint32_t day = (uint32_t)rec;
    dc.ev = precip_timing(draw24(e.seed, site, day, 0), draw24(e.seed, site, day, 1), dc.rec.precip, e.dtime);
}

// Fill one run's parameter source from its vector (planes [IBIS_RUN_PARAMS][ld]).
// Derived values are formed exactly as the host forms them for a uniform
// parameter record (make_dev_params), so a run here and the same column run
// with that vector as its IbisParams give the same bits.
__device__ __forceinline__ void load_run_params(RunQ<float>& q, const float* __restrict__ v, int ld,
                                                const DevParams<float>& P) {
    auto g = [&](int k) { return __ldg(v + (size_t)k * ld); };
#pragma unroll
    for (int j = 0; j < 12; ++j) q.vmax_[j] = g(IBIS_RUN_VMAX + j);
#pragma unroll
    for (int j = 0; j < 5; ++j) q.coefm_[j] = g(IBIS_RUN_COEFM + j);
    q.stressfac_ = g(IBIS_RUN_STRESSFAC);
    q.znorm_ = (float)(1.0 - exp((double)q.stressfac_));
    q.beta_ = g(IBIS_RUN_SOIL_BETA_POWER);
    q.wliqumax_ = g(IBIS_RUN_WLIQUMAX);
    q.wliqsmax_ = g(IBIS_RUN_WLIQSMAX);
    q.wliqlmax_ = g(IBIS_RUN_WLIQLMAX);
    q.fmax_ = g(IBIS_RUN_FMAX);
    q.wliqmin_ = (float)(0.001 * ((double)P.dtime / 3600.0) * ((double)q.wliqumax_ / 0.2));
    q.r_ch4_ = g(IBIS_RUN_R_CH4);
    q.q10p_ = g(IBIS_RUN_Q10P);
    q.z_tau_ = g(IBIS_RUN_Z_TAU);
    q.tau_oxid_ = g(IBIS_RUN_TAU_OXID);
    q.z_wt_max_ = g(IBIS_RUN_Z_WT_MAX);
    const float per_s = (float)((double)P.ndaypy * 86400.0), mol = (float)(1000.0 / 12.0);
    q.rwood_ = __fmul_rn(__fdiv_rn(g(IBIS_RUN_RWOOD), per_s), mol);
    q.rroot_ = __fmul_rn(__fdiv_rn(g(IBIS_RUN_RROOT), per_s), mol);
    q.keep_ = __fsub_rn(1.0f, g(IBIS_RUN_RGROWTH));
}

__device__ __forceinline__ void yearly_snapshot(const EnsArgs& e, const Acc<float>& A, int r, int y) {
#pragma unroll
    for (int k = 0; k < IBIS_YEARLY_COUNT; ++k) {
        const float* v = A.base + (size_t)yearly_plane(k) * A.ld;
        float t = *v;
        if (A.kahan) t = t - v[(size_t)IBIS_ACC_COUNT * A.ld];
        e.yearly[((size_t)y * IBIS_YEARLY_COUNT + k) * e.ld_run + r] = t;
    }
}

__device__ __forceinline__ void flag_nonfinite(const EnsArgs& e, float sum, int r) {
    if (e.status && !isfinite(sum)) {
        atomicOr(e.status, 1);
        atomicMin(e.status + 1, r);
    }
}

// Persistent form: grid = SMs x resident blocks; each warp takes work items of
// 32 consecutive entries of `order` from the device counter e.queue until the
// items run out, and runs each of its runs from its first hour to its last.
// blockDim.x is a multiple of 32 (checked by the host), so every warp is whole
// for the __shfl_sync that shares the item number.
// With DAILY, each run's hours are generated from its site's day records as it
// steps (the day's terms once a day, then one diurnal hour per step), so the
// forcing read from memory is one 48-byte record per site-day instead of one
// per site-hour; a run's hours start at midnight of record run_forc.
// With X3 the runs step with the IBIS 3.0 extensions (IBIS_FLAGS_X3).
template <bool X3>
using RunSource = std::conditional_t<X3, RunQ3<float>, RunQ<float>>;

template <int NT, bool SU, bool SL, bool DAILY, bool X3>
__global__ void __launch_bounds__(256, 1) ensemble_kernel(const EnsArgs e, const DevParams<float> P) {
    extern __shared__ unsigned char smem_raw[];
    Col<float>& c = reinterpret_cast<Col<float>*>(smem_raw)[threadIdx.x];
    RunSource<X3>& q =
        reinterpret_cast<RunSource<X3>*>(smem_raw + blockDim.x * sizeof(Col<float>))[threadIdx.x];
    DayCache* const dc =
        DAILY ? reinterpret_cast<DayCache*>(smem_raw + blockDim.x * (sizeof(Col<float>) + sizeof(RunQ<float>))) +
                    threadIdx.x
              : nullptr;
    const int lane = threadIdx.x & 31;
    const int nitem = (e.nwork + 31) >> 5;
    const bool kahan = (P.flags & IBIS_FLAG_KAHAN) != 0;
    const Diag<float> D{nullptr, 0};
    for (;;) {
        int item = 0;
        if (lane == 0) item = atomicAdd(e.queue, 1);
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= nitem) break;
        const int idx = item * 32 + lane;
        const int r = idx < e.nwork ? (e.order ? __ldg(e.order + idx) : idx) : -1;
        const bool in = r >= 0 && r < e.nrun;
        const int site = in ? __ldg(e.run_site + r) : -1;
        const int nstep = in ? __ldg(e.run_nstep + r) : 0;
        const long long first = in ? __ldg(e.run_forc + r) : -1;
        const int pos = in && e.run_pos ? __ldg(e.run_pos + r) : 0;
        if (idx < e.nwork && run_ok(e, r, site, nstep, first, pos)) {
            const float* f = DAILY ? nullptr : e.forc + (size_t)first * IBIS_FORC_COUNT;
            if constexpr (DAILY) {
                const double xlat = (double)__ldg(e.site_lat + site) * (3.14159265358979323846 / 180.0);
                dc->sinlat = (float)sin(xlat);
                dc->coslat = (float)cos(xlat);
            }
            load_col(c, e.prog + r, e.ld_run);
            load_run_params(q, e.run_params + r, e.ld_run, P);
            const Stat<float> S{e.stat + site, e.ld_site};
            Acc<float> A{e.acc ? e.acc + r : nullptr, e.ld_run, kahan};
            // steps of this call until the run's next year end, and that year's index
            int next_year = e.year_steps - pos % e.year_steps;
            int year = pos / e.year_steps;
#pragma unroll 1
            for (int s = 0; s < nstep; ++s) {
                Forc<float> F;
                if constexpr (DAILY) {
                    const int d = s / e.nh, h = s - d * e.nh;
                    if (h == 0) load_day(*dc, e, site, first + d);
                    F = diurnal_hour(dc->rec, dc->g, dc->sinlat, dc->coslat, (float)h * e.dtime, dc->ev,
                                     draw24(e.seed, site, (uint32_t)(first + d), 2 + h), e.dtime, e.obs_fira);
                } else {
                    F = load_forc_record(f + (size_t)s * IBIS_FORC_COUNT);
                }
                A.last = (s + 1 == nstep);
                column_step<float, NT, SU, SL>(c, F, S, D, A, P, q);
                if (s + 1 == next_year) {
                    if (e.yearly && year < e.nyear) yearly_snapshot(e, A, r, year);
                    ++year;
                    next_year += e.year_steps;
                }
            }
            flag_nonfinite(e, store_col(c, e.prog + r, e.ld_run), r);
        }
        __syncwarp();
    }
}

// Plain form: one launch per hour over all runs; run r takes its step when the
// hour (*hour0 + k) is inside its record.  The hour is read from device memory
// so a captured sequence of launches can be replayed (advance_hour moves it).
template <int NT, bool SU, bool SL, bool X3>
__global__ void __launch_bounds__(128, 2) ensemble_hour_kernel(const EnsArgs e, const DevParams<float> P,
                                                               const int* __restrict__ hour0, int k) {
    // hour0 is written only by advance_hour, a later launch on the same stream
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= e.nrun) return;
    const int hour = *hour0 + k;
    const int nstep = __ldg(e.run_nstep + r);
    if (hour >= nstep) return;
    const int site = __ldg(e.run_site + r);
    const long long first = __ldg(e.run_forc + r);
    const int pos = e.run_pos ? __ldg(e.run_pos + r) : 0;
    if (!run_ok(e, r, site, nstep, first, pos)) return;
    extern __shared__ unsigned char smem_raw[];
    Col<float>& c = reinterpret_cast<Col<float>*>(smem_raw)[threadIdx.x];
    RunSource<X3>& q =
        reinterpret_cast<RunSource<X3>*>(smem_raw + blockDim.x * sizeof(Col<float>))[threadIdx.x];
    load_col(c, e.prog + r, e.ld_run);
    load_run_params(q, e.run_params + r, e.ld_run, P);
    const Stat<float> S{e.stat + site, e.ld_site};
    const Acc<float> A{e.acc ? e.acc + r : nullptr, e.ld_run, (P.flags & IBIS_FLAG_KAHAN) != 0, hour + 1 == nstep};
    const Forc<float> F = load_forc_record(e.forc + (size_t)(first + hour) * IBIS_FORC_COUNT);
    column_step<float, NT, SU, SL>(c, F, S, Diag<float>{nullptr, 0}, A, P, q);
    if (e.yearly && (pos + hour + 1) % e.year_steps == 0) {
        const int y = (pos + hour + 1) / e.year_steps - 1;
        if (y < e.nyear) yearly_snapshot(e, A, r, y);
    }
    flag_nonfinite(e, store_col(c, e.prog + r, e.ld_run), r);
}

static __global__ void advance_hour(int* hour0, int n) { *hour0 += n; }

constexpr int kEnsHourBlock = 128;

inline size_t ens_smem(int block, bool daily = false) {
    return (size_t)block * (sizeof(Col<float>) + sizeof(RunQ<float>) + (daily ? sizeof(DayCache) : 0));
}

template <int NT, bool SU, bool SL, bool DAILY = false, bool X3 = false>
cudaError_t launch_ensemble(const EnsArgs& e, const DevParams<float>& P, int block, int grid, cudaStream_t s) {
    auto k = ensemble_kernel<NT, SU, SL, DAILY, X3>;
    const size_t smem = ens_smem(block, DAILY);
    cudaError_t err = fit_smem(k, block, smem, ens_smem(256, DAILY));
    if (err != cudaSuccess) return err;
    k<<<grid, block, smem, s>>>(e, P);
    return cudaGetLastError();
}

template <int NT, bool SU, bool SL, bool X3 = false>
cudaError_t launch_ensemble_hours(const EnsArgs& e, const DevParams<float>& P, int* hour0, int nhour,
                                  cudaStream_t s) {
    auto k = ensemble_hour_kernel<NT, SU, SL, X3>;
    const size_t smem = ens_smem(kEnsHourBlock);
    static unsigned long long fitted = 0;
    cudaError_t err = fit_smem_once(fitted, k, kEnsHourBlock, smem, smem);
    if (err != cudaSuccess) return err;
    const int grid = (e.nrun + kEnsHourBlock - 1) / kEnsHourBlock;
    for (int h = 0; h < nhour; ++h) k<<<grid, kEnsHourBlock, smem, s>>>(e, P, hour0, h);
    advance_hour<<<1, 1, 0, s>>>(hour0, nhour);
    return cudaGetLastError();
}

// Resident blocks of `block` threads per SM for the persistent kernel.
template <int NT, bool SU, bool SL, bool DAILY = false, bool X3 = false>
int ensemble_occupancy(int block) {
    int n = 0;
    auto k = ensemble_kernel<NT, SU, SL, DAILY, X3>;
    if (fit_smem(k, block, ens_smem(block, DAILY), ens_smem(256, DAILY)) != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, block, ens_smem(block, DAILY)) != cudaSuccess) return 0;
    return n;
}

#define IBIS_ENS_VARIANTS(X, NT) X(NT, false, false) X(NT, true, false) X(NT, false, true) X(NT, true, true)

}  // namespace ibis
