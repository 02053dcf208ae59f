// Wetland (inundated) area of the monthly methane: the dynamic area, the
// learned wetland's monthly feature builder and its tree-ensemble fraction.
// Monthly work of a few hundred thousand values: plain kernels, float64
// arithmetic in the reference's operation order (built without FMA contraction).
#include <errno.h>
#include <math.h>
#include <stdio.h>

#include "../../include/ibis_b200.h"

namespace {

constexpr int kRootLayers = 4;          // wetland_area.py:18, wetland_learned.py:36
constexpr int kBox = 5;                 // wetland_learned.py:37 (5 x 5 neighbourhood)
constexpr double kTFreeze = 273.16;     // wetland_area.py:19
constexpr int kNStat = 12;              // STAT_FEATS (wetland_learned.py:30)

int launched(const char* what) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        fprintf(stderr, "%s: launch failed: %s\n", what, cudaGetErrorString(e));
        return -(int)e - 1000;
    }
    return 0;
}

__device__ __forceinline__ double clip(double x, double lo, double hi) { return fmin(fmax(x, lo), hi); }

// ---------------------------------------------------------------------------
// dynamic wetland area (wetland_area.py:22-39)
// ---------------------------------------------------------------------------
__global__ void dynamic_kernel(const float* __restrict__ prog, const float* __restrict__ stat,
                               const double* __restrict__ area, float* __restrict__ f_out, int ncell, int ld,
                               double h0, double h1, double h2, double h3) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ncell) return;
    const double h[kRootLayers] = {h0, h1, h2, h3};
    double W = 0.0;
#pragma unroll
    for (int k = 0; k < kRootLayers; ++k) {
        const double w = (double)prog[(size_t)(IBIS_PROG_WSOI + k) * ld + i] *
                         (double)stat[(size_t)(IBIS_STAT_POROS + k) * ld + i] * h[k];
        const double t = (double)prog[(size_t)(IBIS_PROG_TSOI + k) * ld + i];
        W = W + (t > kTFreeze ? w : 0.0);
    }
    const double fclim = area[i], mu = area[(size_t)ld + i], sd = area[(size_t)2 * ld + i];
    const double beta = area[(size_t)3 * ld + i], fmin_ = area[(size_t)4 * ld + i], fmax_ = area[(size_t)5 * ld + i];
    double A = sd > 1e-9 ? (W - mu) / fmax(sd, 1e-9) : 0.0;
    if ((double)prog[(size_t)IBIS_PROG_TSOI * ld + i] <= kTFreeze) A = 0.0;
    const double f = fmin(fmax(fclim * (1.0 + beta * A), fmin_), fmax_);
    f_out[i] = (float)clip(f, 0.0, 1.0);
}

// ---------------------------------------------------------------------------
// the learned wetland's feature builder (wetland_learned.py:40-104)
// ---------------------------------------------------------------------------
// Buffer of `keep` months in planes [p0, p0 + keep) of b, oldest first, `len`
// of them filled before this month: append v (dropping the oldest when full)
// and return the new length.
__device__ __forceinline__ int push(double* __restrict__ b, int p0, int keep, int len, int i, int ld, double v) {
    if (len == keep) {
        for (int k = 0; k + 1 < keep; ++k) b[(size_t)(p0 + k) * ld + i] = b[(size_t)(p0 + k + 1) * ld + i];
        b[(size_t)(p0 + keep - 1) * ld + i] = v;
        return keep;
    }
    b[(size_t)(p0 + len) * ld + i] = v;
    return len + 1;
}

__device__ __forceinline__ double at(const double* __restrict__ b, int p0, int k, int i, int ld) {
    return b[(size_t)(p0 + k) * ld + i];
}

// np.mean(lst[-3:], axis=0): the last min(3, len) entries summed oldest first, over their count
__device__ __forceinline__ double mean3(const double* __restrict__ b, int p0, int len, int i, int ld) {
    const int n = len < 3 ? len : 3;
    double s = at(b, p0, len - n, i, ld);
    for (int k = len - n + 1; k < len; ++k) s = s + at(b, p0, k, i, ld);
    return s / (double)n;
}

// lst[-1 - L] if len(lst) > L else lst[-1]
__device__ __forceinline__ double lag(const double* __restrict__ b, int p0, int len, int L, int i, int ld) {
    return at(b, p0, len > L ? len - 1 - L : len - 1, i, ld);
}

// entries a buffer of `keep` months holds after `nmonth` months
__host__ __device__ constexpr int held(int nmonth, int keep) { return nmonth < keep ? nmonth : keep; }

enum Feat {
    F_W, F_WICE, F_WS1, F_WI1 = F_WS1 + 6, F_WI2, F_T1, F_T14, F_TG, F_FRZ1, F_PRCP, F_AET, F_RUNOFF, F_W_L1,
    F_W_L2, F_W_L3, F_W_3MO, F_P3, F_P3_L1, F_P3_L3, F_R3, F_R3_L1, F_R3_L3, F_NP3, F_NP3_L1, F_NP3_L2, F_NR3,
    F_NR3_L1, F_NR3_L2, F_COUNT
};
static_assert(F_COUNT == IBIS_WETLAND_NFEAT, "the model's 33 monthly predictors");

// The month's own predictors; pushes W, precipitation and runoff, their
// 3-month means, and puts the means of precipitation and runoff on the grids.
__global__ void features_kernel(IbisWetlandBuilder b, const float* __restrict__ means,
                                const float* __restrict__ totals, double* __restrict__ feats,
                                double* __restrict__ gp, double* __restrict__ gr) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= b.npoi) return;
    const int ld = b.ld;
    auto mean = [&](int q) { return (double)means[(size_t)q * ld + i]; };
    auto put = [&](int f, double v) { feats[(size_t)f * ld + i] = v; };
    double W = 0.0, Wice = 0.0, t14 = 0.0, hsum = 0.0;
#pragma unroll
    for (int k = 0; k < kRootLayers; ++k) {
        const double p = b.poros[(size_t)k * ld + i];
        const double wk = mean(6 + k) * p * b.hsoi[k];
        const double ik = mean(12 + k) * p * b.hsoi[k];
        W = k ? W + wk : wk;
        Wice = k ? Wice + ik : ik;
        const double tk = mean(k) * b.hsoi[k];
        t14 = k ? t14 + tk : tk;
        hsum = k ? hsum + b.hsoi[k] : b.hsoi[k];
    }
    put(F_W, W);
    put(F_WICE, Wice);
    for (int l = 0; l < 6; ++l) put(F_WS1 + l, mean(6 + l));
    const double wi1 = mean(12), ws1 = mean(6);
    put(F_WI1, wi1);
    put(F_WI2, mean(13));
    put(F_T1, mean(0));
    put(F_T14, t14 / hsum);
    put(F_TG, mean(18));
    put(F_FRZ1, wi1 / fmax(ws1 + wi1, 1e-6));
    const double prcp = (double)totals[i], aet = (double)totals[(size_t)ld + i];
    const double runoff = (double)totals[(size_t)2 * ld + i];
    put(F_PRCP, prcp);
    put(F_AET, aet);
    put(F_RUNOFF, runoff);
    double* buf = b.buf;
    const int m = b.nmonth;
    const int lw = push(buf, IBIS_WFB_W, 4, held(m, 4), i, ld, W);
    const int lp = push(buf, IBIS_WFB_PRCP, 3, held(m, 3), i, ld, prcp);
    const int lr = push(buf, IBIS_WFB_RUNOFF, 3, held(m, 3), i, ld, runoff);
    const double w3 = mean3(buf, IBIS_WFB_W, lw, i, ld);
    const double p3 = mean3(buf, IBIS_WFB_PRCP, lp, i, ld);
    const double r3 = mean3(buf, IBIS_WFB_RUNOFF, lr, i, ld);
    const int l3 = push(buf, IBIS_WFB_W3, 4, held(m, 4), i, ld, w3);
    push(buf, IBIS_WFB_P3, 4, held(m, 4), i, ld, p3);
    push(buf, IBIS_WFB_R3, 4, held(m, 4), i, ld, r3);
    put(F_W_L1, lag(buf, IBIS_WFB_W, lw, 1, i, ld));
    put(F_W_L2, lag(buf, IBIS_WFB_W, lw, 2, i, ld));
    put(F_W_L3, lag(buf, IBIS_WFB_W, lw, 3, i, ld));
    put(F_W_3MO, at(buf, IBIS_WFB_W3, l3 - 1, i, ld));
    put(F_P3, p3);
    put(F_P3_L1, lag(buf, IBIS_WFB_P3, l3, 1, i, ld));
    put(F_P3_L3, lag(buf, IBIS_WFB_P3, l3, 3, i, ld));
    put(F_R3, r3);
    put(F_R3_L1, lag(buf, IBIS_WFB_R3, l3, 1, i, ld));
    put(F_R3_L3, lag(buf, IBIS_WFB_R3, l3, 3, i, ld));
    const size_t g = (size_t)b.cell_i[i] * b.nlon + b.cell_j[i];
    gp[g] = p3;
    gr[g] = r3;
}

// One pass of the box filter over lines of length n (stride `step` between a
// line's values, `line_step` between lines), periodic at both ends: the first
// window summed in order, then moved by += entering - leaving; each output the
// running sum over the width.  One thread per line; `nline` lines per grid,
// the grids `grid_step` apart.
__global__ void box_kernel(const double* __restrict__ in, double* __restrict__ out, int n, int nline,
                           long long step, long long line_step, int ngrid, long long grid_step) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nline * ngrid) return;
    const int gi = t / nline, line = t - gi * nline;
    const double* x = in + gi * grid_step + line * line_step;
    double* y = out + gi * grid_step + line * line_step;
    constexpr int s1 = kBox / 2;
    auto ext = [&](int k) {                    // extended line: index k - s1, wrapped
        int q = (k - s1) % n;
        if (q < 0) q += n;
        return x[q * step];
    };
    double tmp = ext(0);
    for (int k = 1; k < kBox; ++k) tmp = tmp + ext(k);
    y[0] = tmp / (double)kBox;
    for (int l = 1; l < n; ++l) {
        tmp = tmp + (ext(l + kBox - 1) - ext(l - 1));
        y[l * step] = tmp / (double)kBox;
    }
}

// The neighbourhood means of this month and the lag predictors that need them.
__global__ void neighbour_kernel(IbisWetlandBuilder b, const double* __restrict__ fp,
                                 const double* __restrict__ fr, double* __restrict__ feats) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= b.npoi) return;
    const int ld = b.ld;
    const size_t g = (size_t)b.cell_i[i] * b.nlon + b.cell_j[i];
    const double lf = fmax(b.lf[g], 1e-6);
    const int m = b.nmonth;
    const int len = held(m, 3);
    const int ln = push(b.buf, IBIS_WFB_NP3, 3, len, i, ld, fp[g] / lf);
    push(b.buf, IBIS_WFB_NR3, 3, len, i, ld, fr[g] / lf);
    auto put = [&](int f, double v) { feats[(size_t)f * ld + i] = v; };
    put(F_NP3, at(b.buf, IBIS_WFB_NP3, ln - 1, i, ld));
    put(F_NP3_L1, lag(b.buf, IBIS_WFB_NP3, ln, 1, i, ld));
    put(F_NP3_L2, lag(b.buf, IBIS_WFB_NP3, ln, 2, i, ld));
    put(F_NR3, at(b.buf, IBIS_WFB_NR3, ln - 1, i, ld));
    put(F_NR3_L1, lag(b.buf, IBIS_WFB_NR3, ln, 1, i, ld));
    put(F_NR3_L2, lag(b.buf, IBIS_WFB_NR3, ln, 2, i, ld));
}

__global__ void mask_kernel(IbisWetlandBuilder b, double* __restrict__ grid) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= b.npoi) return;
    grid[(size_t)b.cell_i[i] * b.nlon + b.cell_j[i]] = 1.0;
}

// 2-D box filter of `ngrid` grids in place: rows' axis (columns as lines), then
// the columns' axis (rows as lines), through `tmp` (ngrid grids).
int box_filter(double* grids, double* tmp, int ngrid, int nlat, int nlon, cudaStream_t s) {
    const long long gs = (long long)nlat * nlon;
    const int block = 128;
    int lines = nlon * ngrid;
    box_kernel<<<(lines + block - 1) / block, block, 0, s>>>(grids, tmp, nlat, nlon, nlon, 1, ngrid, gs);
    lines = nlat * ngrid;
    box_kernel<<<(lines + block - 1) / block, block, 0, s>>>(tmp, grids, nlon, nlat, 1, nlon, ngrid, gs);
    return launched("ibis_wetland box filter");
}

bool builder_ok(const IbisWetlandBuilder* b) {
    return b && b->npoi >= 0 && b->ld >= b->npoi && b->ld % 32 == 0 && b->nlat > 0 && b->nlon > 0 &&
           b->cell_i && b->cell_j && b->lf && b->work && b->nmonth >= 0;
}

// ---------------------------------------------------------------------------
// learned fraction (wetland_learned.py:107-160)
// ---------------------------------------------------------------------------
__global__ void base_kernel(const float* __restrict__ f_base, float* __restrict__ f_out, int npoi) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < npoi) f_out[i] = (float)clip((double)f_base[i], 0.0, 1.0);
}

// Every index the kernel follows is checked (the host checks the trees when it
// builds the arrays; these guards only keep a malformed array inside bounds): a
// cell whose band has no model keeps its base value, and a tree whose walk
// leaves the tree adds nothing.
__global__ void learned_kernel(IbisForest fo, const double* __restrict__ feats, int ld, const int* __restrict__ pts,
                               const int* __restrict__ band, const double* __restrict__ fclim,
                               const double* __restrict__ pbar, const double* __restrict__ fmax_,
                               const double* __restrict__ stat, const double* __restrict__ lam, int ncells, int npoi,
                               float* __restrict__ f_out) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= ncells) return;
    const int pt = pts[p], b = band[p];
    if (b < 0 || b >= fo.nband || pt < 0 || pt >= npoi) return;
    auto x = [&](int f) -> float {
        return f < IBIS_WETLAND_NFEAT ? (float)feats[(size_t)f * ld + pt]
                                      : (float)stat[(size_t)p * kNStat + (f - IBIS_WETLAND_NFEAT)];
    };
    float out = fo.base_margin[b];
    for (int t = fo.tree_first[b]; t < fo.tree_first[b + 1]; ++t) {
        const int n0 = fo.node_first[t], nn = fo.node_first[t + 1] - n0;
        if (nn <= 0) continue;
        int node = 0;
        for (int depth = 0; node >= 0 && depth < nn && fo.left[n0 + node] >= 0; ++depth) {   // at most nn steps
            const int q = n0 + node;
            const int f = fo.feature[q];
            const float v = (f >= 0 && f < fo.nfeat) ? x(f) : __int_as_float(0x7fc00000);
            const bool go_left = isnan(v) ? fo.default_left[q] != 0 : v < fo.value[q];
            node = go_left ? fo.left[q] : fo.right[q];
            if (node >= nn) node = -1;
        }
        if (node >= 0 && fo.left[n0 + node] < 0) out = __fadd_rn(out, fo.value[n0 + node]);
    }
    if (fo.transform[b] == 1) out = 1.0f / (1.0f + expf(-out));
    const double P = (double)fminf(fmaxf(out, 0.0f), 1.0f);
    const double h = clip(fclim[p] + lam[b] * (P - pbar[p]), 0.0, fmax_[p]);
    f_out[pt] = (float)clip(h, 0.0, 1.0);
}

}  // namespace

extern "C" int ibis_wetland_dynamic_f32(const float* prog, const float* stat, const double* area, float* f_out,
                                        int ncell, int ld, const IbisParams* params, void* stream) {
    if (!prog || !stat || !area || !f_out || !params) return -EINVAL;
    if (ncell < 0 || ld < ncell || ld % 32) return -EINVAL;
    if (ncell == 0) return 0;
    const int block = 128;
    dynamic_kernel<<<(ncell + block - 1) / block, block, 0, (cudaStream_t)stream>>>(
        prog, stat, area, f_out, ncell, ld, params->hsoi[0], params->hsoi[1], params->hsoi[2], params->hsoi[3]);
    return launched("ibis_wetland_dynamic_f32");
}

extern "C" int ibis_wetland_grid(const IbisWetlandBuilder* b, void* stream) {
    if (!builder_ok(b)) return -EINVAL;
    cudaStream_t s = (cudaStream_t)stream;
    const size_t gs = (size_t)b->nlat * b->nlon;
    cudaError_t e = cudaMemsetAsync(b->lf, 0, gs * sizeof(double), s);
    if (e != cudaSuccess) return -(int)e - 1000;
    if (b->npoi > 0) mask_kernel<<<(b->npoi + 127) / 128, 128, 0, s>>>(*b, b->lf);
    const int rc = launched("ibis_wetland_grid");
    return rc ? rc : box_filter(b->lf, b->work, 1, b->nlat, b->nlon, s);
}

extern "C" int ibis_wetland_features(const IbisWetlandBuilder* b, const float* means, const float* totals,
                                     double* feats, void* stream) {
    if (!builder_ok(b) || !b->poros || !b->buf || !means || !totals || !feats) return -EINVAL;
    if (b->npoi == 0) return 0;
    cudaStream_t s = (cudaStream_t)stream;
    const size_t gs = (size_t)b->nlat * b->nlon;
    double* gp = b->work;
    double* gr = b->work + gs;
    cudaError_t e = cudaMemsetAsync(gp, 0, 2 * gs * sizeof(double), s);
    if (e != cudaSuccess) return -(int)e - 1000;
    const int block = 128, grid = (b->npoi + block - 1) / block;
    features_kernel<<<grid, block, 0, s>>>(*b, means, totals, feats, gp, gr);
    int rc = launched("ibis_wetland_features");
    if (!rc) rc = box_filter(gp, b->work + 2 * gs, 2, b->nlat, b->nlon, s);
    if (rc) return rc;
    neighbour_kernel<<<grid, block, 0, s>>>(*b, gp, gr, feats);
    return launched("ibis_wetland_features");
}

extern "C" int ibis_wetland_learned(const IbisForest* forest, const double* feats, int npoi, int ld, const int* pts,
                                    const int* band, const double* fclim, const double* pbar, const double* fmax,
                                    const double* stat, const double* lam, int ncells, const float* f_base,
                                    float* f_out, void* stream) {
    if (!forest || !feats || !f_base || !f_out || npoi < 0 || ld < npoi || ld % 32 || ncells < 0) return -EINVAL;
    if (ncells > 0 && (!pts || !band || !fclim || !pbar || !fmax || !stat || !lam)) return -EINVAL;
    if (forest->nband < 0 || forest->nfeat != IBIS_WETLAND_NFEAT + kNStat) return -EINVAL;
    if (forest->nband > 0 && (!forest->tree_first || !forest->node_first || !forest->left || !forest->right ||
                              !forest->feature || !forest->value || !forest->default_left ||
                              !forest->base_margin || !forest->transform))
        return -EINVAL;
    cudaStream_t s = (cudaStream_t)stream;
    if (npoi > 0) base_kernel<<<(npoi + 127) / 128, 128, 0, s>>>(f_base, f_out, npoi);
    int rc = launched("ibis_wetland_learned");
    if (rc || ncells == 0) return rc;
    learned_kernel<<<(ncells + 127) / 128, 128, 0, s>>>(*forest, feats, ld, pts, band, fclim, pbar, fmax, stat, lam,
                                                         ncells, npoi, f_out);
    return launched("ibis_wetland_learned");
}
