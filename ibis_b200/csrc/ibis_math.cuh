// Scalar math helpers shared by the column kernels.
//
// Every routine works on one column (one cell per thread).  R is the bulk
// arithmetic type (float for the production kernels, double for the float64
// kernels); a few solves are always carried out in double (see ibis_column.cuh).
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

namespace ibis {

__device__ __forceinline__ float ex(float x) { return expf(x); }
__device__ __forceinline__ double ex(double x) { return exp(x); }
__device__ __forceinline__ float lg(float x) { return logf(x); }
__device__ __forceinline__ double lg(double x) { return log(x); }
__device__ __forceinline__ float sq(float x) { return sqrtf(x); }
__device__ __forceinline__ double sq(double x) { return sqrt(x); }
__device__ __forceinline__ float pw(float x, float y) { return powf(x, y); }
__device__ __forceinline__ double pw(double x, double y) { return pow(x, y); }
__device__ __forceinline__ float em1(float x) { return expm1f(x); }
__device__ __forceinline__ double em1(double x) { return expm1(x); }
__device__ __forceinline__ float mx(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ double mx(double a, double b) { return fmax(a, b); }
__device__ __forceinline__ float mn(float a, float b) { return fminf(a, b); }
__device__ __forceinline__ double mn(double a, double b) { return fmin(a, b); }
__device__ __forceinline__ float ab(float x) { return fabsf(x); }
__device__ __forceinline__ double ab(double x) { return fabs(x); }
__device__ __forceinline__ bool finite(float x) { return isfinite(x); }
__device__ __forceinline__ bool finite(double x) { return isfinite(x); }

template <typename R>
__device__ __forceinline__ R clip(R x, R lo, R hi) { return mn(mx(x, lo), hi); }

// x**3 and x**4 as XLA evaluates a static integer power (repeated squaring).
template <typename R>
__device__ __forceinline__ R cube(R x) { return x * (x * x); }
template <typename R>
__device__ __forceinline__ R quart(R x) { R x2 = x * x; return x2 * x2; }

// x**n for a small non-negative integer n (n <= 40), by repeated squaring.
// Reciprocal: correctly rounded in double (the same bits as 1.0 / x, by the
// reciprocal instruction sequence rather than the general division); the
// build's single-precision division in float.
__device__ __forceinline__ double rcp(double x) { return __drcp_rn(x); }
__device__ __forceinline__ float rcp(float x) { return 1.0f / x; }

// a / b inside the FP64 islands.  The FP32 kernels (R = float) multiply by the
// reciprocal, which is shorter than a correctly rounded division and moves the
// result by about one unit in the last place of a double -- far below their
// FP32 error.  The FP64 kernels (R = double) keep the division, so they follow
// the reference's float64 arithmetic operation for operation.
template <typename R>
__device__ __forceinline__ double dv(double a, double b) {
    if constexpr (sizeof(R) == 4) return a * rcp(b);
    else return a / b;
}

__device__ __forceinline__ double ipow(double x, int n) {
    double r = 1.0, b = x;
    bool any = false;
#pragma unroll
    for (int k = 0; k < 6; ++k) {                 // predicated: no per-cell trip count
        if (n & 1) { r = any ? r * b : b; any = true; }
        n >>= 1;
        if (n) b = b * b;
    }
    return any ? r : 1.0;
}

__device__ __forceinline__ float ipow(float x, int n) {
    float r = 1.0f, b = x;
    bool any = false;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        if (n & 1) { r = any ? r * b : b; any = true; }
        n >>= 1;
        if (n) b = b * b;
    }
    return any ? r : 1.0f;
}

// ---------------------------------------------------------------------------
// Lowe (1977) saturation vapour pressure and its derivative, both branches
// evaluated on clamped offsets (reference physics/thermo.py:38-174).
// ---------------------------------------------------------------------------
// Both branches of the polynomial are evaluated on offsets clamped to their range.
#define IBIS_LOWE(t, L0, L1, L2, L3, L4, L5, L6, I0, I1, I2, I3, I4, I5, I6)                                  \
    do {                                                                                                     \
        R d_ = (t) - R(273.16);                                                                              \
        R dl_ = clip(d_, R(0.0), R(100.0));                                                                  \
        R di_ = clip(d_, R(-60.0), R(0.0));                                                                  \
        R base_ = ((t) >= R(273.16)) ? R(L0) : R(I0);                                                        \
        R pl_ = dl_ * (R(L1) + dl_ * (R(L2) + dl_ * (R(L3) + dl_ * (R(L4) + dl_ * (R(L5) + dl_ * R(L6))))));  \
        R pi_ = di_ * (R(I1) + di_ * (R(I2) + di_ * (R(I3) + di_ * (R(I4) + di_ * (R(I5) + di_ * R(I6))))));  \
        return R(100.0) * (base_ + pl_ + pi_);                                                               \
    } while (0)

template <typename R>
__device__ __forceinline__ R esat(R t) {
    IBIS_LOWE(t, 6.1078000, 4.4365185e-1, 1.4289458e-2, 2.6506485e-4, 3.0312404e-6, 2.0340809e-8, 6.1368209e-11,
              6.1091780, 5.0346990e-1, 1.8860134e-2, 4.1762237e-4, 5.8247203e-6, 4.8388032e-8, 1.8388269e-10);
}
template <typename R>
__device__ __forceinline__ R desat(R t) {
    IBIS_LOWE(t, 4.4381000e-1, 2.8570026e-2, 7.9380540e-4, 1.2152151e-5, 1.0365614e-7, 3.5324218e-10, -7.0902448e-13,
              5.0303052e-1, 3.7732550e-2, 1.2679954e-3, 2.4775631e-5, 3.0056931e-7, 2.1585425e-9, 7.1310977e-12);
}
#undef IBIS_LOWE

template <typename R>
__device__ __forceinline__ R qsat(R e, R p) {
    return R(0.622) * e / mx(p - R(1.0 - 0.622) * e, R(0.622) * e);
}
template <typename R>
__device__ __forceinline__ R dqsat(R t, R q, R e) {
    return desat(t) * q * (R(1.0) + q * R(1.0 / 0.622 - 1.0)) / e;
}

}  // namespace ibis
