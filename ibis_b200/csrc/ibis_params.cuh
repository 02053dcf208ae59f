// Device copy of the parameter record, converted once on the host to the
// kernel's arithmetic type, plus constants derived from it in double.
#pragma once
#include "../../include/ibis_layout.h"

namespace ibis {

template <typename R>
struct DevParams {
#define IBIS_S(name) R name;
#define IBIS_A(name, n) R name[n];
    IBIS_PARAM_LIST(IBIS_S, IBIS_A)
#undef IBIS_S
#undef IBIS_A
    unsigned int flags;
    // ---- derived in double on the host (kept in the same precision the reference forms them)
    R tfac;            // 1 / 0.999**cappa (canopy_exchange.py:206)
    R vonk2;           // vonk**2
    R cdmax;           // 300 / (2 dtime)
    R zweight;         // exp(-1 / (10 * 86400 / dtime)) (stomata.py:486)
    R wliqmin, wsnomin;  // interception.py:292-293
    R znorm;           // 1 - exp(stressfac) (stomata.py:545)
    R rdt;             // 1 / dtime
    R zir;             // 4 * 0.95 * stef (loops.py:170; canopy_exchange.py:566)
    // soil-water solve geometry, always double (soil_physics.py:238-330)
    double sw_hm[6];   // interface k (1..5): 0.5 * (h[k-1] + h[k])
    double sw_wp[6];   // 0.5 * h[k] / sw_hm[k]
    double sw_wm[6];   // 1 - sw_wp[k]
    double sw_hb[6];   // row k: max(0.5 h[0] | 0.5 h[k-1] + 0.5 h[k], 1e-30)
    double sw_hp[6];   // row k < 5: max(0.5 * (h[k] + h[k+1]), 1e-30)
    // the same geometry as multipliers, so the solve divides only by values
    // that change per cell: 1/sw_hm, 1/sw_hb, 1/sw_hp, 0.5 h[k]/sw_hb,
    // 0.5 h[k+1]/sw_hp, 0.5 h[k-1]/sw_hb, 0.5 h[k]/sw_hp
    double sw_rhm[6], sw_rhb[6], sw_rhp[6], sw_c1[6], sw_c3[6], sw_c5[6], sw_c6[6];
    double rdt64;      // 1 / dtime in double
    double rrhow64;    // 1 / rhow in double
    // float copies of sw_wp, sw_wm and the multipliers, for the FP32 kernels'
    // increment-form soil-water solve
    float sw32_wp[6], sw32_wm[6], sw32_rhm[6], sw32_rhb[6], sw32_rhp[6], sw32_c1[6], sw32_c3[6], sw32_c5[6],
        sw32_c6[6];
    R rwood_s[12], rroot_s[12], keep[12];  // float32-formed respiration rates (loops_gswp3.py:185-190)
    R ch4_w;           // float32(dtime / 86400)
    R rh_conv;         // float32(12e-3 * 86400)
    R ch4_wtop[6];     // thickness weights of the wetland water-table average (methane.py:266-270)
    R ch4_wtot;        // their sum, floored at 1e-12
    R hsoi_top[6], hsoi_bot[6];  // layer tops/bottoms (cumsum of hsoi)
    // per-PFT capacity increment per unit cropland share (loops.py:218-231): the C4
    // (PFT 10) and C3 (PFT 11) vmax scales less one, formed in float32 as the
    // reference forms them on float32 masks; zero for the other PFTs
    R crop_inc[12];
    // index of the launch's first column in the caller's numbering: a launch
    // over a group of columns (ibis_step_host_f32) reports status[1] in it
    int cell0;
    // per-band thickness weights of the wetland water-table average and their
    // sums (IBIS_FLAG_CH4_BANDS: from ch4b_z_wt_ref as ch4_wtop from z_wt_ref)
    R ch4b_wtop[3][6];
    R ch4b_wtot[3];
};

// The parameters a calibration ensemble varies per run (the 31-parameter
// vector: vmax per plant type, Ball-Berry slopes, soil-stress shape,
// soil-evaporation exponent, interception capacities, wet fraction cap,
// wetland-CH4 parameters, maintenance/growth respiration), and the values
// derived from them.  The physics reads them through one of two sources:
// UniformQ (one parameter record for every cell) or RunQ (one run's values,
// 33 words: an odd stride, so a warp reading one field of its 32 runs' records
// in shared memory touches 32 different banks).
//
// ``x3`` marks the sources of the kernels compiled with the IBIS 3.0 extensions
// of the step (IBIS_FLAGS_X3): the F77 kernels carry none of their code.
template <typename R>
struct UniformQ {
    static constexpr bool x3 = false;
    const DevParams<R>& P;
    __device__ __forceinline__ R vmax(int j) const { return P.vmax_pft[j]; }
    __device__ __forceinline__ R coefm(int g) const { return P.coefm[g]; }
    __device__ __forceinline__ R stressfac() const { return P.stressfac; }
    __device__ __forceinline__ R znorm() const { return P.znorm; }
    __device__ __forceinline__ R beta_power() const { return P.soil_beta_power; }
    __device__ __forceinline__ R wliqumax() const { return P.wliqumax; }
    __device__ __forceinline__ R wliqsmax() const { return P.wliqsmax; }
    __device__ __forceinline__ R wliqlmax() const { return P.wliqlmax; }
    __device__ __forceinline__ R fmax() const { return P.fmax; }
    __device__ __forceinline__ R wliqmin() const { return P.wliqmin; }
    __device__ __forceinline__ R r_ch4() const { return P.r_ch4; }
    __device__ __forceinline__ R q10p() const { return P.q10p; }
    __device__ __forceinline__ R z_tau() const { return P.z_tau; }
    __device__ __forceinline__ R tau_oxid() const { return P.tau_oxid; }
    __device__ __forceinline__ R z_wt_max() const { return P.z_wt_max; }
    __device__ __forceinline__ R rwood(int j) const { return P.rwood_s[j]; }
    __device__ __forceinline__ R rroot(int j) const { return P.rroot_s[j]; }
    __device__ __forceinline__ R keep(int j) const { return P.keep[j]; }
};

// One parameter record for every cell, in the kernels that carry the IBIS 3.0
// extensions.
template <typename R>
struct UniformQ3 : UniformQ<R> {
    static constexpr bool x3 = true;
};

template <typename R>
struct RunQ {
    static constexpr bool x3 = false;
    R vmax_[12], coefm_[5], stressfac_, znorm_, beta_, wliqumax_, wliqsmax_, wliqlmax_, fmax_, wliqmin_;
    R r_ch4_, q10p_, z_tau_, tau_oxid_, z_wt_max_, rwood_, rroot_, keep_;
    __device__ __forceinline__ R vmax(int j) const { return vmax_[j]; }
    __device__ __forceinline__ R coefm(int g) const { return coefm_[g]; }
    __device__ __forceinline__ R stressfac() const { return stressfac_; }
    __device__ __forceinline__ R znorm() const { return znorm_; }
    __device__ __forceinline__ R beta_power() const { return beta_; }
    __device__ __forceinline__ R wliqumax() const { return wliqumax_; }
    __device__ __forceinline__ R wliqsmax() const { return wliqsmax_; }
    __device__ __forceinline__ R wliqlmax() const { return wliqlmax_; }
    __device__ __forceinline__ R fmax() const { return fmax_; }
    __device__ __forceinline__ R wliqmin() const { return wliqmin_; }
    __device__ __forceinline__ R r_ch4() const { return r_ch4_; }
    __device__ __forceinline__ R q10p() const { return q10p_; }
    __device__ __forceinline__ R z_tau() const { return z_tau_; }
    __device__ __forceinline__ R tau_oxid() const { return tau_oxid_; }
    __device__ __forceinline__ R z_wt_max() const { return z_wt_max_; }
    __device__ __forceinline__ R rwood(int) const { return rwood_; }
    __device__ __forceinline__ R rroot(int) const { return rroot_; }
    __device__ __forceinline__ R keep(int) const { return keep_; }
};

// One run's parameters in the kernels that carry the IBIS 3.0 extensions (the
// same record; the extensions' own tables come from the parameter record).
template <typename R>
struct RunQ3 : RunQ<R> {
    static constexpr bool x3 = true;
};
static_assert(sizeof(RunQ3<float>) == sizeof(RunQ<float>), "the run record's shared-memory size is one");

}  // namespace ibis
