// Monthly wetland methane at the month's ends (python-port/ibis/bgc/methane.py:431-496,
// called by the GSWP3 month driver, timestepping/loops_gswp3.py:740-760, and
// composed with the learned-area scaling and the carbon partition as in
// scripts/run_global.py:786-839).  One thread per cell over the WET planes.
#pragma once
#include "ibis_ground.cuh"

namespace ibis {

// Month start: zero the step's CH4 day-mean accumulator (and its compensation),
// keep the heterotrophic respiration total (ayco2mic) the carbon partition
// needs, and at a new year clear the annual sums (reset_annual, methane.py:477-480).
template <typename R>
__global__ void __launch_bounds__(128) month_begin_kernel(R* __restrict__ acc, R* __restrict__ wet,
                                                          const R* __restrict__ dayst, int ncell, int ld,
                                                          bool new_year) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ncell) return;
    acc[(size_t)IBIS_ACC_CH4 * ld + i] = R(0.0);
    acc[(size_t)(IBIS_ACC_CH4 + IBIS_ACC_COUNT) * ld + i] = R(0.0);
    wet[(size_t)IBIS_WET_RH0 * ld + i] = dayst ? dayst[(size_t)IBIS_DAYST_AYCO2MIC * ld + i] : R(0.0);
    if (new_year) {
        wet[(size_t)IBIS_WET_ANNUAL * ld + i] = R(0.0);
        wet[(size_t)IBIS_WET_CH4C * ld + i] = R(0.0);
    }
}

// Month end: methane_step (the flux from the end-of-month state, methane.py:431-456)
// or methane_step_from_mean (the month's mean of the hourly fluxes,
// methane.py:459-474), then scale_month (methane.py:483-489) where a per-cell
// inundated fraction is given, then ch4_carbon_from_rh (methane.py:492-496)
// booked out of ayco2mic when partitioning.
template <typename R>
__global__ void __launch_bounds__(128) month_end_kernel(const R* __restrict__ prog, const R* __restrict__ stat,
                                                        const R* __restrict__ acc, R* __restrict__ wet,
                                                        R* __restrict__ dayst, const R* __restrict__ scale,
                                                        int ncell, int ld, int ndays, const DevParams<R> P,
                                                        bool from_mean, bool partition) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ncell) return;
    auto G = [&](int p) { return prog[(size_t)p * ld + i]; };
    auto S = [&](int p) { return stat[(size_t)p * ld + i]; };
    R* W = wet + i;
    R t[NL], w[NL], ic[NL];
#pragma unroll
    for (int k = 0; k < NL; ++k) {
        t[k] = G(IBIS_PROG_TSOI + k);
        w[k] = G(IBIS_PROG_WSOI + k);
        ic[k] = G(IBIS_PROG_WISOI + k);
    }
    const UniformQ<R> q{P};
    const Ch4Par<R> m = ch4_params((P.flags & IBIS_FLAG_CH4_BANDS) ? S(IBIS_STAT_CH4_BAND) : R(0.0), P, q);
    const R zo = (P.flags & IBIS_FLAG_ZWT_OBS) ? S(IBIS_STAT_ZWT_OBS) : R(NAN);
    const R nd = R(ndays);
    const R a0 = W[(size_t)IBIS_WET_ANNUAL * ld];
    R flux;
    if (from_mean) {
        flux = (acc[(size_t)IBIS_ACC_CH4 * ld + i] - acc[(size_t)(IBIS_ACC_CH4 + IBIS_ACC_COUNT) * ld + i]) / nd;
    } else {
        const R rh = S(IBIS_STAT_TCO2MIC) * P.rh_conv;
        flux = methane(S(IBIS_STAT_F_INUND), rh, t, w, ic, zo, m, P);
    }
    const R zwt = wetland_water_table(w, ic, m, zo);
    R annual = a0 + flux * nd;
    if (scale) {
        const R f = R((float)scale[i]);
        flux = flux * f;
        annual = a0 + (annual - a0) * f;
    }
    W[(size_t)IBIS_WET_FLUX * ld] = flux;
    W[(size_t)IBIS_WET_ANNUAL * ld] = annual;
    W[(size_t)IBIS_WET_ZWT * ld] = zwt;
    if (partition) {
        R* ay = dayst + (size_t)IBIS_DAYST_AYCO2MIC * ld + i;
        const R rh_now = *ay;
        const R take = mn(mx(annual - a0, R(0.0)), mx(rh_now - W[(size_t)IBIS_WET_RH0 * ld], R(0.0)));
        *ay = rh_now - take;
        W[(size_t)IBIS_WET_CH4C * ld] = W[(size_t)IBIS_WET_CH4C * ld] + take;
    }
}

}  // namespace ibis
