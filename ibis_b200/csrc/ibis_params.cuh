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
    R rwood_s[12], rroot_s[12], keep[12];  // float32-formed respiration rates (loops_gswp3.py:185-190)
    R ch4_w;           // float32(dtime / 86400)
    R rh_conv;         // float32(12e-3 * 86400)
    R ch4_wtop[6];     // thickness weights of the wetland water-table average (methane.py:266-270)
    R ch4_wtot;        // their sum, floored at 1e-12
    R hsoi_top[6], hsoi_bot[6];  // layer tops/bottoms (cumsum of hsoi)
};

}  // namespace ibis
