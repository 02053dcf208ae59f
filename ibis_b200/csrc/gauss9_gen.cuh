// Generated by gen_gauss9.py -- do not edit.
// No-pivot Gaussian elimination of the 9x9 canopy system on its filled
// nonzero pattern (45 entries), then back substitution.
#pragma once

namespace ibis {

struct Sys9 {
    double a00, a03, a05, a11, a13, a15, a22, a24, a26, a30, a31, a33, a34, a35, a42, a43, a44, a45, a46, a47, a48, a50, a51, a53, a54, a55, a56, a57, a58, a62, a64, a65, a66, a67, a68, a74, a75, a76, a77, a78, a84, a85, a86, a87, a88;
    double b0, b1, b2, b3, b4, b5, b6, b7, b8;
};

__device__ __forceinline__ void sys9_zero(Sys9& s) {
    s.a00 = 0.0; s.a03 = 0.0; s.a05 = 0.0; s.a11 = 0.0; s.a13 = 0.0; s.a15 = 0.0; s.a22 = 0.0; s.a24 = 0.0; s.a26 = 0.0; s.a30 = 0.0; s.a31 = 0.0; s.a33 = 0.0; s.a34 = 0.0; s.a35 = 0.0; s.a42 = 0.0; s.a43 = 0.0; s.a44 = 0.0; s.a45 = 0.0; s.a46 = 0.0; s.a47 = 0.0; s.a48 = 0.0; s.a50 = 0.0; s.a51 = 0.0; s.a53 = 0.0; s.a54 = 0.0; s.a55 = 0.0; s.a56 = 0.0; s.a57 = 0.0; s.a58 = 0.0; s.a62 = 0.0; s.a64 = 0.0; s.a65 = 0.0; s.a66 = 0.0; s.a67 = 0.0; s.a68 = 0.0; s.a74 = 0.0; s.a75 = 0.0; s.a76 = 0.0; s.a77 = 0.0; s.a78 = 0.0; s.a84 = 0.0; s.a85 = 0.0; s.a86 = 0.0; s.a87 = 0.0; s.a88 = 0.0;
}

// Each pivot's reciprocal is formed once and reused by the rows below it and by
// the back substitution (one division per unknown instead of one per update).
__device__ __forceinline__ void sys9_solve(Sys9& s, double (&x)[9]) {
    double f;
    double r0, r1, r2, r3, r4, r5, r6, r7, r8;
    r0 = rcp(s.a00);
    f = s.a30 * r0;
    s.a33 = s.a33 - f * s.a03;
    s.a35 = s.a35 - f * s.a05;
    s.b3 = s.b3 - f * s.b0;
    f = s.a50 * r0;
    s.a53 = s.a53 - f * s.a03;
    s.a55 = s.a55 - f * s.a05;
    s.b5 = s.b5 - f * s.b0;
    r1 = rcp(s.a11);
    f = s.a31 * r1;
    s.a33 = s.a33 - f * s.a13;
    s.a35 = s.a35 - f * s.a15;
    s.b3 = s.b3 - f * s.b1;
    f = s.a51 * r1;
    s.a53 = s.a53 - f * s.a13;
    s.a55 = s.a55 - f * s.a15;
    s.b5 = s.b5 - f * s.b1;
    r2 = rcp(s.a22);
    f = s.a42 * r2;
    s.a44 = s.a44 - f * s.a24;
    s.a46 = s.a46 - f * s.a26;
    s.b4 = s.b4 - f * s.b2;
    f = s.a62 * r2;
    s.a64 = s.a64 - f * s.a24;
    s.a66 = s.a66 - f * s.a26;
    s.b6 = s.b6 - f * s.b2;
    r3 = rcp(s.a33);
    f = s.a43 * r3;
    s.a44 = s.a44 - f * s.a34;
    s.a45 = s.a45 - f * s.a35;
    s.b4 = s.b4 - f * s.b3;
    f = s.a53 * r3;
    s.a54 = s.a54 - f * s.a34;
    s.a55 = s.a55 - f * s.a35;
    s.b5 = s.b5 - f * s.b3;
    r4 = rcp(s.a44);
    f = s.a54 * r4;
    s.a55 = s.a55 - f * s.a45;
    s.a56 = s.a56 - f * s.a46;
    s.a57 = s.a57 - f * s.a47;
    s.a58 = s.a58 - f * s.a48;
    s.b5 = s.b5 - f * s.b4;
    f = s.a64 * r4;
    s.a65 = s.a65 - f * s.a45;
    s.a66 = s.a66 - f * s.a46;
    s.a67 = s.a67 - f * s.a47;
    s.a68 = s.a68 - f * s.a48;
    s.b6 = s.b6 - f * s.b4;
    f = s.a74 * r4;
    s.a75 = s.a75 - f * s.a45;
    s.a76 = s.a76 - f * s.a46;
    s.a77 = s.a77 - f * s.a47;
    s.a78 = s.a78 - f * s.a48;
    s.b7 = s.b7 - f * s.b4;
    f = s.a84 * r4;
    s.a85 = s.a85 - f * s.a45;
    s.a86 = s.a86 - f * s.a46;
    s.a87 = s.a87 - f * s.a47;
    s.a88 = s.a88 - f * s.a48;
    s.b8 = s.b8 - f * s.b4;
    r5 = rcp(s.a55);
    f = s.a65 * r5;
    s.a66 = s.a66 - f * s.a56;
    s.a67 = s.a67 - f * s.a57;
    s.a68 = s.a68 - f * s.a58;
    s.b6 = s.b6 - f * s.b5;
    f = s.a75 * r5;
    s.a76 = s.a76 - f * s.a56;
    s.a77 = s.a77 - f * s.a57;
    s.a78 = s.a78 - f * s.a58;
    s.b7 = s.b7 - f * s.b5;
    f = s.a85 * r5;
    s.a86 = s.a86 - f * s.a56;
    s.a87 = s.a87 - f * s.a57;
    s.a88 = s.a88 - f * s.a58;
    s.b8 = s.b8 - f * s.b5;
    r6 = rcp(s.a66);
    f = s.a76 * r6;
    s.a77 = s.a77 - f * s.a67;
    s.a78 = s.a78 - f * s.a68;
    s.b7 = s.b7 - f * s.b6;
    f = s.a86 * r6;
    s.a87 = s.a87 - f * s.a67;
    s.a88 = s.a88 - f * s.a68;
    s.b8 = s.b8 - f * s.b6;
    r7 = rcp(s.a77);
    f = s.a87 * r7;
    s.a88 = s.a88 - f * s.a78;
    s.b8 = s.b8 - f * s.b7;
    r8 = rcp(s.a88);
    x[8] = s.b8 * r8;
    x[7] = (s.b7 - s.a78 * x[8]) * r7;
    x[6] = (s.b6 - (s.a67 * x[7] + s.a68 * x[8])) * r6;
    x[5] = (s.b5 - ((s.a56 * x[6] + s.a57 * x[7]) + s.a58 * x[8])) * r5;
    x[4] = (s.b4 - (((s.a45 * x[5] + s.a46 * x[6]) + s.a47 * x[7]) + s.a48 * x[8])) * r4;
    x[3] = (s.b3 - (s.a34 * x[4] + s.a35 * x[5])) * r3;
    x[2] = (s.b2 - (s.a24 * x[4] + s.a26 * x[6])) * r2;
    x[1] = (s.b1 - (s.a13 * x[3] + s.a15 * x[5])) * r1;
    x[0] = (s.b0 - (s.a03 * x[3] + s.a05 * x[5])) * r0;
}

}  // namespace ibis
