// Self-written exp and erfc for the GAMERA step, usable from host and device.
//
// The MHD face fluxes call erfc four times and exp twice per face
// (stress.F90:432-599, GasKinFlux / MagKinFlux). Library implementations of
// these functions differ by an ulp or two between the host libm and the GPU,
// which is enough to stop a bit-for-bit comparison of a GPU step against a CPU
// step. These two functions use only IEEE operations that both sides round
// the same way: +, -, *, /, fma (called explicitly: one rounding), comparisons
// and exact scalings, so a GPU kernel and a CPU build produce identical bits
// (the kernels of the strict step are built without implicit FMA contraction,
// the CPU restatement with -ffp-contract=off; the explicit fma calls below are
// fused on both).
//
// Construction (see gen_gam_math.py, which generates the coefficients):
//   gam_exp(a, b) = e^(a+b): table-driven (Tang, ACM TOMS 15(2), 1989):
//     a+b = (128 m + j) ln2/128 + r, |r| <= ln2/256 (ln2/128 split in a
//     32-bit head and a tail, k*head exact), e^(a+b) = 2^m (T_hi + T_lo) e^r
//     with 2^(j/128) = T_hi + T_lo from a 128-entry table and e^r - 1 by its
//     degree-5 Taylor polynomial; the result is T_hi + (T_hi p + T_lo), one
//     rounding of a sum whose small part carries ~2^-60 relative error
//     (about 0.51 ulp in total). The split argument lets erfc pass -x^2 as an
//     exact head plus a small tail.
//   gam_erfc(x) = exp(-x^2) * g(s) / (x + 4), s = (A x - B)/(x + 4) for x >= 0,
//     g a degree-22 Chebyshev fit of erfcx(x)*(x+4) on [0, 27.5], evaluated by
//     Estrin's scheme with fmas; erfc(x) = 2 - erfc(-x) for x < 0.
// Accuracy against mpmath: exp within 0.51 ulp, erfc within a few ulp (the
// golden values in tests/golden/erfc_exp.json, checked by
// test_erfc_exp_golden in tests/test_oracle.py).
#pragma once

#include <stdint.h>
#include <math.h>
#include "gam_math_coeffs.h"

#if defined(__CUDACC__)
#define GAM_HD __host__ __device__ __forceinline__
#else
#define GAM_HD static inline
#endif

namespace gam {

// 2^k as a double, for -1022 <= k <= 1023.
GAM_HD double pow2i(int k) {
    uint64_t u = (uint64_t)(k + 1023) << 52;
#if defined(__CUDA_ARCH__)
    return __longlong_as_double((long long)u);
#else
    double d;
    __builtin_memcpy(&d, &u, sizeof(d));
    return d;
#endif
}

GAM_HD double round_even(double x) {
#if defined(__CUDA_ARCH__)
    return rint(x);
#else
    return __builtin_rint(x);  // default rounding mode: nearest, ties to even
#endif
}

// 2^(j/128) = T_hi + T_lo, j = 0..127 (pairs), for host and device code
#if defined(__CUDACC__)
static __device__ const double gam_exp_tab_d[2 * GAM_EXP_N] = GAM_EXP_TAB_INIT;
#endif
static const double gam_exp_tab_h[2 * GAM_EXP_N] = GAM_EXP_TAB_INIT;

GAM_HD double exp_tab(int i) {
#if defined(__CUDA_ARCH__)
    return __ldg(&gam_exp_tab_d[i]);
#else
    return gam_exp_tab_h[i];
#endif
}

// e^(a+b) from the reduced argument: x = a + b = k ln2/128 + r, e^x =
// 2^(k/128) e^r with 2^(j/128) from the table (j = k mod 128) and the scale
// 2^m = 2^((k-j)/128) applied in one (m in the normal range) or two steps.
GAM_HD double exp_ab_core(double a, double b, double x, bool wide) {
    const double kd = round_even(x * GAM_INV_LN2N);
    const int k = (int)kd;
    double r = fma(-kd, GAM_LN2N_HI, a) + b;  // a - k*head is exact
    r = fma(-kd, GAM_LN2N_LO, r);
    // e^r - 1 = r + r^2 (C2 + r (C3 + r (C4 + r C5)))
    double c = fma(r, GAM_EXP_C5, GAM_EXP_C4);
    c = fma(r, c, GAM_EXP_C3);
    c = fma(r, c, GAM_EXP_C2);
    const double p = fma(r * r, c, r);
    const int j = k & (GAM_EXP_N - 1);
    const int m = (k - j) / GAM_EXP_N;  // exact: k - j is a multiple of 128
    const double th = exp_tab(2 * j), tl = exp_tab(2 * j + 1);
    const double y = th + fma(th, p, tl);
    if (wide) {
        if (m > 1023) return (y * 2.0) * pow2i(m - 1);
        if (m < -1021) return (y * pow2i(m + 600)) * pow2i(-600);
    }
    return y * pow2i(m);
}

// the arguments near or beyond the ends of the range, and NaN
GAM_HD double exp_ab_edge(double a, double b, double x) {
    if (!(x < 709.78)) {  // overflow threshold, also catches NaN
        if (x != x) return x;
        if (x > 709.782712893384) return INFINITY;
    }
    if (x < -745.2) return 0.0;
    return exp_ab_core(a, b, x, true);
}

// e^(a+b); b may carry a small tail of the exponent that a could not hold.
// |x| < 707 keeps k / 128 within [-1020, 1020]: one scaling, no special cases.
GAM_HD double exp_ab(double a, double b) {
    const double x = a + b;
    if (fabs(x) < 707.0) return exp_ab_core(a, b, x, false);
    return exp_ab_edge(a, b, x);
}

GAM_HD double gam_exp(double x) { return exp_ab(x, 0.0); }

GAM_HD double gam_erfc(double x) {
    const double ax = fabs(x);
    double res;
    if (ax > 27.5) {
        res = 0.0;
    } else {
        const double q = 1.0 / (ax + GAM_ERFC_L);
        const double s = fma(GAM_ERFC_A, ax, -GAM_ERFC_B) * q;
        // g(s) by Estrin's scheme with fmas (dependency depth 6 instead of 22)
        const double s2 = s * s, s4 = s2 * s2, s8 = s4 * s4, s16 = s8 * s8;
        const double a0 = fma(GAM_ERFC_G1, s, GAM_ERFC_G0), a1 = fma(GAM_ERFC_G3, s, GAM_ERFC_G2);
        const double a2 = fma(GAM_ERFC_G5, s, GAM_ERFC_G4), a3 = fma(GAM_ERFC_G7, s, GAM_ERFC_G6);
        const double a4 = fma(GAM_ERFC_G9, s, GAM_ERFC_G8), a5 = fma(GAM_ERFC_G11, s, GAM_ERFC_G10);
        const double a6 = fma(GAM_ERFC_G13, s, GAM_ERFC_G12), a7 = fma(GAM_ERFC_G15, s, GAM_ERFC_G14);
        const double a8 = fma(GAM_ERFC_G17, s, GAM_ERFC_G16), a9 = fma(GAM_ERFC_G19, s, GAM_ERFC_G18);
        const double a10 = fma(GAM_ERFC_G21, s, GAM_ERFC_G20);
        const double b0 = fma(a1, s2, a0), b1 = fma(a3, s2, a2), b2 = fma(a5, s2, a4), b3 = fma(a7, s2, a6);
        const double b4 = fma(a9, s2, a8), b5 = fma(GAM_ERFC_G22, s2, a10);
        const double c0 = fma(b1, s4, b0), c1 = fma(b3, s4, b2), c2 = fma(b5, s4, b4);
        const double d0 = fma(c1, s8, c0);
        const double g = fma(c2, s16, d0);
        // -x^2 = -xh^2 (exact, xh = x truncated to 1/16) - (x-xh)(x+xh)
        const double xh = trunc(ax * 16.0) * 0.0625;
        const double e = exp_ab(-(xh * xh), -((ax - xh) * (ax + xh)));
        res = (g * q) * e;
    }
    if (x < 0.0) res = 2.0 - res;
    if (x != x) res = x;
    return res;
}

}  // namespace gam
