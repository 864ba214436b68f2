// Self-written exp and erfc for the GAMERA step, usable from host and device.
//
// The MHD face fluxes call erfc four times and exp twice per face
// (stress.F90:432-599, GasKinFlux / MagKinFlux). Library implementations of
// these functions differ by an ulp or two between the host libm and the GPU,
// which is enough to stop a bit-for-bit comparison of a GPU step against a CPU
// step. These two functions use only +, -, *, / and comparisons (all IEEE
// correctly rounded on both sides), so a GPU kernel built without FMA
// contraction and a CPU build with -ffp-contract=off produce identical bits.
//
// Construction (see gen_gam_math.py, which generates the coefficients):
//   gam_exp(a, b) = e^(a+b): x = k*ln2 + r with ln2 split in a 32-bit head and
//     a tail (k*ln2_hi exact), e^r from its Taylor series to degree 13 (Estrin
//     evaluation, short dependency chains for the GPU), exact scaling by 2^k.
//     The split argument lets erfc pass -x^2 as an exact head plus a small tail.
//   gam_erfc(x) = exp(-x^2) * g(s) / (x + 4), s = (A x - B)/(x + 4) for x >= 0,
//     g a degree-22 Chebyshev fit of erfcx(x)*(x+4) on [0, 27.5], evaluated by
//     Estrin's scheme;
//     erfc(x) = 2 - erfc(-x) for x < 0.
// Accuracy against mpmath: a few ulp over the whole range (tests/test_gam_math.py).
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

// e^(a+b); b may carry a small tail of the exponent that a could not hold.
GAM_HD double exp_ab(double a, double b) {
    const double x = a + b;
    if (!(x < 709.78)) {  // overflow threshold, also catches NaN
        if (x != x) return x;
        if (x > 709.782712893384) return INFINITY;
    }
    if (x < -745.2) return 0.0;
    const double kd = round_even(x * GAM_INV_LN2);
    const int k = (int)kd;
    double r = (a - kd * GAM_LN2_HI) + b;  // a - k*ln2_hi is exact
    r = r - kd * GAM_LN2_LO;
    // Taylor polynomial by Estrin's scheme (dependency depth 5 instead of 13)
    const double r2 = r * r, r4 = r2 * r2, r8 = r4 * r4;
    const double p01 = GAM_EXP_C0 + GAM_EXP_C1 * r, p23 = GAM_EXP_C2 + GAM_EXP_C3 * r;
    const double p45 = GAM_EXP_C4 + GAM_EXP_C5 * r, p67 = GAM_EXP_C6 + GAM_EXP_C7 * r;
    const double p89 = GAM_EXP_C8 + GAM_EXP_C9 * r, pab = GAM_EXP_C10 + GAM_EXP_C11 * r;
    const double pcd = GAM_EXP_C12 + GAM_EXP_C13 * r;
    const double q0 = p01 + p23 * r2, q1 = p45 + p67 * r2, q2 = p89 + pab * r2;
    const double o0 = q0 + q1 * r4, o1 = q2 + pcd * r4;
    const double p = o0 + o1 * r8;
    if (k > 1023) return (p * 2.0) * pow2i(k - 1);
    if (k < -1021) return (p * pow2i(k + 600)) * pow2i(-600);
    return p * pow2i(k);
}

GAM_HD double gam_exp(double x) { return exp_ab(x, 0.0); }

GAM_HD double gam_erfc(double x) {
    const double ax = fabs(x);
    double res;
    if (ax > 27.5) {
        res = 0.0;
    } else {
        const double q = 1.0 / (ax + GAM_ERFC_L);
        const double s = (GAM_ERFC_A * ax - GAM_ERFC_B) * q;
        // g(s) by Estrin's scheme (dependency depth 6 instead of 22)
        const double s2 = s * s, s4 = s2 * s2, s8 = s4 * s4, s16 = s8 * s8;
        const double a0 = GAM_ERFC_G0 + GAM_ERFC_G1 * s, a1 = GAM_ERFC_G2 + GAM_ERFC_G3 * s;
        const double a2 = GAM_ERFC_G4 + GAM_ERFC_G5 * s, a3 = GAM_ERFC_G6 + GAM_ERFC_G7 * s;
        const double a4 = GAM_ERFC_G8 + GAM_ERFC_G9 * s, a5 = GAM_ERFC_G10 + GAM_ERFC_G11 * s;
        const double a6 = GAM_ERFC_G12 + GAM_ERFC_G13 * s, a7 = GAM_ERFC_G14 + GAM_ERFC_G15 * s;
        const double a8 = GAM_ERFC_G16 + GAM_ERFC_G17 * s, a9 = GAM_ERFC_G18 + GAM_ERFC_G19 * s;
        const double a10 = GAM_ERFC_G20 + GAM_ERFC_G21 * s;
        const double b0 = a0 + a1 * s2, b1 = a2 + a3 * s2, b2 = a4 + a5 * s2, b3 = a6 + a7 * s2;
        const double b4 = a8 + a9 * s2, b5 = a10 + GAM_ERFC_G22 * s2;
        const double c0 = b0 + b1 * s4, c1 = b2 + b3 * s4, c2 = b4 + b5 * s4;
        const double d0 = c0 + c1 * s8;
        const double g = d0 + c2 * s16;
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
