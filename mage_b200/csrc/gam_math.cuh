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
//     a tail (k*ln2_hi exact), e^r from its Taylor series to degree 13, exact
//     scaling by 2^k. The split argument lets erfc pass -x^2 as an exact head
//     plus a small tail.
//   gam_erfc(x) = exp(-x^2) * g(s) / (x + 4), s = (A x - B)/(x + 4) for x >= 0,
//     g a degree-22 Chebyshev fit of erfcx(x)*(x+4) on [0, 27.5];
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
    double p = GAM_EXP_C13;
    p = p * r + GAM_EXP_C12;
    p = p * r + GAM_EXP_C11;
    p = p * r + GAM_EXP_C10;
    p = p * r + GAM_EXP_C9;
    p = p * r + GAM_EXP_C8;
    p = p * r + GAM_EXP_C7;
    p = p * r + GAM_EXP_C6;
    p = p * r + GAM_EXP_C5;
    p = p * r + GAM_EXP_C4;
    p = p * r + GAM_EXP_C3;
    p = p * r + GAM_EXP_C2;
    p = p * r + GAM_EXP_C1;
    p = p * r + GAM_EXP_C0;
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
        double g = GAM_ERFC_G22;
        g = g * s + GAM_ERFC_G21;
        g = g * s + GAM_ERFC_G20;
        g = g * s + GAM_ERFC_G19;
        g = g * s + GAM_ERFC_G18;
        g = g * s + GAM_ERFC_G17;
        g = g * s + GAM_ERFC_G16;
        g = g * s + GAM_ERFC_G15;
        g = g * s + GAM_ERFC_G14;
        g = g * s + GAM_ERFC_G13;
        g = g * s + GAM_ERFC_G12;
        g = g * s + GAM_ERFC_G11;
        g = g * s + GAM_ERFC_G10;
        g = g * s + GAM_ERFC_G9;
        g = g * s + GAM_ERFC_G8;
        g = g * s + GAM_ERFC_G7;
        g = g * s + GAM_ERFC_G6;
        g = g * s + GAM_ERFC_G5;
        g = g * s + GAM_ERFC_G4;
        g = g * s + GAM_ERFC_G3;
        g = g * s + GAM_ERFC_G2;
        g = g * s + GAM_ERFC_G1;
        g = g * s + GAM_ERFC_G0;
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
