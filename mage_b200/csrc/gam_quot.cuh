// IEEE quotients a/d for several numerators that share one divisor, equal to
// the correctly rounded a/d bit for bit, at a fraction of the cost of one
// full division per numerator. Usable from host and device code.
//
// Method (Markstein's correction of a faithful quotient; P. Markstein,
// "Computation of elementary functions on the IBM RISC System/6000 processor",
// IBM J. Res. Develop. 34(1), 1990; stated as the division theorem of
// J.-M. Muller et al., "Handbook of Floating-Point Arithmetic", ch. 4: if y is
// within half an ulp of 1/d and q within one ulp of a/d, then r = a - d*q is
// exact and RN(q + r*y) = RN(a/d), in binary arithmetic without underflow or
// overflow):
//
//   per divisor   yh = RN(1/d)                   (one IEEE division)
//                 yl = RN(RN(1 - d*yh) * yh)     (1 - d*yh by one fma)
//   per numerator q0 = RN(a*yh + RN(a*yl))       (one fma)
//                 r  = RN(a - d*q0)              (one fma, exact)
//                 q  = RN(q0 + r*yh)             (one fma) = RN(a/d)
//
// yh + yl equals 1/d to a relative 2^-104, so the exact sum that q0 rounds is
// a/d to a relative 2^-103 and q0 is within half an ulp plus 2^-51 ulp of a/d:
// faithful. yh = RN(1/d) by construction; Markstein's theorem then makes q the
// correctly rounded quotient. The theorem needs every intermediate in the
// normal range: |d| and |a| in [2^-450, 2^450) keep q, r (about |a| 2^-53)
// and yl (about 2^-53/|d|) normal. Outside that range (and for NaN, infinity
// or subnormal operands) the plain IEEE division is taken. A zero numerator
// takes the fast path and gets its sign from a*yh (the sign of a/d), since a
// sum of two zeros of different signs would otherwise round to +0.
//
// Checked against IEEE division on 1e9 random operand pairs over the whole
// exponent range and on quotients next to rounding midpoints
// (tests/test_quot_host.py compiles this header for the host), and bit for
// bit by the GPU parity tests of the strict step.
#pragma once

#include <math.h>
#include <stdint.h>
#include <string.h>

#if defined(__CUDACC__)
#define GAMQ_HD __host__ __device__ __forceinline__
#else
#define GAMQ_HD inline
#endif

namespace gam {

// 2^-450 <= |x| < 2^450, from the biased exponent in the high word
GAMQ_HD bool quot_in_range(double x) {
#if defined(__CUDA_ARCH__)
    const unsigned h = (unsigned)__double2hiint(x) & 0x7fffffffu;
#else
    uint64_t u;
    memcpy(&u, &x, sizeof u);
    const unsigned h = (unsigned)(u >> 32) & 0x7fffffffu;
#endif
    return h - ((1023u - 450u) << 20) < (900u << 20);
}

struct QuotExact {
    double d, yh, yl;
    bool dok;
    GAMQ_HD explicit QuotExact(double dd) : d(dd) {
        yh = 1.0 / dd;
        yl = fma(-dd, yh, 1.0) * yh;
        dok = quot_in_range(dd);
    }
    GAMQ_HD double operator()(double a) const {
        if (dok && (a == 0.0 || quot_in_range(a))) {
            const double q0 = fma(a, yh, a * yl);
            const double r = fma(-d, q0, a);
            const double q = fma(r, yh, q0);
            return a == 0.0 ? a * yh : q;
        }
        return a / d;
    }
};

}  // namespace gam
