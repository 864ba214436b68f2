// Kernels of one GAMERA MHD time step on sm_100a.
//
// This header is compiled twice (gam_step_strict.cu without FMA contraction,
// gam_step_fast.cu with it) inside the namespace named by GAM_NS, and each
// kernel is templated on the real type R of the bulk data (double for the
// drop-in form, float for the precision form; scalars, the dt reduction and
// the totals stay double).
//
// Step = stepGamera (gamapp.F90:73-91):
//   k_step_begin     AdvanceMHD time trap, AB2 spacing      (mhdgroup.F90:25-31, 457)
//   k_predict        Predictor/PredictCell/ExtrapAB2 + bFlux2Fld of the
//                    half state; per-cell primitives of both states and
//                    per-face B = flux/area, computed once for all stencils
//                                                           (mhdgroup.F90:444-615)
//   k_mom2face(eD)   Mom2Face                               (fields.F90:235-285)
//   k_vxb(eD)        GetCornerV/D/B, EdgeLRs, edge EMF      (fields.F90:184-228, 288-517)
//   k_stress(d)      Fluxes: recon + PDM, MagKinFlux, GasKinFlux, HOGS
//                                                           (stress.F90:204-599, recon.F90)
//   k_update_faces   E2Flux on the new buffer               (fields.F90:18-51)
//   k_update_cells   Flux2Deltas, CellReynolds, bFlux2Fld, CellMaxwell, and the
//                    per-cell CFL dt with a block min       (stress.F90:148-194,
//                    mhdgroup.F90:79-329, gridutils.F90:49-106)
//   k_dt_finalize    time bookkeeping + CalcDT checks       (gamapp.F90:110-111, step.F90:58-168)
//   k_bc_periodic    EnforceBCs (periodic / none) fused with bFlux2Fld of
//                    the cells whose faces changed          (bcs.F90:279-450, gamapp.F90:86-88)
//
// Every expression keeps the reference's evaluation order (Fortran a+b+c is
// (a+b)+c, x**2.0 is x*x, dot_product is a sequential sum from 0), so the
// strict build reproduces an IEEE-strict CPU step bit for bit.
#pragma once

#include <algorithm>
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include <stdint.h>
#include <type_traits>
#include "gam_layout.cuh"
#include "gam_math.cuh"
#include "gam_quot.cuh"
#include "gam_types.cuh"

#ifndef GAM_NS
#error "GAM_NS must name the namespace of this build"
#endif
#ifndef GAM_STRICT_KERNELS
#define GAM_STRICT_KERNELS 0  // 1: the strict build (launch bounds measured for it)
#endif

namespace GAM_NS {

static constexpr double TINY = 1.0e-12;
static constexpr double HUGE_DT = 1.0e12;
static constexpr double PI_D = 3.141592653589793;
static constexpr double SQRT_PI_D = 1.7724538509055159;  // sqrt(pi) rounded to double

// interpolation weights (recon.F90:22-23, 28-29)
__device__ __forceinline__ double w8(int n) {
    switch (n) {
        case 0: return -3.0 / 840.0;
        case 1: return 29.0 / 840.0;
        case 2: return -139.0 / 840.0;
        case 3: return 533.0 / 840.0;
        case 4: return 533.0 / 840.0;
        case 5: return -139.0 / 840.0;
        case 6: return 29.0 / 840.0;
        default: return -3.0 / 840.0;
    }
}
__device__ __forceinline__ double up7c(int n) {
    switch (n) {
        case 0: return -3.0 / 420.0;
        case 1: return 25.0 / 420.0;
        case 2: return -101.0 / 420.0;
        case 3: return 319.0 / 420.0;
        case 4: return 214.0 / 420.0;
        case 5: return -38.0 / 420.0;
        default: return 4.0 / 420.0;
    }
}

template <class R> __device__ __forceinline__ R Rc(double x) { return (R)x; }

template <class R> struct Mth;
template <> struct Mth<double> {
#ifdef GAM_CUDA_MATH
    // product build: CUDA's erfc/exp (a few ulp, like libm's, and cheaper)
    static __device__ __forceinline__ double erfc_(double x) { return erfc(x); }
    static __device__ __forceinline__ double exp_(double x) { return exp(x); }
#else
    // strict build: the self-written erfc/exp shared with the CPU restatement
    static __device__ __forceinline__ double erfc_(double x) { return gam::gam_erfc(x); }
    static __device__ __forceinline__ double exp_(double x) { return gam::gam_exp(x); }
#endif
    static __device__ __forceinline__ double sqrt_(double x) { return sqrt(x); }
    static __device__ __forceinline__ double rsqrt_(double x) { return rsqrt(x); }
};
template <> struct Mth<float> {
    static __device__ __forceinline__ float erfc_(float x) { return erfcf(x); }
    static __device__ __forceinline__ float exp_(float x) { return expf(x); }
    static __device__ __forceinline__ float sqrt_(float x) { return sqrtf(x); }
    static __device__ __forceinline__ float rsqrt_(float x) { return rsqrtf(x); }
};

// Quotients a/d that share the divisor d. The FMA form (GAM_FAST_RECIP)
// takes one reciprocal and multiplies (at most one ulp more than the division,
// and a fraction of its instructions). Every other build returns the IEEE
// quotient bit for bit: FP64 through gam::QuotExact (one division per divisor,
// three fmas and a multiply per numerator), FP32 by plain division.
// Quot1 is the same for a divisor with a single numerator, where QuotExact
// would cost more than the division it replaces.
template <class R> struct Quot {
#ifdef GAM_FAST_RECIP
    R r;
    __device__ __forceinline__ explicit Quot(R d) : r((R)1 / d) {}
    __device__ __forceinline__ R operator()(R a) const { return a * r; }
#else
    R d;
    __device__ __forceinline__ explicit Quot(R dd) : d(dd) {}
    __device__ __forceinline__ R operator()(R a) const { return a / d; }
#endif
};
#ifndef GAM_FAST_RECIP
template <> struct Quot<double> {
    gam::QuotExact q;
    __device__ __forceinline__ explicit Quot(double d) : q(d) {}
    __device__ __forceinline__ double operator()(double a) const { return q(a); }
};
#endif
// a/d for a finite nonzero divisor d, equal to the IEEE quotient. A zero
// numerator returns a*d (the signed zero of a/d) without entering the
// division, whose IEEE routine leaves its fast path for a zero numerator;
// zero numerators are common in the step (velocities and field components
// that are exactly zero over much of a grid).
template <class R> __device__ __forceinline__ R qdiv(R a, R d) { return a == (R)0 ? a * d : a / d; }
template <class R> struct Quot1 {
#ifdef GAM_FAST_RECIP
    R r;
    __device__ __forceinline__ explicit Quot1(R d) : r((R)1 / d) {}
    __device__ __forceinline__ R operator()(R a) const { return a * r; }
#else
    R d;
    __device__ __forceinline__ explicit Quot1(R dd) : d(dd) {}
    __device__ __forceinline__ R operator()(R a) const { return qdiv(a, d); }
#endif
};

// std::max / std::min semantics: max(a,b) = (a < b) ? b : a, min(a,b) = (b < a) ? b : a
template <class R> __device__ __forceinline__ R rmax(R a, R b) { return (a < b) ? b : a; }
template <class R> __device__ __forceinline__ R rmin(R a, R b) { return (b < a) ? b : a; }
template <class R> __device__ __forceinline__ R sgn1(R b) { return copysign((R)1, b); }

__device__ __forceinline__ bool thread_ijk(const Range& r, int& ii, int& jj, int& kk) {
    ii = r.i0 + blockIdx.x * blockDim.x + threadIdx.x;
    jj = r.j0 + blockIdx.y * blockDim.y + threadIdx.y;
    kk = r.k0 + blockIdx.z * blockDim.z + threadIdx.z;
    return ii <= r.i1 && jj <= r.j1 && kk <= r.k1;
}

__device__ __forceinline__ long lidx(const GamBox& b, int ii, int jj, int kk) {
    return (long)ii + (long)b.sx * jj + b.sk * kk;
}
__device__ __forceinline__ long dstride(const GamBox& b, int d) { return d == 0 ? 1L : (d == 1 ? (long)b.sx : b.sk); }

// ----------------------------------------------------------------- recon
// pdmLR (recon.F90:231-272) on a 4-point limiter stencil nq[0..3] = cells -2..1
template <class R>
__device__ __forceinline__ void pdm_lr(R pdmb, const R* v, R Qi, R& Ql, R& Qr) {
    R v0 = v[0], v1 = v[1], v2 = v[2], v3 = v[3];
    R maxV = rmax(v1, v2), minV = rmin(v1, v2);
    R vN = rmax(minV, rmin(Qi, maxV));
    R dv0 = pdmb * (v1 - v0), dv1 = pdmb * (v2 - v1), dv2 = pdmb * (v3 - v2);
    R s0 = sgn1(dv0), s1 = sgn1(dv1), s2 = sgn1(dv2);
    R q0 = fabs(s0 + s1), q1 = fabs(s1 + s2);
    R dvL = vN - v1, dvR = v2 - vN;
    Ql = vN - s1 * rmax((R)0, fabs(dvL) - q0 * fabs(dv0));
    Qr = vN + s1 * rmax((R)0, fabs(dvR) - q1 * fabs(dv2));
}
// PDM (recon.F90:275-301)
template <class R>
__device__ __forceinline__ R pdm1(R pdmb, R q0, R q1, R q2, R qI) {
    R maxQ = rmax(q1, q2), minQ = rmin(q1, q2);
    R qN = rmax(minQ, rmin(qI, maxQ));
    R dq0 = pdmb * (q1 - q0), dq1 = pdmb * (q2 - q1);
    R s0 = sgn1(dq0), s1 = sgn1(dq1);
    R s01 = fabs(s0 + s1);
    R dqL = qN - q1;
    return qN - s1 * rmax((R)0, fabs(dqL) - s01 * fabs(dq0));
}
template <class R> __device__ __forceinline__ R central8(const R* q) {
    R s = (R)0;
#pragma unroll
    for (int n = 0; n < 8; n++) s += Rc<R>(w8(n)) * q[n];
    return s;
}
// GetLRs = Cen8LRs (recon.F90:125-158) or Up7LRs (:162-198) on the volume
// weighted stencil QdV[0..7] = dV*Q at cells -4..3 (precomputed per cell),
// limiter nq[0..3] at cells -2..1, and the volume interpolant Vi.
template <class R, class Q>
__device__ __forceinline__ void lrs_from_qdv(const DevParams<R>& P, const R* QdV, const R* nq, const Q& Vi, R& Ql,
                                             R& Qr) {
    if (!P.up7) {
        R s = (R)0;
#pragma unroll
        for (int n = 0; n < 8; n++) s += Rc<R>(w8(n)) * QdV[n];
        R Qi = Vi(s);
        pdm_lr(P.pdmb, nq, Qi, Ql, Qr);
    } else {
        R a = QdV[0] * Rc<R>(up7c(0));
#pragma unroll
        for (int n = 1; n < 7; n++) a = a + QdV[n] * Rc<R>(up7c(n));
        R b = QdV[7] * Rc<R>(up7c(0));
#pragma unroll
        for (int n = 1; n < 7; n++) b = b + QdV[7 - n] * Rc<R>(up7c(n));
        Ql = Vi(a);
        Qr = Vi(b);
        Ql = pdm1(P.pdmb, nq[0], nq[1], nq[2], Ql);
        Qr = pdm1(P.pdmb, nq[3], nq[2], nq[1], Qr);
    }
}

// ----------------------------------------------------------------- EOS
// BlockCon2Prim (recon.F90:62-91)
template <class R>
__device__ __forceinline__ void block_c2p(const DevParams<R>& P, const R* U, R* W) {
    R D = rmax(U[0], P.dFloor);
    const Quot<R> qD(D);
    R Mx = U[1], My = U[2], Mz = U[3], E = U[4];
    R KinE = qD((R)0.5 * (Mx * Mx + My * My + Mz * Mz));
    R Pr = rmax(P.gm1 * (E - KinE), P.pFloor);
    W[0] = D;
    W[1] = qD(Mx);
    W[2] = qD(My);
    W[3] = qD(Mz);
    W[4] = Pr;
}
// CellC2P (gamutils.F90:301-321)
template <class R>
__device__ __forceinline__ void cell_c2p(const DevParams<R>& P, const R* U, R* W) {
    R rho = U[0];
    const Quot<R> qr(rho);
    R Vx = qr(U[1]), Vy = qr(U[2]), Vz = qr(U[3]);
    R E = U[4];
    R KinE = (R)0.5 * rho * (Vx * Vx + Vy * Vy + Vz * Vz);
    W[0] = rmax(rho, P.dFloor);
    W[1] = Vx;
    W[2] = Vy;
    W[3] = Vz;
    W[4] = rmax(P.gm1 * (E - KinE), P.pFloor);
}
// CellP2C (gamutils.F90:362-383)
template <class R>
__device__ __forceinline__ void cell_p2c(const DevParams<R>& P, const R* W, R* U) {
    R rho = rmax(W[0], P.dFloor);
    R Vx = W[1], Vy = W[2], Vz = W[3];
    R IntE = rmax(W[4], P.pFloor) / P.gm1;
    R KinE = (R)0.5 * rho * (Vx * Vx + Vy * Vy + Vz * Vz);
    U[0] = rho;
    U[1] = rho * Vx;
    U[2] = rho * Vy;
    U[3] = rho * Vz;
    U[4] = IntE + KinE;
}

// norm2 as gfortran evaluates it (scaled sum of squares)
__device__ __forceinline__ double norm2s3(const double* a) {
    double scale = 1.0, res = 0.0;
#pragma unroll
    for (int q = 0; q < 3; q++) {
        if (a[q] != 0.0) {
            double ax = fabs(a[q]);
            if (scale < ax) {
                double val = scale / ax;
                res = 1.0 + res * val * val;
                scale = ax;
            } else {
                double val = ax / scale;
                res += val * val;
            }
        }
    }
    return scale * sqrt(res);
}
// sqrt(2.0) of the nuclear option's interface speed (stress.F90:405): a
// default-real constant in the reference, which gfortran folds to this float
#define GAM_SQRT2_R4 ((double)1.41421354f)

// PredictCell (mhdgroup.F90:528-562, AB2, single fluid): the half-step
// conserved state from State n (Q) and n-1 (oQ)
template <class R>
__device__ __forceinline__ void predict_cell(const DevParams<R>& P, const R* Q, const R* oQ, R pdt, const Quot<R>& odt,
                                             R* pQ) {
    R W[5], oW[5], pW[5];
    cell_c2p(P, oQ, oW);
    cell_c2p(P, Q, W);
#pragma unroll
    for (int v = 0; v < 5; v++) {
        R dQ = odt(W[v] - oW[v]);
        pW[v] = W[v] + pdt * dQ;
    }
    pW[0] = rmax(pW[0], P.dFloor);
    pW[4] = rmax(pW[4], P.pFloor);
    cell_p2c(P, pW, pQ);
}

// ExtrapAB3 (mhdgroup.F90:721-731)
template <class R> __device__ __forceinline__ R extrap_ab3(R dt, R Q, R oQ, R ooQ, R odt, R oodt) {
    R dQ = qdiv(Q - oQ, odt);
    R odQ = qdiv(oQ - ooQ, oodt);
    R tScl = (dt + odt) / (odt + oodt);
    return Q + dt * dQ + dt * tScl * (dQ - odQ);
}
// PredictCell with doAB3: the third level of the gas is oState's
// (ooQ = oState%Gas, mhdgroup.F90:500-502), as in the reference
template <class R>
__device__ __forceinline__ void predict_cell_ab3(const DevParams<R>& P, const R* Q, const R* oQ, R pdt, R odt, R oodt,
                                                 R* pQ) {
    R W[5], oW[5], ooW[5], pW[5];
    cell_c2p(P, oQ, oW);
    cell_c2p(P, Q, W);
    cell_c2p(P, oQ, ooW);
#pragma unroll
    for (int v = 0; v < 5; v++) pW[v] = extrap_ab3(pdt, W[v], oW[v], ooW[v], odt, oodt);
    pW[0] = rmax(pW[0], P.dFloor);
    pW[4] = rmax(pW[4], P.pFloor);
    cell_p2c(P, pW, pQ);
}

// Boris-limited speed Ca v / sqrt(Ca^2 + v^2) (fields.F90:211-213,
// gridutils.F90:91-93, gamutils.F90:356-358)
template <class T> __device__ __forceinline__ T boris_speed(T Ca, T v) { return Ca * v / sqrt(Ca * Ca + v * v); }

// gamCellBxyz (gridutils.F90:648-680) from the six face fluxes of cell c,
// with the quotient by the cell volume qV
template <class R>
__device__ __forceinline__ void cell_bxyz(const GamBox& b, const Geo<R>& g, long c, R fI, R fIp, R fJ, R fJp, R fK,
                                          R fKp, const Quot<R>& qV, R* B) {
    const long fs = b.fs;
    if constexpr (std::is_same<R, float>::value) {
        // sum of flux x (face centroid - cell centroid): the same value as the
        // form below, without the cancellation of absolute coordinates
#pragma unroll
        for (int x = 0; x < 3; x++) {
            const R* d = g.dxf + (long)x * fs + c;
            R t = fIp * d[3 * fs] + fJp * d[9 * fs] + fKp * d[15 * fs] - fI * d[0] - fJ * d[6 * fs] - fK * d[12 * fs];
            B[x] = qV(t);
        }
        return;
    }
    R Div = fIp - fI + fJp - fJ + fKp - fK;
#pragma unroll
    for (int x = 0; x < 3; x++) {
        R xfI = g.xfc[(x + 0) * fs + c];
        R xfJ = g.xfc[(x + 3) * fs + c];
        R xfK = g.xfc[(x + 6) * fs + c];
        R xfIp = g.xfc[(x + 0) * fs + c + 1];
        R xfJp = g.xfc[(x + 3) * fs + c + b.sx];
        R xfKp = g.xfc[(x + 6) * fs + c + b.sk];
        R t = qV(fIp * xfIp + fJp * xfJp + fKp * xfKp - fI * xfI - fJ * xfJ - fK * xfK);
        B[x] = t - qV(Div * g.xyzcc[x * fs + c]);
    }
}
template <class R>
__device__ __forceinline__ void cell_bxyz(const GamBox& b, const Geo<R>& g, long c, R fI, R fIp, R fJ, R fJp, R fK,
                                          R fKp, R* B) {
    cell_bxyz(b, g, c, fI, fIp, fJ, fJp, fK, fKp, Quot<R>(g.vol[c]), B);
}

// ----------------------------------------------------------------- bounds checks
// Built with -DGAM_BOUNDS_CHECK (libgamgpu_check.so): every kernel checks the
// lowest and highest linear box index its stencils will touch before loading
// anything; a failed check records the kernel and the index in the scalars
// and the thread returns without touching memory (no trap). The host reads
// the record after the call. Without the macro the checks compile to nothing.
#ifdef GAM_BOUNDS_CHECK
__device__ __forceinline__ bool box_ok(const GamBox& b, long lo, long hi, const GamScalars* csc, int kid) {
    GamScalars* sc = const_cast<GamScalars*>(csc);
    const long lim = sc->oobLimit > 0 ? (long)sc->oobLimit : b.nbox;
    if (lo >= 0 && hi < lim) return true;
    if (atomicExch(&sc->oob, 1) == 0) {
        sc->oobKernel = kid;
        sc->oobIndex = lo < 0 ? lo : hi;
    }
    return false;
}
#define GAM_BOX_CHECK(lo, hi, kid) \
    if (!box_ok(b, (long)(lo), (long)(hi), sc, (kid))) return
// for kernels whose threads must reach a later barrier: a value, not a return
#define GAM_BOX_OK(lo, hi, kid) box_ok(b, (long)(lo), (long)(hi), sc, (kid))
#else
#define GAM_BOX_OK(lo, hi, kid) true
#define GAM_BOX_CHECK(lo, hi, kid) \
    do {                           \
    } while (0)
#endif

// ----------------------------------------------------------------- LFM pole
// Index maps across the LFM axis (ringutils.F90:482-659, box indices): the
// pole at js (doS) / je+1 (doE), k shifted by half a ring (WrapK).
__device__ __forceinline__ int ring_wrapk(const GamBox& b, int kk) {
    int kp = kk + b.Nkp / 2;
    if (kp > GAM_NG + b.Nkp - 1) kp -= b.Nkp;
    return kp;
}
// lfmIJKcc for a ghost row across the pole: its conjugate cell (true) or
// nothing (false)
__device__ __forceinline__ bool ring_conj_cc(const GamBox& b, const RingData& Rg, int& jj, int& kk) {
    const int G = GAM_NG;
    if (Rg.doS && jj < G) {
        jj = 2 * G - 1 - jj;
        kk = ring_wrapk(b, kk);
        return true;
    }
    if (Rg.doE && jj > G + b.Njp - 1 && jj <= G + b.Njp + 3) {
        jj = 2 * G + 2 * b.Njp - 1 - jj;
        kk = ring_wrapk(b, kk);
        return true;
    }
    return false;
}
// The pole boundary lfmIn / lfmOut (bcs.F90:1019-1106) as a map of value
// comp (-1 cell, 0..2 face normal) at (jj, kk): the source and its sign
// (J and K faces reversed); the J faces' pole face itself is not mirrored
__device__ __forceinline__ int ring_bc_jmap(const GamBox& b, const RingData& Rg, int comp, int& jj, int& kk) {
    const int G = GAM_NG, N = b.Njp;
    if (comp == 1) {
        if (Rg.doS && jj < G) {
            jj = 2 * G - jj;
            kk = ring_wrapk(b, kk);
            return -1;
        }
        if (Rg.doE && jj >= G + N + 1 && jj <= G + N + 4) {
            jj = 2 * G + 2 * N - jj;
            kk = ring_wrapk(b, kk);
            return -1;
        }
        return 1;
    }
    if (ring_conj_cc(b, Rg, jj, kk)) return comp == 2 ? -1 : 1;
    return 1;
}

// ----------------------------------------------------------------- kernels
// AdvanceMHD entry: time trap and AB2 spacing (mhdgroup.F90:25-31, 457)
__global__ void k_step_begin(GamScalars* sc) {
    if (sc->halted) return;
    if (fabs(sc->otime - sc->time) < TINY) sc->otime = sc->time - sc->dt;
    sc->odt = sc->time - sc->otime;
    sc->oodt = sc->otime - sc->ootime;  // Predictor (mhdgroup.F90:459-463), used with doAB3
    sc->pdt = 0.5 * sc->dt;
}

// Predictor over every face and cell of the ghosted box. Besides the half
// state it stores the operands every later stencil uses, each computed once:
// volume * primitive (the recon operand QdV of Cen8LRs/Up7LRs), the limiter
// primitives, volume * momentum / density (Mom2Face), and per face
// area * flux/max(area,TINY) and flux/max(area,TINY) (EdgeLRs), flux/area (Fluxes).
template <class R, int MINB, bool AB3 = false>
__global__ void __launch_bounds__(256, MINB) k_predict(GamBox b, DevParams<R> P, Geo<R> g, StateBuf<R> cur,
                                                 StateBuf<R> old, Work<R> w, const GamScalars* sc,
                                                 const R* __restrict__ oomf) {
    if (sc->halted) return;
    int ii, jj, kk;
    Range r{0, b.Ni, 0, b.Nj, 0, b.Nk};
    if (!thread_ijk(r, ii, jj, kk)) return;
    const long fs = b.fs;
    const long c = lidx(b, ii, jj, kk);
    const R pdt = (R)sc->pdt, odt = (R)sc->odt;
    const bool isCell = ii < b.Ni && jj < b.Nj && kk < b.Nk;
    GAM_BOX_CHECK(c, isCell ? c + b.sk : c, 1);
    // The state and work pointers may alias as far as the compiler knows, so
    // every state load is issued before the first store.
    R fQ[3], foQ[3], fA[3], Q[5], oQ[5], uQ[3], uoQ[3];
    R fooQ[3], uooQ[3];  // AB3: ooState fluxes of the lower / upper faces
    if (P.doMHD) {
#pragma unroll
        for (int d = 0; d < 3; d++) {
            fQ[d] = cur.mf[d * fs + c];
            foQ[d] = old.mf[d * fs + c];
            fA[d] = g.face[d * fs + c];
            if constexpr (AB3) fooQ[d] = oomf[d * fs + c];
        }
    }
    if (isCell) {
#pragma unroll
        for (int v = 0; v < 5; v++) {
            Q[v] = cur.Gas[v * fs + c];
            oQ[v] = old.Gas[v * fs + c];
        }
        if (P.doMHD) {
            const long off[3] = {1, (long)b.sx, b.sk};
#pragma unroll
            for (int d = 0; d < 3; d++) {
                uQ[d] = cur.mf[d * fs + c + off[d]];
                uoQ[d] = old.mf[d * fs + c + off[d]];
                if constexpr (AB3) uooQ[d] = oomf[d * fs + c + off[d]];
            }
        }
    }
    R hm[3];
    const Quot<R> qodt(odt);
    [[maybe_unused]] R oodt = (R)0;
    if constexpr (AB3) oodt = (R)sc->oodt;
    if (P.doMHD) {
#pragma unroll
        for (int d = 0; d < 3; d++) {
            if constexpr (AB3) {
                hm[d] = extrap_ab3(pdt, fQ[d], foQ[d], fooQ[d], odt, oodt);
            } else {
                R dQ = qodt(fQ[d] - foQ[d]);
                hm[d] = fQ[d] + pdt * dQ;  // ExtrapAB2
            }
            R A = fA[d];
            R Am = rmax(A, (R)TINY);
            const Quot<R> qAm(Am);
            R bh = qAm(hm[d]);
            w.abh[d * fs + c] = A * bh;
            w.Bnf[d * fs + c] = qdiv(hm[d], A);
            w.bn[d * fs + c] = P.doLFMLim ? qAm(fQ[d]) : bh;
        }
    }
    if (!isCell) return;
    R pQ[5];
    if constexpr (AB3)
        predict_cell_ab3(P, Q, oQ, pdt, odt, oodt, pQ);
    else
        predict_cell(P, Q, oQ, pdt, qodt, pQ);
    R Wh[5], Wn[5];
    block_c2p(P, pQ, Wh);
    if (P.doLFMLim) block_c2p(P, Q, Wn);
    const R vol = g.vol[c];
#pragma unroll
    for (int v = 0; v < 5; v++) {
        w.QW[v * fs + c] = vol * Wh[v];
        w.Wn[v * fs + c] = P.doLFMLim ? Wn[v] : Wh[v];
    }
    w.Dh[c] = Wh[0];
    const R Dm = rmax(pQ[0], P.dFloor);
    const Quot<R> qDm(Dm);
#pragma unroll
    for (int x = 0; x < 3; x++) w.VdV[x * fs + c] = qDm(vol * pQ[1 + x]);
    if (P.doMHD) {
        // upper faces of this cell, recomputed with the same ExtrapAB2
        R up[3];
#pragma unroll
        for (int d = 0; d < 3; d++) {
            if constexpr (AB3) {
                up[d] = extrap_ab3(pdt, uQ[d], uoQ[d], uooQ[d], odt, oodt);
            } else {
                R dQ = qodt(uQ[d] - uoQ[d]);
                up[d] = uQ[d] + pdt * dQ;
            }
        }
        R B[3];
        int jc = jj, kc = kk;
        if (P.ring.on && ring_conj_cc(b, P.ring, jc, kc)) {
            // RingFlux2FieldFix in the predictor's bFlux2Fld: the conjugate
            // cell's field from its own extrapolated fluxes
            const long cc = lidx(b, ii, jc, kc);
            const long off[3] = {1, (long)b.sx, b.sk};
            R lo[3], hi[3];
#pragma unroll
            for (int d = 0; d < 3; d++) {
                const long f0 = d * fs + cc, f1 = f0 + off[d];
                if constexpr (AB3) {
                    lo[d] = extrap_ab3(pdt, cur.mf[f0], old.mf[f0], oomf[f0], odt, oodt);
                    hi[d] = extrap_ab3(pdt, cur.mf[f1], old.mf[f1], oomf[f1], odt, oodt);
                } else {
                    lo[d] = cur.mf[f0] + pdt * qodt(cur.mf[f0] - old.mf[f0]);
                    hi[d] = cur.mf[f1] + pdt * qodt(cur.mf[f1] - old.mf[f1]);
                }
            }
            cell_bxyz(b, g, cc, lo[0], hi[0], lo[1], hi[1], lo[2], hi[2], B);
        } else {
            cell_bxyz(b, g, c, hm[0], up[0], hm[1], up[1], hm[2], up[2], B);
        }
#pragma unroll
        for (int x = 0; x < 3; x++) {
            w.QB[x * fs + c] = vol * B[x];
            if (!P.doLFMLim) w.Bl[x * fs + c] = B[x];
        }
    }
}

// Edge geometry of the EMF in direction eD (fields.F90:84-170): face
// direction dT1 (Mom2Face sweep), dT2 (corner sweep)
__device__ __forceinline__ void edge_dirs(int eD, int& dT1, int& dT2) {
    dT1 = (eD + 1) % 3;
    dT2 = (eD + 2) % 3;
}

// Mom2Face for edge direction eD over the reference's loop range; stores
// area(dT1) * Vf, the operand of GetCornerV's weighted interpolation.
template <class R>
__global__ void __launch_bounds__(256) k_mom2face(GamBox b, DevParams<R> P, Geo<R> g, Work<R> w, int eD, Range r,
                                                  const GamScalars* sc) {
    if (sc->halted) return;
    int ii, jj, kk;
    if (!thread_ijk(r, ii, jj, kk)) return;
    int dT1, dT2;
    edge_dirs(eD, dT1, dT2);
    const long fs = b.fs;
    const long c = lidx(b, ii, jj, kk);
    const long s = dstride(b, dT1);
    GAM_BOX_CHECK(c - 4 * s, c + 3 * s, 2 + 2 * eD);
    R vol[8];
#pragma unroll
    for (int n = 0; n < 8; n++) vol[n] = g.vol[c + (n - 4) * s];
    R dV = rmax(central8(vol), (R)TINY);
    const Quot<R> qdV(dV);
    const R A = g.face[dT1 * fs + c];
    R out[3];
#pragma unroll
    for (int x = 0; x < 3; x++) {
        R q[8];
#pragma unroll
        for (int n = 0; n < 8; n++) q[n] = w.VdV[x * fs + c + (n - 4) * s];
        out[x] = A * qdV(central8(q));
    }
#pragma unroll
    for (int x = 0; x < 3; x++) w.AVf[(x + 3 * eD) * fs + c] = out[x];
}

// EdgeLRs (fields.F90:288-362): flux of faces of direction a, stencil along b
template <class R>
__device__ __forceinline__ void edge_lrs(const GamBox& b, const DevParams<R>& P, const Geo<R>& g, const Work<R>& w,
                                         long c, int a, int bd, R* area, R& bL, R& bR, R& fA) {
    const long fs = b.fs;
    const long s = dstride(b, bd);
    R qdv[8], nmag[4];
#pragma unroll
    for (int n = 0; n < 8; n++) {
        area[n] = g.face[a * fs + c + (n - 4) * s];
        qdv[n] = w.abh[a * fs + c + (n - 4) * s];
    }
#pragma unroll
    for (int m = 0; m < 4; m++) nmag[m] = w.bn[a * fs + c + (m - 2) * s];
    const R Vi = central8(area);
    if (P.up7)
        lrs_from_qdv(P, qdv, nmag, Quot<R>(Vi), bL, bR);
    else
        lrs_from_qdv(P, qdv, nmag, Quot1<R>(Vi), bL, bR);
    fA = Vi;  // dot_product(interpWgt, AreaB) again: the same value
    bL = bL * fA;
    bR = bR * fA;
}

// VxB edge loop for direction eD (fields.F90:184-228). SAVE (the
// differentiation form's forward) also stores the corner values in w.esv.
template <class R, int MINB = 1, bool SAVE = false>
__global__ void __launch_bounds__(128, MINB) k_vxb(GamBox b, DevParams<R> P, Geo<R> g, Work<R> w, int eD, Range r,
                                             const GamScalars* sc) {
    if (sc->halted) return;
    int ii, jj, kk;
    if (!thread_ijk(r, ii, jj, kk)) return;
    int dT1, dT2;
    edge_dirs(eD, dT1, dT2);
    const long fs = b.fs;
    const long c = lidx(b, ii, jj, kk);
    // GetCornerD (fields.F90:427-454): normal-plane unit offsets e1 < e2
    const int e1 = eD == 0 ? 1 : 0, e2 = eD == 2 ? 1 : 2;
    const long s1 = dstride(b, e1), s2 = dstride(b, e2);
    {
        const long sA = dstride(b, dT1), sB = dstride(b, dT2), sM = sA > sB ? sA : sB;
        [[maybe_unused]] const long lo = c - s1 - s2 < c - 4 * sM ? c - s1 - s2 : c - 4 * sM;
        GAM_BOX_CHECK(lo, c + 3 * sM, 3 + 2 * eD);
    }
    R Dc = (R)0.25 * (w.Dh[c] + w.Dh[c - s1] + w.Dh[c - s2] + w.Dh[c - s1 - s2]);
    // GetCornerB: EdgeLRs for dT1 faces along dT2 and dT2 faces along dT1
    R area1[8], area2[8];
    R bT1L, bT1R, fA1, bT2L, bT2R, fA2;
    edge_lrs(b, P, g, w, c, dT1, dT2, area1, bT1L, bT1R, fA1);
    edge_lrs(b, P, g, w, c, dT2, dT1, area2, bT2L, bT2R, fA2);
    // GetCornerV (fields.F90:457-517); its area stencil equals area1
    R dA = rmax(fA1, (R)TINY);
    const Quot<R> qdA(dA);
    R VC[3];
    const long s2v = dstride(b, dT2);
#pragma unroll
    for (int x = 0; x < 3; x++) {
        R acc = (R)0;
#pragma unroll
        for (int n = 0; n < 8; n++) acc += Rc<R>(w8(n)) * w.AVf[(x + 3 * eD) * fs + c + (n - 4) * s2v];
        VC[x] = qdA(acc);
    }
    const R* Te = g.Te;
    R v1 = VC[0] * Te[(3 + 9 * eD) * fs + c] + VC[1] * Te[(4 + 9 * eD) * fs + c] + VC[2] * Te[(5 + 9 * eD) * fs + c];
    R v2 = VC[0] * Te[(6 + 9 * eD) * fs + c] + VC[1] * Te[(7 + 9 * eD) * fs + c] + VC[2] * Te[(8 + 9 * eD) * fs + c];
    R vDiff = Mth<R>::sqrt_(v1 * v1 + v2 * v2);
    R xni = g.Teb[(0 + 4 * eD) * fs + c], yni = g.Teb[(1 + 4 * eD) * fs + c];
    R xnj = g.Teb[(2 + 4 * eD) * fs + c], ynj = g.Teb[(3 + 4 * eD) * fs + c];
    R detT = (R)1 / (xni * ynj - xnj * yni);
    const Quot<R> qA1(fA1), qA2(fA2);
    R bT1 = qA1((R)0.5 * (bT1L + bT1R));
    R bT2 = qA2((R)0.5 * (bT2L + bT2R));
    R db1 = qA1(bT1R - bT1L);
    R db2 = qA2(bT2R - bT2L);
    R Jd = db2 - db1;
    R b1 = detT * (ynj * bT1 - yni * bT2);
    R b2 = detT * (-(xnj * bT1) + xni * bT2);
    if (P.doBackground) {
        b1 = b1 + (R)g.edgB0[(0 + 2 * eD) * fs + c];
        b2 = b2 + (R)g.edgB0[(1 + 2 * eD) * fs + c];
    }
    R vA = qdiv(Mth<R>::sqrt_(b1 * b1 + b2 * b2), Mth<R>::sqrt_(Dc));
    if (P.doBoris) vA = boris_speed((R)P.Ca, vA);
    vDiff = vDiff + vA;
    const R edge = g.edge[eD * fs + c];
    vDiff = rmin(vDiff, P.CFL * edge / (R)sc->dt);
    R e = -(v1 * b2 - v2 * b1) + P.Vd0 * vDiff * Jd;
    w.E[eD * fs + c] = e * edge;
    if constexpr (SAVE) {
        R* o = w.esv + (long)(GAM_ESV_NC * eD) * fs + c;
        o[0] = Dc;
        o[fs] = bT1L;
        o[2 * fs] = bT1R;
        o[3 * fs] = fA1;
        o[4 * fs] = bT2L;
        o[5 * fs] = bT2R;
        o[6 * fs] = fA2;
#pragma unroll
        for (int x = 0; x < 3; x++) o[(7 + x) * fs] = VC[x];
    }
}

// One-sided Gaussian-moment fluxes for one side q (sgn = -1 LEFT, +1 RIGHT).
// MagKinFlux (stress.F90:513-599).
template <class R, bool BORIS = false>
__device__ __forceinline__ void mag_kin_flux(const DevParams<R>& P, R sgn, const R* W, const R* Bm, R Bn,
                                             const R* T, const double* B0, double B0n, R* mF, R& bbD, R& VaD) {
    R D = W[0], Pr = W[4];
    const Quot<R> qD(D);
    R Bx = Bm[0], By = Bm[1], Bz = Bm[2];
    R dPb = (R)0.5 * (Bx * Bx + By * By + Bz * Bz);
    R Va2;
    R B0x = (R)0, B0y = (R)0, B0z = (R)0;
    if (P.doBackground) {
        B0x = (R)B0[0]; B0y = (R)B0[1]; B0z = (R)B0[2];
        R sx = Bx + B0x, sy = By + B0y, sz = Bz + B0z;
        Va2 = qD(sx * sx + sy * sy + sz * sz);
        bbD = bbD + (R)0.5 * (sx * sx + sy * sy + sz * sz);
    } else {
        Va2 = qD((R)2 * dPb);
        bbD = bbD + (R)0.5 * (Bx * Bx + By * By + Bz * Bz);
    }
    R Vac2 = Va2;
    if constexpr (BORIS) {  // Boris-corrected Va^2
        const R Ca = (R)P.Ca;
        Vac2 = Va2 / ((R)1 + (Va2 / (Ca * Ca)));
    }
    R Nx = T[0], Ny = T[1], Nz = T[2];
    R Vn = Nx * W[1] + Ny * W[2] + Nz * W[3];
#ifdef GAM_FAST_RECIP
    // sqrt(1/x) as one reciprocal square root (about one ulp)
    const R sqlam = Mth<R>::rsqrt_(qD((R)2 * Pr) + Vac2);
#else
    R lambda = (R)1 / (qD((R)2 * Pr) + Vac2);
    const R sqlam = Mth<R>::sqrt_(lambda);
#endif
    R Vn0 = (R)0.5 * Mth<R>::erfc_(sgn * sqlam * Vn);
    VaD = VaD + (R)0.5 * Mth<R>::sqrt_(Vac2);
    mF[0] = mF[0] + Vn0 * (dPb * Nx - Bx * Bn);
    mF[1] = mF[1] + Vn0 * (dPb * Ny - By * Bn);
    mF[2] = mF[2] + Vn0 * (dPb * Nz - Bz * Bn);
    if (P.doBackground) {
        R B0nR = (R)B0n;
        R BdB0 = B0x * Bx + B0y * By + B0z * Bz;
        mF[0] = mF[0] + Vn0 * (-(B0x * Bn) - Bx * B0nR + BdB0 * Nx);
        mF[1] = mF[1] + Vn0 * (-(B0y * Bn) - By * B0nR + BdB0 * Ny);
        mF[2] = mF[2] + Vn0 * (-(B0z * Bn) - Bz * B0nR + BdB0 * Nz);
    }
}
// GasKinFlux (stress.F90:432-511)
template <class R>
__device__ __forceinline__ void gas_kin_flux(const DevParams<R>& P, R sgn, const R* W, const R* T, R* gF, R* dW) {
    R D = W[0], Pr = W[4], Vx = W[1], Vy = W[2], Vz = W[3];
    R E = (R)0.5 * D * (Vx * Vx + Vy * Vy + Vz * Vz) + Pr / P.gm1;
    R lambda = D / ((R)2 * Pr);
    R Vn = T[0] * Vx + T[1] * Vy + T[2] * Vz;
    R Vt1 = T[3] * Vx + T[4] * Vy + T[5] * Vz;
    R Vt2 = T[6] * Vx + T[7] * Vy + T[8] * Vz;
    const R sqlam = Mth<R>::sqrt_(lambda);
    R Vn0 = (R)0.5 * Mth<R>::erfc_(sgn * sqlam * Vn);
#ifdef GAM_FAST_RECIP
    // sqrt(pi lambda) = sqrt(pi) sqrt(lambda): one square root instead of two
    R Vn1 = Vn * Vn0 - qdiv((R)0.5 * sgn * Mth<R>::exp_(-(lambda * Vn * Vn)), (R)SQRT_PI_D * sqlam);
#else
    R Vn1 = Vn * Vn0 - qdiv((R)0.5 * sgn * Mth<R>::exp_(-(lambda * Vn * Vn)), Mth<R>::sqrt_((R)PI_D * lambda));
#endif
    gF[0] = gF[0] + D * Vn1;
    gF[4] = gF[4] + (E + (R)0.5 * Pr) * Vn1 + (R)0.5 * Pr * Vn0 * Vn;
    R fMn = D * Vn * Vn1 + Pr * Vn0;
    R fMt1 = D * Vt1 * Vn1;
    R fMt2 = D * Vt2 * Vn1;
    R fMx = T[0] * fMn + T[3] * fMt1 + T[6] * fMt2;
    R fMy = T[1] * fMn + T[4] * fMt1 + T[7] * fMt2;
    R fMz = T[2] * fMn + T[5] * fMt1 + T[8] * fMt2;
    gF[1] = gF[1] + fMx;
    gF[2] = gF[2] + fMy;
    gF[3] = gF[3] + fMz;
    dW[0] = dW[0] + sgn * D;
    dW[1] = dW[1] + sgn * D * Vx;
    dW[2] = dW[2] + sgn * D * Vy;
    dW[3] = dW[3] + sgn * D * Vz;
    dW[4] = dW[4] + sgn * E;
}

// Face fluxes of direction D (Fluxes, stress.F90:204-429), one face per
// thread. The stencil operands are the per-cell products volume*primitive and
// volume*B of the half state (QdV of Cen8LRs) and the limiter values, read
// along D through L1; MINB bounds the registers for occupancy. SAVE (the
// differentiation form's forward) also stores the face states in w.fsv.
template <class R, int D, int MINB, bool BORIS = false, bool SAVE = false>
__global__ void __launch_bounds__(128, MINB) k_stress(GamBox b, DevParams<R> P, Geo<R> g, const R* __restrict__ Blim,
                                                      Work<R> w, Range r, const GamScalars* sc,
                                                      const R* __restrict__ gasN, const R* __restrict__ gasO) {
    if (sc->halted) return;
    int ii, jj, kk;
    if (!thread_ijk(r, ii, jj, kk)) return;
    const long fs = b.fs;
    const long c = lidx(b, ii, jj, kk);
    const long s = D == 0 ? 1L : (D == 1 ? (long)b.sx : b.sk);
    GAM_BOX_CHECK(c - 4 * s, c + 3 * s, 8 + D);
    R T[9];
#pragma unroll
    for (int n = 0; n < 9; n++) T[n] = g.Tf[(n + 9 * D) * fs + c];
    const R fa = g.face[D * fs + c];
    R vol[8];
#pragma unroll
    for (int n = 0; n < 8; n++) vol[n] = g.vol[c + (n - 4) * s];
    const Quot<R> Vi(central8(vol));
    R MagL[3] = {(R)0, (R)0, (R)0}, MagR[3] = {(R)0, (R)0, (R)0};
    R Bn = (R)0;
    double B0[3] = {0.0, 0.0, 0.0}, B0n = 0.0;
    if (P.doMHD) {
        Bn = w.Bnf[D * fs + c];
#pragma unroll
        for (int x = 0; x < 3; x++) {
            R q[8], nq[4];
            const R* qp = w.QB + x * fs + c - 4 * s;
            const R* lp = Blim + x * fs + c - 2 * s;
#pragma unroll
            for (int n = 0; n < 8; n++) q[n] = qp[n * s];
#pragma unroll
            for (int m = 0; m < 4; m++) nq[m] = lp[m * s];
            lrs_from_qdv(P, q, nq, Vi, MagL[x], MagR[x]);
        }
        if (P.doBackground) {
#pragma unroll
            for (int x = 0; x < 3; x++) B0[x] = g.fcB0[(x + 3 * D) * fs + c];
            B0n = qdiv(g.bFlux0[D * fs + c], (double)fa);
        }
    }
    R WL[5], WR[5];
#pragma unroll
    for (int v = 0; v < 5; v++) {
        R q[8], nq[4];
        const R* qp = w.QW + v * fs + c - 4 * s;
        const R* lp = w.Wn + v * fs + c - 2 * s;
#pragma unroll
        for (int n = 0; n < 8; n++) q[n] = qp[n * s];
#pragma unroll
        for (int m = 0; m < 4; m++) nq[m] = lp[m * s];
        lrs_from_qdv(P, q, nq, Vi, WL[v], WR[v]);
    }
    R VaD = (R)0, bbD = (R)0;
    if (P.doMHD) {
        R mF[3] = {(R)0, (R)0, (R)0};
        mag_kin_flux<R, BORIS>(P, (R)-1, WL, MagL, Bn, T, B0, B0n, mF, bbD, VaD);
        mag_kin_flux<R, BORIS>(P, (R)1, WR, MagR, Bn, T, B0, B0n, mF, bbD, VaD);
        if constexpr (BORIS) {  // Boris hogs on the magnetic fluxes (stress.F90:335-349)
            const R Ca = (R)P.Ca;
#pragma unroll
            for (int x = 0; x < 3; x++) {
                R deeV = WR[1 + x] - WL[1 + x];
                R deeP = qdiv(bbD * deeV, Ca * Ca);
                mF[x] = mF[x] - P.cHogM * VaD * deeP;
            }
        }
#pragma unroll
        for (int x = 0; x < 3; x++) w.mF[(x + 3 * D) * fs + c] = fa * mF[x];
    }
    R gF[5] = {(R)0, (R)0, (R)0, (R)0, (R)0}, dW[5] = {(R)0, (R)0, (R)0, (R)0, (R)0};
    gas_kin_flux(P, (R)-1, WL, T, gF, dW);
    gas_kin_flux(P, (R)1, WR, T, gF, dW);
    R gv[5];
#pragma unroll
    for (int v = 0; v < 5; v++) gv[v] = gF[v] - (R)1 * P.cHogH * VaD * dW[v];
    if constexpr (BORIS) {
        // the nuclear option (stress.F90:399-417, cLim = 1.5): where the mean
        // interface speed reaches cLim Ca, diffuse with speed Ca on the jump of
        // the half-step conserved state between the face's two cells, which is
        // recomputed here (the predictor keeps primitives only)
        double vl[3] = {(double)WL[1], (double)WL[2], (double)WL[3]}, vr[3] = {(double)WR[1], (double)WR[2], (double)WR[3]};
        const R vL = (R)norm2s3(vl), vR = (R)norm2s3(vr);
        const R Vn = Mth<R>::sqrt_(vL * vL + vR * vR) / (R)GAM_SQRT2_R4;
        const R Ca = (R)P.Ca;
        if (Vn >= (R)1.5 * Ca) {
            R Ql[5], oQl[5], Qr[5], oQr[5], pQl[5], pQr[5];
#pragma unroll
            for (int v = 0; v < 5; v++) {
                Ql[v] = gasN[v * fs + c - s];
                oQl[v] = gasO[v * fs + c - s];
                Qr[v] = gasN[v * fs + c];
                oQr[v] = gasO[v * fs + c];
            }
            const R pdt = (R)sc->pdt, odt = (R)sc->odt;
            if (P.doAB3) {
                const R oodt = (R)sc->oodt;
                predict_cell_ab3(P, Ql, oQl, pdt, odt, oodt, pQl);
                predict_cell_ab3(P, Qr, oQr, pdt, odt, oodt, pQr);
            } else {
                const Quot<R> qodt(odt);
                predict_cell(P, Ql, oQl, pdt, qodt, pQl);
                predict_cell(P, Qr, oQr, pdt, qodt, pQr);
            }
#pragma unroll
            for (int v = 0; v < 5; v++) gv[v] = gv[v] - Ca * (pQr[v] - pQl[v]);
        }
    }
#pragma unroll
    for (int v = 0; v < 5; v++) w.gF[(v + 5 * D) * fs + c] = fa * gv[v];
    if constexpr (SAVE) {
        R* o = w.fsv + (long)(GAM_FSV_NC * D) * fs + c;
#pragma unroll
        for (int v = 0; v < 5; v++) {
            o[v * fs] = WL[v];
            o[(5 + v) * fs] = WR[v];
            o[(17 + v) * fs] = dW[v];
        }
#pragma unroll
        for (int x = 0; x < 3; x++) {
            o[(10 + x) * fs] = MagL[x];
            o[(13 + x) * fs] = MagR[x];
        }
        o[16 * fs] = VaD;
    }
}

// E2Flux into the new buffer; faces outside its range are copied. With
// doAB3 the buffer's old content (oState, n-1) first moves to ooState
// (CopyState(oState, ooState), mhdgroup.F90:100-102).
template <class R>
__global__ void __launch_bounds__(256) k_update_faces(GamBox b, DevParams<R> P, StateBuf<R> cur, StateBuf<R> nxt,
                                                      Work<R> w, const GamScalars* sc, R* __restrict__ oomf) {
    if (sc->halted) return;
    int ii, jj, kk;
    Range r{0, b.Ni, 0, b.Nj, 0, b.Nk};
    if (!thread_ijk(r, ii, jj, kk)) return;
    const long fs = b.fs;
    const long c = lidx(b, ii, jj, kk);
    const int G = GAM_NG;
    {
        const bool inr0 = P.doMHD && ii >= G && ii <= G + b.Nip && jj >= G && jj <= G + b.Njp && kk >= G &&
                          kk <= G + b.Nkp;
        GAM_BOX_CHECK(c, inr0 ? c + b.sk : c, 11);
    }
    if (oomf) {
#pragma unroll
        for (int x = 0; x < 3; x++) oomf[x * fs + c] = nxt.mf[x * fs + c];
    }
    const bool inr = P.doMHD && ii >= G && ii <= G + b.Nip && jj >= G && jj <= G + b.Njp && kk >= G && kk <= G + b.Nkp;
    if (!inr) {
#pragma unroll
        for (int x = 0; x < 3; x++) nxt.mf[x * fs + c] = cur.mf[x * fs + c];
        return;
    }
    const R* E = w.E;
    const long sj = b.sx, sk = b.sk;
    const R dt = (R)sc->dt;
    R dfi = E[2 * fs + c + sj] - E[2 * fs + c] - E[1 * fs + c + sk] + E[1 * fs + c];
    R dfj = E[0 * fs + c + sk] - E[0 * fs + c] - E[2 * fs + c + 1] + E[2 * fs + c];
    R dfk = E[1 * fs + c + 1] - E[1 * fs + c] - E[0 * fs + c + sj] + E[0 * fs + c];
    nxt.mf[0 * fs + c] = cur.mf[0 * fs + c] - dt * dfi;
    nxt.mf[1 * fs + c] = cur.mf[1 * fs + c] - dt * dfj;
    nxt.mf[2 * fs + c] = cur.mf[2 * fs + c] - dt * dfk;
}

__device__ __forceinline__ unsigned long long dbits(double x) { return (unsigned long long)__double_as_longlong(x); }

// CellDT (gridutils.F90:49-106), evaluated in FP64
template <class R, bool BORIS>
__device__ __forceinline__ double cell_dt(const DevParams<R>& P, const double* U, const double* Bt, double dl,
                                          double gamma, double gm1, double CFL) {
    double rho = U[0];
    const Quot<double> qr(rho);
    double Vx = qr(U[1]), Vy = qr(U[2]), Vz = qr(U[3]);
    double MagV = sqrt(Vx * Vx + Vy * Vy + Vz * Vz);
    double ke = 0.5 * rho * (MagV * MagV);
    double e = U[4] - ke;
    double Pr = gm1 * e;
    double Cs = sqrt(gamma * Pr / rho);
    double Valf = 0.0;
    if (P.doMHD) {
        double MagB = sqrt(Bt[0] * Bt[0] + Bt[1] * Bt[1] + Bt[2] * Bt[2]);
        Valf = qdiv(MagB, sqrt(rho));
        if constexpr (BORIS) Valf = boris_speed(P.Ca, Valf);
    }
    double vCFL = MagV + sqrt(Cs * Cs + Valf * Valf) + 0.0;
    return CFL * dl / vCFL;
}

// CellBoris (mhdgroup.F90:334-382, single fluid): U2 the hydro-updated state
// (in place), U0 State n, B2 and B0 the total fields at n+1 and n
template <class R>
__device__ __forceinline__ void cell_boris(const DevParams<R>& P, R* U2, const R* U0, const R* B2, const R* B0,
                                           const R* dGasH, const R* dGasM, R Ca, R dt) {
    R W2[5];
    cell_c2p(P, U2, W2);
    const R D2 = rmax(W2[0], P.dFloor);
    const R P2 = rmax(W2[4], P.pFloor);
    const R D0 = rmax(U0[0], P.dFloor);
    R V0[3], B1[3], dPGas[3], dPMag[3], bhat1[3], dMom[3];
#pragma unroll
    for (int x = 0; x < 3; x++) {
        V0[x] = qdiv(U0[1 + x], D0);
        B1[x] = (R)0.5 * (B2[x] + B0[x]);
    }
    const R alpha = (B1[0] * B1[0] + B1[1] * B1[1] + B1[2] * B1[2]) / (D2 * Ca * Ca);
    const R dRho = dt * dGasH[0];
#pragma unroll
    for (int x = 0; x < 3; x++) {
        dPGas[x] = dt * dGasH[1 + x];
        dPMag[x] = dt * dGasM[x];
    }
    const R pCon = (R)1 / ((R)1 + alpha);
    // normVec (math.F90:332-343)
    const R nA = Mth<R>::sqrt_(B1[0] * B1[0] + B1[1] * B1[1] + B1[2] * B1[2]);
#pragma unroll
    for (int x = 0; x < 3; x++) bhat1[x] = nA <= (R)TINY ? (R)0 : B1[x] / nA;
    if (alpha > (R)TINY) {
        R sum[3];
#pragma unroll
        for (int x = 0; x < 3; x++) sum[x] = dPGas[x] + dPMag[x];
        const R pg = dPGas[0] * bhat1[0] + dPGas[1] * bhat1[1] + dPGas[2] * bhat1[2];
        const R ps = sum[0] * bhat1[0] + sum[1] * bhat1[1] + sum[2] * bhat1[2];
        const R pv = V0[0] * bhat1[0] + V0[1] * bhat1[1] + V0[2] * bhat1[2];
#pragma unroll
        for (int x = 0; x < 3; x++)
            dMom[x] = pg * bhat1[x] + pCon * (sum[x] - ps * bhat1[x]) + alpha * pCon * dRho * (V0[x] - pv * bhat1[x]);
    } else {
#pragma unroll
        for (int x = 0; x < 3; x++) dMom[x] = dPGas[x] + dPMag[x];
    }
    W2[0] = D2;
#pragma unroll
    for (int x = 0; x < 3; x++) W2[1 + x] = (D0 * V0[x] + dMom[x]) / D2;
    W2[4] = P2;
    cell_p2c(P, W2, U2);
}

// Flux2Deltas + CellReynolds + bFlux2Fld + CellMaxwell for active cells,
// copy + bFlux2Fld for ghost cells, then the CFL dt of cells in the dt range.
template <class R, int MINB, bool BORIS = false>
__global__ void __launch_bounds__(128, MINB) k_update_cells(GamBox b, DevParams<R> P, Geo<R> g, StateBuf<R> cur,
                                                      StateBuf<R> nxt, Work<R> w, GamScalars* sc, double gamma_d,
                                                      double gm1_d) {
    __shared__ double smin[32];
    if (sc->halted) return;
    int ii, jj, kk;
    Range r{0, b.Ni - 1, 0, b.Nj - 1, 0, b.Nk - 1};
    bool ok = thread_ijk(r, ii, jj, kk);
    ok = ok && GAM_BOX_OK(lidx(b, ii, jj, kk), lidx(b, ii, jj, kk) + b.sk, 12);
    double mydt = HUGE_DT;
    bool bad = false;
    if (ok) {
        const long fs = b.fs;
        const long c = lidx(b, ii, jj, kk);
        const int G = GAM_NG;
        const bool active = ii >= G && ii < G + b.Nip && jj >= G && jj < G + b.Njp && kk >= G && kk < G + b.Nkp;
        const R dt = (R)sc->dt;
        R U[5];
        R Bc[3] = {(R)0, (R)0, (R)0};
        // bFlux2Fld and Flux2Deltas divide by the same cell volume
        const Quot<R> qdV(g.vol[c]);
        if (P.doMHD) {
            const long sj = b.sx, sk = b.sk;
            int jc = jj, kc = kk;
            // RingFlux2FieldFix: a cell across the pole takes its conjugate's
            // field (the same volume, so the same quotient)
            const long cb = (P.ring.on && ring_conj_cc(b, P.ring, jc, kc)) ? lidx(b, ii, jc, kc) : c;
            cell_bxyz(b, g, cb, nxt.mf[cb], nxt.mf[cb + 1], nxt.mf[fs + cb], nxt.mf[fs + cb + sj], nxt.mf[2 * fs + cb],
                      nxt.mf[2 * fs + cb + sk], qdV, Bc);
        }
        if (active) {
            const long sj = b.sx, sk = b.sk;
            R dGasH[5];
#pragma unroll
            for (int v = 0; v < 5; v++) {
                const R* gI = w.gF + (v + 0) * fs;
                const R* gJ = w.gF + (v + 5) * fs;
                const R* gK = w.gF + (v + 10) * fs;
                dGasH[v] = qdV(gI[c] - gI[c + 1] + gJ[c] - gJ[c + sj] + gK[c] - gK[c + sk]);
                U[v] = cur.Gas[v * fs + c] + dt * dGasH[v];
            }
            if (P.doMHD) {
                R dGasM[3];
#pragma unroll
                for (int x = 0; x < 3; x++) {
                    const R* mI = w.mF + (x + 0) * fs;
                    const R* mJ = w.mF + (x + 3) * fs;
                    const R* mK = w.mF + (x + 6) * fs;
                    dGasM[x] = qdV(mI[c] - mI[c + 1] + mJ[c] - mJ[c + sj] + mK[c] - mK[c + sk]);
                    if (P.doBackground) dGasM[x] = dGasM[x] + (R)g.dpB0[x * fs + c];
                }
                if constexpr (BORIS) {
                    R U0[5], B2[3], B0[3];
#pragma unroll
                    for (int v = 0; v < 5; v++) U0[v] = cur.Gas[v * fs + c];
#pragma unroll
                    for (int x = 0; x < 3; x++) {
                        B2[x] = Bc[x];
                        B0[x] = cur.B[x * fs + c];
                        if (P.doBackground) {
                            const R b0 = (R)g.B0[x * fs + c];
                            B2[x] = B2[x] + b0;
                            B0[x] = B0[x] + b0;
                        }
                    }
                    cell_boris(P, U, U0, B2, B0, dGasH, dGasM, (R)P.Ca, dt);
                } else {
                // CellMaxwell (mhdgroup.F90:299-329)
                R D = rmax(U[0], P.dFloor);
                const Quot<R> qD(D);
                R Mx = U[1], My = U[2], Mz = U[3], TotE = U[4];
                R KinE = qD((R)0.5 * (Mx * Mx + My * My + Mz * Mz));
                R Pr = rmax(P.gm1 * (TotE - KinE), P.pFloor);
                Mx = Mx + dt * dGasM[0];
                My = My + dt * dGasM[1];
                Mz = Mz + dt * dGasM[2];
                KinE = qD((R)0.5 * (Mx * Mx + My * My + Mz * Mz));
                U[0] = D;
                U[1] = Mx;
                U[2] = My;
                U[3] = Mz;
                U[4] = KinE + Pr / P.gm1;
                }
            }
        } else {
#pragma unroll
            for (int v = 0; v < 5; v++) U[v] = cur.Gas[v * fs + c];
        }
        // dt range isDT..ieDT = is-1..ie+1 (init.F90:511-530, single domain);
        // evaluated before the stores so that none of its loads waits on them
        // (PushIon and NudgeSW change the first shells and the last one after
        // the update: their dt is taken after them, by k_ion_push / k_nudge_sw)
        const bool indt = ii >= G - P.dtIlo && ii <= G + b.Nip - 1 + P.dtIhi && jj >= G - P.dtJlo &&
                          jj <= G + b.Njp - 1 + P.dtJhi && kk >= G - P.dtKlo &&
                          kk <= G + b.Nkp - 1 + P.dtKhi && !(P.ion.push && active && ii < G + P.ion.nIonP) &&
                          !(P.ion.wind && active && ii == G + b.Nip - 1);
        if (indt && !sc->fixedTimestep && !P.ring.on) {
            double Ud[5], Bt[3];
#pragma unroll
            for (int v = 0; v < 5; v++) Ud[v] = (double)U[v];
#pragma unroll
            for (int x = 0; x < 3; x++) {
                Bt[x] = (double)Bc[x];
                if (P.doBackground) Bt[x] = Bt[x] + g.B0[x * fs + c];
            }
            double dtc = cell_dt<R, BORIS>(P, Ud, Bt, (double)g.dl[c], gamma_d, gm1_d, sc->CFL);
            if (dtc > 0.0 && dtc < 1.0e300) mydt = dtc;  // finite positive
            else bad = true;
        }
#pragma unroll
        for (int v = 0; v < 5; v++) nxt.Gas[v * fs + c] = U[v];
        if (P.doMHD) {
#pragma unroll
            for (int x = 0; x < 3; x++) nxt.B[x * fs + c] = Bc[x];
        }
    }
    // block min
    for (int o = 16; o > 0; o >>= 1) mydt = fmin(mydt, __shfl_xor_sync(0xffffffffu, mydt, o));
    const int lane = (threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z)) & 31;
    const int wid = (threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z)) >> 5;
    const int nw = (blockDim.x * blockDim.y * blockDim.z + 31) >> 5;
    if (lane == 0) smin[wid] = mydt;
    unsigned anybad = __syncthreads_or(bad ? 1 : 0);
    if (wid == 0) {
        double v = lane < nw ? smin[lane] : HUGE_DT;
        for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (lane == 0) {
            if (v < HUGE_DT) atomicMin(&sc->dtmin_bits, dbits(v));
            if (anybad) atomicAdd(&sc->nbad, 1);
        }
    }
}

// ---- model hooks of the ionospheric boundary (bc[0] = 7; earthcmi.F90)
// HackE, first part: IonEFix (msphutils.F90:214-240), the J and K EMFs of
// the first shell i = is over jsg..jeg, ksg..keg from the coupling field
// (edge length x inEijk(5), formed on the host)
template <class R>
__global__ void __launch_bounds__(256) k_ion_efix(GamBox b, DevParams<R> P, Work<R> w, const GamScalars* sc) {
    if (sc->halted) return;
    const long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (q >= (long)b.Nj * b.Nk) return;
    const int jj = (int)(q % b.Nj), kk = (int)(q / b.Nj);
    const long c = lidx(b, GAM_NG, jj, kk);
    GAM_BOX_CHECK(c, c, 15);
    w.E[b.fs + c] = (R)P.ion.Ee[2 * q];
    w.E[2 * b.fs + c] = (R)P.ion.Ee[2 * q + 1];
}
// HackE, last part: FixEFieldLFM (gamdebug.F90:149-175), the I and J EMFs
// of k = ks and ke+1 set to their mean, i = is..ie+1, j = j0..j1 (js..je+1)
template <class R>
__global__ void __launch_bounds__(256) k_fix_e_lfm(GamBox b, R* __restrict__ E, int j0, int j1, const GamScalars* sc) {
    if (sc->halted) return;
    const int G = GAM_NG;
    const long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
    const int ni = b.Nip + 1;
    if (q >= (long)ni * (j1 - j0 + 1)) return;
    const int ii = G + (int)(q % ni), jj = j0 + (int)(q / ni);
    const long c0 = lidx(b, ii, jj, G), c1 = lidx(b, ii, jj, G + b.Nkp);
    GAM_BOX_CHECK(c0, c1, 15);
    const long fs = b.fs;
    const R Ei = (R)0.5 * (E[c0] + E[c1]);
    const R Ej = (R)0.5 * (E[fs + c0] + E[fs + c1]);
    E[c0] = Ei;
    E[c1] = Ei;
    E[fs + c0] = Ej;
    E[fs + c1] = Ej;
}
// HackStep: PushIon (earthcmi.F90:586-663) on the first nIonP active
// shells after the update, then CalcDT's CellDT of those cells (k_update_cells
// leaves them out) into the step's dt minimum
template <class R, bool BORIS>
__global__ void __launch_bounds__(128) k_ion_push(GamBox b, DevParams<R> P, Geo<R> g, StateBuf<R> nxt,
                                                  GamScalars* sc, double gamma_d, double gm1_d) {
    __shared__ double smin[32];
    if (sc->halted) return;
    const int G = GAM_NG;
    const long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
    const int np = P.ion.nIonP;
    double mydt = HUGE_DT;
    bool bad = false;
    if (q < (long)np * b.Njp * b.Nkp) {
        const int ii = G + (int)(q % np);
        const long r = q / np;
        const int jj = G + (int)(r % b.Njp), kk = G + (int)(r / b.Njp);
        const long fs = b.fs, c = lidx(b, ii, jj, kk);
        GAM_BOX_CHECK(c, c, 15);
        R U[5], W[5];
#pragma unroll
        for (int v = 0; v < 5; v++) U[v] = nxt.Gas[v * fs + c];
        if (!(U[0] < (R)0)) {  // RhoMin(BLK) = 0
            cell_c2p(P, U, W);
            const int dN = ii - G + 1;
            double f = sc->dt / ((double)dN * P.ion.dtCpl);
            f = (1.0 < f) ? 1.0 : f;  // min(dt, 1.0)
            const R fr = (R)f;
            const double* Vp = P.ion.Vp + 3 * q;
#pragma unroll
            for (int x = 0; x < 3; x++) {
                const R dV = (R)Vp[x] - W[1 + x];
                W[1 + x] = W[1 + x] + fr * dV;
            }
            cell_p2c(P, W, U);
#pragma unroll
            for (int v = 0; v < 5; v++) nxt.Gas[v * fs + c] = U[v];
        }
        if (!sc->fixedTimestep && !P.ring.on) {  // with rings, CalcDT runs after the ring average
            double Ud[5], Bt[3];
#pragma unroll
            for (int v = 0; v < 5; v++) Ud[v] = (double)U[v];
#pragma unroll
            for (int x = 0; x < 3; x++) {
                Bt[x] = (double)nxt.B[x * fs + c];
                if (P.doBackground) Bt[x] = Bt[x] + g.B0[x * fs + c];
            }
            const double dtc = cell_dt<R, BORIS>(P, Ud, Bt, (double)g.dl[c], gamma_d, gm1_d, sc->CFL);
            if (dtc > 0.0 && dtc < 1.0e300) mydt = dtc;
            else bad = true;
        }
    }
    for (int o = 16; o > 0; o >>= 1) mydt = fmin(mydt, __shfl_xor_sync(0xffffffffu, mydt, o));
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    if (lane == 0) smin[wid] = mydt;
    unsigned anybad = __syncthreads_or(bad ? 1 : 0);
    if (wid == 0) {
        double v = lane < nw ? smin[lane] : HUGE_DT;
        for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (lane == 0) {
            if (v < HUGE_DT) atomicMin(&sc->dtmin_bits, dbits(v));
            if (anybad) atomicAdd(&sc->nbad, 1);
        }
    }
}

// HackE, wind part: WindEFix (apps/wind.F90:489-566), the EMFs of shells
// ie-2..ie+1 blended with the wind's (weights and wind EMFs formed on the
// host), then DiffuseOuter (:570-616) on the outermost, from State n's fluxes
template <class R>
__global__ void __launch_bounds__(256) k_wind_efix(GamBox b, DevParams<R> P, Geo<R> g, StateBuf<R> S, Work<R> w,
                                                   const GamScalars* sc) {
    if (sc->halted) return;
    const int G = GAM_NG;
    const long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (q >= 4L * (b.Njp + 1) * (b.Nkp + 1)) return;
    const int sh = (int)(q & 3);
    const long r = q >> 2;
    const int jj = G + (int)(r % (b.Njp + 1)), kk = G + (int)(r / (b.Njp + 1));
    const int ii = G + b.Nip - 3 + sh;
    const long fs = b.fs, c = lidx(b, ii, jj, kk);
    GAM_BOX_CHECK(c - b.sk, c, 15);
    const double* t = P.ion.We + 7 * q;
    // CalcElecField starts every step from E = 0 (fields.F90:88): the edges it
    // does not compute (I edges at ie+1, J edges at je+1, K edges at ke+1) hold
    // zero when the wind blends into them; here they hold last step's blend
    const bool computed[3] = {ii < G + b.Nip, jj < G + b.Njp, kk < G + b.Nkp};
#pragma unroll
    for (int n = 0; n < 3; n++) {
        const R mhdE = computed[n] ? w.E[n * fs + c] : (R)0;
        if (t[n] >= 0.0) {
            const R wSW = (R)t[n];
            w.E[n * fs + c] = ((R)1 - wSW) * mhdE + wSW * (R)t[3 + n];
        } else {
            w.E[n * fs + c] = mhdE;
        }
    }
    if (sh != 3) return;
    const long sj = b.sx, sk = b.sk;
    const R* mf = S.mf;
    const R* fa = g.face;
    R bP = mf[fs + c] / rmax(fa[fs + c], (R)TINY);
    R bM = mf[fs + c - 1] / rmax(fa[fs + c - 1], (R)TINY);
    R db2 = bP - bM;
    bP = mf[c] / fa[c];
    bM = mf[c - sj] / fa[c - sj];
    R db1 = bP - bM;
    const R JdK = db2 - db1;
    bP = mf[c] / fa[c];
    bM = mf[c - sk] / fa[c - sk];
    db2 = bP - bM;
    bP = mf[2 * fs + c] / fa[2 * fs + c];
    bM = mf[2 * fs + c - 1] / fa[2 * fs + c - 1];
    db1 = bP - bM;
    const R JdJ = db2 - db1;
    const R dl = Mth<R>::sqrt_(g.edge[fs + c] * g.edge[2 * fs + c]);
    const R Vd = rmin((R)P.ion.vSW, P.CFL * dl / (R)sc->dt);
    const R Ed[3] = {(R)0, Vd * JdJ * dl, Vd * JdK * dl};
    const R wK = (R)t[6];
#pragma unroll
    for (int x = 0; x < 3; x++) w.E[x * fs + c] = w.E[x * fs + c] + wK * Ed[x];
}
// HackStep, wind part: NudgeSW (apps/wind.F90:394-486), the last active cell
// nudged towards the wind, then its CellDT into the step's dt minimum
template <class R, bool BORIS>
__global__ void __launch_bounds__(128) k_nudge_sw(GamBox b, DevParams<R> P, Geo<R> g, StateBuf<R> nxt,
                                                  GamScalars* sc, double gamma_d, double gm1_d) {
    __shared__ double smin[32];
    if (sc->halted) return;
    const int G = GAM_NG;
    const long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
    double mydt = HUGE_DT;
    bool bad = false;
    if (q < (long)b.Njp * b.Nkp) {
        const int jj = G + (int)(q % b.Njp), kk = G + (int)(q / b.Njp), ii = G + b.Nip - 1;
        const long fs = b.fs, c = lidx(b, ii, jj, kk);
        GAM_BOX_CHECK(c, c, 15);
        R U[5];
#pragma unroll
        for (int v = 0; v < 5; v++) U[v] = nxt.Gas[v * fs + c];
        const double wSW = P.ion.Wn[q];
        if (wSW > TINY) {
            const double a = P.ion.dtSW0 / wSW, dt = sc->dt;
            const double dtSW = (a < dt) ? dt : a;  // max(dtSW0 / wSW, dt)
            const R f = (R)(dt / dtSW);
            const double* ws = P.wind.state;
            const R gWs[5] = {(R)ws[0], (R)ws[2], (R)ws[3], (R)ws[4], (R)ws[1]};
            R gWm[5], gW[5];
            cell_c2p(P, U, gWm);
#pragma unroll
            for (int v = 0; v < 5; v++) gW[v] = gWm[v] + f * (gWs[v] - gWm[v]);
            cell_p2c(P, gW, U);
#pragma unroll
            for (int v = 0; v < 5; v++) nxt.Gas[v * fs + c] = U[v];
        }
        if (!sc->fixedTimestep && !P.ring.on) {  // with rings, CalcDT runs after the ring average
            double Ud[5], Bt[3];
#pragma unroll
            for (int v = 0; v < 5; v++) Ud[v] = (double)U[v];
#pragma unroll
            for (int x = 0; x < 3; x++) {
                Bt[x] = (double)nxt.B[x * fs + c];
                if (P.doBackground) Bt[x] = Bt[x] + g.B0[x * fs + c];
            }
            const double dtc = cell_dt<R, BORIS>(P, Ud, Bt, (double)g.dl[c], gamma_d, gm1_d, sc->CFL);
            if (dtc > 0.0 && dtc < 1.0e300) mydt = dtc;
            else bad = true;
        }
    }
    for (int o = 16; o > 0; o >>= 1) mydt = fmin(mydt, __shfl_xor_sync(0xffffffffu, mydt, o));
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    if (lane == 0) smin[wid] = mydt;
    unsigned anybad = __syncthreads_or(bad ? 1 : 0);
    if (wid == 0) {
        double v = lane < nw ? smin[lane] : HUGE_DT;
        for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (lane == 0) {
            if (v < HUGE_DT) atomicMin(&sc->dtmin_bits, dbits(v));
            if (anybad) atomicAdd(&sc->nbad, 1);
        }
    }
}


// ----------------------------------------------------------------- ring averaging
// Ring averaging about the LFM axis (ringav.F90, ringrecon.F90,
// ringutils.F90; gid "lfm" with the reference's defaults: no shift, no
// velocity cleaning, ring variables rho, momentum, internal energy). One
// thread per ring (pole, slice i, ring nR): the ring is the k circle of row
// js+nR-1 (S) or je-nR+1 (E); its work is sequential along k in the
// reference's order, so the bits match the CPU restatement.

// PoleE (ringav.F90:394-430) over slices i0..i1, or the same touch-up of
// WindEFix (apps/wind.F90:549-564): on each pole row the K EMFs zero and the
// I EMFs their mean over ks..ke, over the whole ghosted k range
// One warp per (pole, slice): the row is staged in shared memory by the
// lanes and summed by lane 0 in k order (the CPU code's sum).
template <class R> __device__ __forceinline__ R ring_row_mean(const R* __restrict__ f, long c0, long sk, int Np, R* row) {
    const int lane = threadIdx.x;
    for (int n = lane; n < Np; n += 32) row[n] = f[c0 + n * sk];
    __syncwarp();
    R sum = (R)0;
    if (lane == 0)
        for (int n = 0; n < Np; n++) sum = sum + row[n];
    sum = __shfl_sync(0xffffffffu, sum, 0);
    return sum / (R)Np;
}
template <class R>
__global__ void __launch_bounds__(32) k_ring_pole_e(GamBox b, RingData Rg, R* __restrict__ E, int i0, int i1,
                                                    const GamScalars* sc) {
    if (sc->halted) return;
    const int G = GAM_NG, ni = i1 - i0 + 1;
    const int pole = blockIdx.x / ni, ii = i0 + (int)(blockIdx.x % ni);
    if (!(pole == 0 ? Rg.doS : Rg.doE)) return;
    const int jp = pole == 0 ? G : G + b.Njp;
    const long fs = b.fs;
    if (!GAM_BOX_OK(lidx(b, ii, jp, 0), lidx(b, ii, jp, b.Nk - 1), 15)) return;
    extern __shared__ __align__(16) unsigned char ring_smem[];
    const R avg = ring_row_mean(E, lidx(b, ii, jp, G), b.sk, Rg.Np, (R*)ring_smem);
    for (int kk = threadIdx.x; kk < b.Nk; kk += 32) {
        const long c = lidx(b, ii, jp, kk);
        E[2 * fs + c] = (R)0;
        E[c] = avg;
    }
}

// RingFlux (ringutils.F90:662-678): no flux through the pole faces (every i,
// k), then FixGasFluxLFM (gamdebug.F90:91-124): the K fluxes of k = ks and
// ke+1 set to their mean, i = is..ie, j = js..je
template <class R>
__global__ void __launch_bounds__(256) k_ring_flux(GamBox b, DevParams<R> P, Work<R> w, const GamScalars* sc) {
    if (sc->halted) return;
    const int G = GAM_NG;
    const long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
    const long fs = b.fs;
    const long nz = (long)b.Ni * b.Nk;
    if (q < 2 * nz) {
        const int pole = (int)(q / nz);
        if (!(pole == 0 ? P.ring.doS : P.ring.doE)) return;
        const long r = q % nz;
        const int ii = (int)(r % b.Ni), kk = (int)(r / b.Ni);
        const long c = lidx(b, ii, pole == 0 ? G : G + b.Njp, kk);
        GAM_BOX_CHECK(c, c, 15);
#pragma unroll
        for (int v = 0; v < 5; v++) w.gF[(v + 5) * fs + c] = (R)0;
        if (P.doMHD) {
#pragma unroll
            for (int x = 0; x < 3; x++) w.mF[(x + 3) * fs + c] = (R)0;
        }
        return;
    }
    if (!P.doMHD) return;
    const long r = q - 2 * nz;
    if (r >= (long)b.Nip * b.Njp) return;
    const int ii = G + (int)(r % b.Nip), jj = G + (int)(r / b.Nip);
    const long c0 = lidx(b, ii, jj, G), c1 = lidx(b, ii, jj, G + b.Nkp);
    GAM_BOX_CHECK(c0, c1, 15);
#pragma unroll
    for (int v = 0; v < 5; v++) {
        R* gK = w.gF + (v + 10) * fs;
        const R gFa = (R)0.5 * (gK[c0] + gK[c1]);
        gK[c0] = gFa;
        gK[c1] = gFa;
    }
#pragma unroll
    for (int x = 0; x < 3; x++) {
        R* mK = w.mF + (x + 6) * fs;
        const R mFa = (R)0.5 * (mK[c0] + mK[c1]);
        mK[c0] = mFa;
        mK[c1] = mFa;
    }
}

// HackFlux = IonFlux (earthcmi.F90:357-404) on the inner tile with rings: the
// I fluxes of the first face ring at each pole (i = is, j = je then js) set
// to their ring mean, one thread per pole and component
template <class R> __global__ void __launch_bounds__(32) k_ion_flux(GamBox b, DevParams<R> P, Work<R> w,
                                                                      const GamScalars* sc) {
    if (sc->halted) return;
    const int G = GAM_NG;
    const int pole = blockIdx.x / 8, comp = blockIdx.x % 8;  // pole 0: E (je), 1: S (js); comp 0-4 gas, 5-7 magnetic
    if (!(pole == 0 ? P.ring.doE : P.ring.doS)) return;
    if (comp >= 5 && !P.doMHD) return;
    const int jr = pole == 0 ? G + b.Njp - 1 : G;
    R* f = comp < 5 ? w.gF + (long)comp * b.fs : w.mF + (long)(comp - 5) * b.fs;  // the I direction's components
    if (!GAM_BOX_OK(lidx(b, G, jr, G), lidx(b, G, jr, G + b.Nkp - 1), 15)) return;
    extern __shared__ __align__(16) unsigned char ring_smem[];
    const R avg = ring_row_mean(f, lidx(b, G, jr, G), b.sk, P.ring.Np, (R*)ring_smem);
    for (int kk = G + threadIdx.x; kk < G + b.Nkp; kk += 32) f[lidx(b, G, jr, kk)] = avg;
}

// the smoothing EMF rows each step starts from zero (InitRAVec): S rows
// js..js+NumR+1, E rows je-NumR..je+1, every i and k
template <class R> __global__ void __launch_bounds__(256) k_ring_zero_e(GamBox b, RingData Rg, const GamScalars* sc) {
    if (sc->halted) return;
    const int G = GAM_NG, nr = Rg.NumR + 2;
    const long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
    const long nrow = (long)b.Ni * b.Nk;
    if (q >= 2L * nr * nrow) return;
    const int pole = (int)(q / (nr * nrow));
    if (!(pole == 0 ? Rg.doS : Rg.doE)) return;
    const long r = q % (nr * nrow);
    const int row = (int)(r / nrow), ii = (int)(r % nrow % b.Ni), kk = (int)(r % nrow / b.Ni);
    const int jj = pole == 0 ? G + row : G + b.Njp - Rg.NumR - 1 + row;
    R* E = (R*)Rg.smoothE;
    const long c = lidx(b, ii, jj, kk), fs = b.fs;
#pragma unroll
    for (int x = 0; x < 3; x++) E[x * fs + c] = (R)0;
}

// minmod (math.F90:192-197): sign() as copysign, min() as a < b
template <class R> __device__ __forceinline__ R ring_min(R a, R b2) { return b2 < a ? b2 : a; }
template <class R> __device__ __forceinline__ R ring_minmod(R x, R y) {
    return (R)0.5 * (copysign((R)1, x) + copysign((R)1, y)) * ring_min(fabs(x), fabs(y));
}
// the interval L/R of a chunk (ringrecon.F90:224-285: PPM, PLM, PCM)
template <class R>
__device__ __forceinline__ void ring_lr(int recon, R fm2, R fm1, R f, R fp1, R fp2, R& vm, R& vp) {
    if (recon == 2) {
        vm = f;
        vp = f;
        return;
    }
    if (recon == 1) {
        const R dwL = f - fm1, dwR = fp1 - f, dwC = (fp1 - fm1) / (R)2;
        const R min1 = ring_min((R)2 * fabs(dwL), (R)2 * fabs(dwR));
        const R min2 = ring_min(min1, fabs(dwC));
        const R dwM = copysign(min2, dwC);
        vp = f + (R)0.5 * dwM;
        vm = f - (R)0.5 * dwM;
        return;
    }
    const R dvm2 = fm1 - fm2, dvm1 = f - fm1, dvp1 = fp1 - f, dvp2 = fp2 - fp1;
    R dvc = (R)0.5 * (dvm2 + dvm1), SM = (R)2 * ring_minmod(dvm2, dvm1);
    const R Sm1 = ring_minmod(dvc, SM);
    dvc = (R)0.5 * (dvm1 + dvp1);
    SM = (R)2 * ring_minmod(dvm1, dvp1);
    const R Sp1 = ring_minmod(dvc, SM);
    dvc = (R)0.5 * (dvp2 + dvp1);
    SM = (R)2 * ring_minmod(dvp2, dvp1);
    const R Sp2 = ring_minmod(dvc, SM);
    vp = (R)0.5 * (f + fp1) - (Sp2 - Sp1) / (R)6;
    vm = (R)0.5 * (f + fm1) - (Sp1 - Sm1) / (R)6;
    R ap = vp - f, am = vm - f;
    if (ap * am >= (R)0) {
        ap = (R)0;
        am = (R)0;
    } else {
        if (fabs(ap) >= (R)2 * fabs(am)) ap = (R)(-2) * am;
        if (fabs(am) >= (R)2 * fabs(ap)) am = (R)(-2) * ap;
    }
    vp = f + ap;
    vm = f + am;
}
// the parabola of chunk c (1-based) from the chunk values chv(1-2 .. Nc+2)
// (ReconstructRing, ringrecon.F90:34-91): coefficients a, b, c
template <class R>
__device__ __forceinline__ void ring_parabola(int recon, const R* chW, int c, R& a, R& bq, R& cq) {
    R fL, fR;
    const R* p = chW + c + 1;  // chv(c) = chW[c + 1]
    ring_lr(recon, p[-2], p[-1], p[0], p[1], p[2], fL, fR);
    const R f = p[0];
    a = (R)3 * (fL + fR - (R)2 * f);
    bq = (R)2 * ((R)3 * f - fR - (R)2 * fL);
    cq = fL;
}
template <class R> __device__ __forceinline__ R ring_interp(R a, R bq, R cq, int m, int dJ) {
    return (a / (R)3) * (R)(3 * m * m - 3 * m + 1) / (R)(dJ * dJ) + (R)0.5 * bq * (R)(2 * m - 1) / (R)dJ + cq;
}
// periodic ghosts of the chunk values chv(1..Nc)
template <class R> __device__ __forceinline__ void ring_chunk_ghosts(R* chW, int Nc) {
    for (int n = 1; n <= 2; n++) {
        chW[1 - n + 1] = chW[Nc - n + 1 + 1];
        chW[Nc + n + 1] = chW[n + 1];
    }
}

// CalcSmoothE (ringav.F90:212-344) for one ring, one warp per ring: the J
// fluxes through the ring (then the I fluxes) cleaned of Fourier modes
// 0..nft, chunk-averaged, reconstructed, dirtied again; the change of each
// face's flux accumulated along its chunk into the I (J) EMFs of the
// smoothing field. Every sum keeps the sequential order of the CPU code
// (one lane per sum); the lanes split the independent cells and chunks.
template <class R>
__global__ void __launch_bounds__(32) k_ring_smooth_e(GamBox b, RingData Rg, StateBuf<R> S, const GamScalars* sc) {
    if (sc->halted) return;
    const int G = GAM_NG, Np = Rg.Np, nsl = b.Nip + 1, lane = threadIdx.x;
    const long t = blockIdx.x;
    const long nper = (long)nsl * Rg.NumR;
    if (t >= 2 * nper) return;
    const int pole = (int)(t / nper);
    if (!(pole == 0 ? Rg.doS : Rg.doE)) return;
    const int nS = G + (int)(t % nper % nsl), nR = 1 + (int)(t % nper / nsl);
    const int NumCh = Rg.Nch[nR - 1], dC = Np / NumCh;
    extern __shared__ __align__(16) unsigned char ring_smem[];
    R* bF = (R*)ring_smem;  // the ring's fluxes
    R* cl = bF + Np;        // cleaned fluxes, then the flux changes
    R* chW = cl + Np;       // chunk values with 2 periodic ghosts each side
    __shared__ R cf[6];     // CleanRing's coefficients (m, cos / sin)
    R* E = (R*)Rg.smoothE;
    const long fs = b.fs;
    const double* cs = Rg.ftab;
    for (int dd = 0; dd < 2; dd++) {
        const int fD = dd == 0 ? 1 : 0, eD = dd == 0 ? 0 : 1;
        const R eScl = dd == 0 ? (R)1 : (R)(-1);
        const int jf = pole == 1 ? G + b.Njp - nR : (fD == 1 ? G + nR : G + nR - 1);
        const int je = pole == 1 ? G + b.Njp - nR : (eD == 0 ? G + nR : G + nR - 1);
        const R* mf = S.mf + fD * fs;
        if (!GAM_BOX_OK(lidx(b, nS, jf, G), lidx(b, nS, jf, G + Np - 1), 15)) return;
        for (int n = lane; n < Np; n += 32) bF[n] = mf[lidx(b, nS, jf, G + n)];
        __syncwarp();
        // CleanRing's coefficients: one lane per sum, sequential over the ring
        if (lane < 2 * (Rg.nft + 1)) {
            const int m = lane >> 1;
            const double* tab = cs + (long)lane * Np;  // (2 m + c) Np
            R acc = (R)0;
            for (int n = 0; n < Np; n++) acc = acc + bF[n] * (R)tab[n];
            cf[lane] = (m == 0 ? (R)0.5 * (R)Rg.aScl : (R)1 * (R)Rg.aScl) * acc;
        }
        __syncwarp();
        for (int n = lane; n < Np; n += 32) {
            R Q = bF[n];
            for (int m = 0; m <= Rg.nft; m++)
                Q = Q - cf[2 * m] * (R)cs[(2 * m) * Np + n] - cf[2 * m + 1] * (R)cs[(2 * m + 1) * Np + n];
            cl[n] = Q;
        }
        __syncwarp();
        for (int c = lane; c < NumCh; c += 32) {
            R sum = (R)0;
            for (int l = c * dC; l < (c + 1) * dC; l++) sum = sum + cl[l];
            chW[c + 2] = sum / (R)dC;
        }
        __syncwarp();
        if (lane == 0) ring_chunk_ghosts(chW, NumCh);
        __syncwarp();
        // reconstruct and dirty each cell, then its flux change
        for (int n = lane; n < Np; n += 32) {
            const int c = n / dC, m = n - c * dC + 1;
            R a, bq, cq;
            ring_parabola(Rg.recon, chW, c + 1, a, bq, cq);
            R ra = ring_interp(a, bq, cq, m, dC);
            for (int mm = 0; mm <= Rg.nft; mm++)
                ra = ra + cf[2 * mm] * (R)cs[(2 * mm) * Np + n] + cf[2 * mm + 1] * (R)cs[(2 * mm + 1) * Np + n];
            cl[n] = ra - bF[n];
        }
        __syncwarp();
        // the changes accumulated along each chunk into the EMFs
        for (int c = lane; c < NumCh; c += 32) {
            R cum = (R)0;
            for (int m = 0; m < dC; m++) {
                const int n = c * dC + m;
                const long ce = eD * fs + lidx(b, nS, je, G + n);
                if (m == 0) {
                    E[ce] = (R)0;
                    cum = -cl[n];
                } else {
                    E[ce] = eScl * cum;
                    cum = cum - cl[n];
                }
            }
        }
        __syncwarp();
        // replicate k = ks at ke+1 (chunk 0 is lane 0's)
        if (lane == 0) E[eD * fs + lidx(b, nS, je, G + Np)] = E[eD * fs + lidx(b, nS, je, G)];
        __syncwarp();
    }
}

// E2Flux with the smoothing field and dt = 1 (fields.F90:18-51) over the
// faces it changes: rows js..js+NumR and je-NumR..je, i = is..ie+1, k = ks..ke+1
template <class R> __global__ void __launch_bounds__(256) k_ring_e2flux(GamBox b, RingData Rg, StateBuf<R> S,
                                                                          const GamScalars* sc) {
    if (sc->halted) return;
    const int G = GAM_NG, nr = Rg.NumR + 1;
    const long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
    const int ni = b.Nip + 1, nk = b.Nkp + 1;
    const long nrow = (long)ni * nk;
    if (q >= 2L * nr * nrow) return;
    const int pole = (int)(q / (nr * nrow));
    if (!(pole == 0 ? Rg.doS : Rg.doE)) return;
    const long r = q % (nr * nrow);
    const int row = (int)(r / nrow), ii = G + (int)(r % nrow % ni), kk = G + (int)(r % nrow / ni);
    const int jj = pole == 0 ? G + row : G + b.Njp - 1 - Rg.NumR + row;
    const R* E = (const R*)Rg.smoothE;
    const long fs = b.fs, c = lidx(b, ii, jj, kk), sj = b.sx, sk = b.sk;
    GAM_BOX_CHECK(c, c + sj + sk + 1, 15);
    const R* Ei = E;
    const R* Ej = E + fs;
    const R* Ek = E + 2 * fs;
    const R dfi = Ek[c + sj] - Ek[c] - Ej[c + sk] + Ej[c];
    const R dfj = Ei[c + sk] - Ei[c] - Ek[c + 1] + Ek[c];
    const R dfk = Ej[c + 1] - Ej[c] - Ei[c + sj] + Ei[c];
    S.mf[c] = S.mf[c] - (R)1 * dfi;
    S.mf[fs + c] = S.mf[fs + c] - (R)1 * dfj;
    S.mf[2 * fs + c] = S.mf[2 * fs + c] - (R)1 * dfk;
}

// CleanLoops (ringav.F90:347-391): the K fluxes of the pole's first ring
// lose their mean, slices is..ie+1
template <class R> __global__ void __launch_bounds__(32) k_ring_clean_loops(GamBox b, RingData Rg, StateBuf<R> S,
                                                                              const GamScalars* sc) {
    if (sc->halted) return;
    const int G = GAM_NG, ni = b.Nip + 1;
    const int pole = blockIdx.x / ni, ii = G + (int)(blockIdx.x % ni);
    if (!(pole == 0 ? Rg.doS : Rg.doE)) return;
    const int jr = pole == 0 ? G : G + b.Njp - 1;
    R* mK = S.mf + 2 * b.fs;
    if (!GAM_BOX_OK(lidx(b, ii, jr, G), lidx(b, ii, jr, G + b.Nkp), 15)) return;
    extern __shared__ __align__(16) unsigned char ring_smem[];
    const R avg = ring_row_mean(mK, lidx(b, ii, jr, G), b.sk, Rg.Np, (R*)ring_smem);
    const R tScl = (R)Rg.tScl;
    for (int kk = G + threadIdx.x; kk <= G + b.Nkp; kk += 32) {
        const long c = lidx(b, ii, jr, kk);
        mK[c] = mK[c] - tScl * avg;
    }
}

// bFlux2Fld with RingFlux2FieldFix over the cells whose faces the ring
// average changed: j rows 0..js+NumR(+1) and je-NumR-1..Nj-1, every i and k
template <class R> __global__ void __launch_bounds__(128) k_ring_bfield(GamBox b, Geo<R> g, RingData Rg,
                                                                          StateBuf<R> S, const GamScalars* sc) {
    if (sc->halted) return;
    const int G = GAM_NG, nr = G + Rg.NumR + 2;
    const long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
    const long nrow = (long)b.Ni * b.Nk;
    if (q >= 2L * nr * nrow) return;
    const int pole = (int)(q / (nr * nrow));
    if (!(pole == 0 ? Rg.doS : Rg.doE)) return;
    const long r = q % (nr * nrow);
    const int row = (int)(r / nrow), ii = (int)(r % nrow % b.Ni), kk = (int)(r % nrow / b.Ni);
    const int jj = pole == 0 ? row : b.Nj - nr + row;
    const long fs = b.fs, c = lidx(b, ii, jj, kk);
    int jc = jj, kc = kk;
    const long cb = ring_conj_cc(b, Rg, jc, kc) ? lidx(b, ii, jc, kc) : c;
    GAM_BOX_CHECK(cb, cb + b.sk, 15);
    R B[3];
    cell_bxyz(b, g, cb, S.mf[cb], S.mf[cb + 1], S.mf[fs + cb], S.mf[fs + cb + b.sx], S.mf[2 * fs + cb],
              S.mf[2 * fs + cb + b.sk], B);
#pragma unroll
    for (int x = 0; x < 3; x++) S.B[x * fs + c] = B[x];
}

// SmoothGas (ringav.F90:78-210) for one ring, one warp per ring: the ring
// variables (rho, momentum, internal energy; Gas2Ring, ringutils.F90:
// 804-830) chunk-averaged, reconstructed per chunk and written back as gas
// (Ring2Gas :832-856); each chunk sum sequential on one lane
template <class R>
__global__ void __launch_bounds__(32) k_ring_smooth_gas(GamBox b, DevParams<R> P, StateBuf<R> S, const GamScalars* sc) {
    if (sc->halted) return;
    const RingData& Rg = P.ring;
    const int G = GAM_NG, Np = Rg.Np, nsl = b.Nip, lane = threadIdx.x;
    const long t = blockIdx.x;
    const long nper = (long)nsl * Rg.NumR;
    if (t >= 2 * nper) return;
    const int pole = (int)(t / nper);
    if (!(pole == 0 ? Rg.doS : Rg.doE)) return;
    const int nS = G + (int)(t % nper % nsl), nR = 1 + (int)(t % nper / nsl);
    const int NumCh = Rg.Nch[nR - 1], dC = Np / NumCh;
    const int jr = pole == 0 ? G + nR - 1 : G + b.Njp - nR;
    const int cst = NumCh + 4;
    extern __shared__ __align__(16) unsigned char ring_smem[];
    R* rW = (R*)ring_smem;  // 5 x Np ring variables
    R* chW = rW + 5 * Np;   // 5 x (NumCh + 4) chunk values
    const long fs = b.fs;
    if (!GAM_BOX_OK(lidx(b, nS, jr, G), lidx(b, nS, jr, G + Np - 1), 15)) return;
    for (int n = lane; n < Np; n += 32) {
        const long c = lidx(b, nS, jr, G + n);
        R W[5];
#pragma unroll
        for (int v = 0; v < 5; v++) W[v] = S.Gas[v * fs + c];
        const R D = rmax(W[0], P.dFloor);
        const R KinE = (R)0.5 * (W[1] * W[1] + W[2] * W[2] + W[3] * W[3]) / D;
        const R Pr = rmax(P.gm1 * (W[4] - KinE), P.pFloor);
        W[0] = D;
        W[4] = Pr / P.gm1;
#pragma unroll
        for (int v = 0; v < 5; v++) rW[v * Np + n] = W[v];
    }
    __syncwarp();
    for (int q = lane; q < 5 * NumCh; q += 32) {
        const int v = q / NumCh, c = q % NumCh;
        R sum = (R)0;
        for (int l = c * dC; l < (c + 1) * dC; l++) sum = sum + rW[v * Np + l];
        chW[v * cst + c + 2] = sum / (R)dC;
    }
    __syncwarp();
    if (lane < 5) ring_chunk_ghosts(chW + lane * cst, NumCh);
    __syncwarp();
    for (int n = lane; n < Np; n += 32) {
        const int c = n / dC, m = n - c * dC + 1;
        R W[5];
#pragma unroll
        for (int v = 0; v < 5; v++) {
            R a, bq, cq;
            ring_parabola(Rg.recon, chW + v * cst, c + 1, a, bq, cq);
            W[v] = ring_interp(a, bq, cq, m, dC);
        }
        const R D = rmax(W[0], P.dFloor);
        R Pr = P.gm1 * W[4];
        Pr = rmax(Pr, P.pFloor);
        const R KinE = (R)0.5 * (W[1] * W[1] + W[2] * W[2] + W[3] * W[3]) / D;
        const long c2 = lidx(b, nS, jr, G + n);
        S.Gas[c2] = D;
        S.Gas[fs + c2] = W[1];
        S.Gas[2 * fs + c2] = W[2];
        S.Gas[3 * fs + c2] = W[3];
        S.Gas[4 * fs + c2] = KinE + Pr / P.gm1;
    }
}

// Con2Fast (gamutils.F90:255-269 with CellPress2Cs :238-253, Boris :356-358)
template <class R> __device__ __forceinline__ R con2fast(const DevParams<R>& P, const R* gCon, const R* Bin) {
    R rho = rmax(gCon[0], P.dFloor);
    R Vx = gCon[1] / rho, Vy = gCon[2] / rho, Vz = gCon[3] / rho;
    R KinE = (R)0.5 * rho * (Vx * Vx + Vy * Vy + Vz * Vz);
    R Pr = rmax(P.gm1 * (gCon[4] - KinE), P.pFloor);
    R Cs = Mth<R>::sqrt_(P.gamma * Pr / rho);
    double Bd[3] = {(double)Bin[0], (double)Bin[1], (double)Bin[2]};
    R MagB = (R)norm2s3(Bd);
    R Va = MagB / Mth<R>::sqrt_(gCon[0]);
    if (P.doBoris) Va = boris_speed((R)P.Ca, Va);
    return Mth<R>::sqrt_(Cs * Cs + Va * Va);
}
// NudgeSW's ring branch (apps/wind.F90:458-484): the last active cell and the
// one across the E pole flow out at the fast speed when they flow in
template <class R>
__global__ void __launch_bounds__(128) k_ring_nudge_axis(GamBox b, DevParams<R> P, StateBuf<R> S, const GamScalars* sc) {
    if (sc->halted) return;
    const int G = GAM_NG;
    const long q = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (q >= 2L * b.Nkp) return;
    const int kk = G + (int)(q % b.Nkp), jj = G + b.Njp - 1 + (int)(q / b.Nkp), ii = G + b.Nip - 1;
    const long fs = b.fs, c = lidx(b, ii, jj, kk);
    GAM_BOX_CHECK(c, c, 15);
    if (!(S.Gas[fs + c] > (R)0)) return;
    R U[5], W[5], B[3];
#pragma unroll
    for (int v = 0; v < 5; v++) U[v] = S.Gas[v * fs + c];
#pragma unroll
    for (int x = 0; x < 3; x++) B[x] = S.B[x * fs + c];
    const R Cx = con2fast(P, U, B);
    cell_c2p(P, U, W);
    W[1] = -Cx;
    cell_p2c(P, W, U);
#pragma unroll
    for (int v = 0; v < 5; v++) S.Gas[v * fs + c] = U[v];
}

// UpdateStateData time bookkeeping + CalcDT decisions (gamapp.F90:110-111,
// mhdgroup.F90:106, step.F90:58-168). A failure halts the remaining kernels.
__global__ void k_dt_finalize(GamScalars* sc) {
    if (sc->halted) return;
    sc->ootime = sc->otime;        // CopyState(oState, ooState) (mhdgroup.F90:100-102)
    sc->otime = sc->time;          // CopyState (mhdgroup.F90:255)
    sc->time = sc->time + sc->dt;  // mhdgroup.F90:106
    sc->ts = sc->ts + 1;
    sc->t = sc->t + sc->dt;
    if (sc->fixedTimestep) return;
    const double dtOld = sc->dt;
    double dtMin = __longlong_as_double((long long)sc->dtmin_bits);
    sc->dtmin_bits = dbits(HUGE_DT);
    bool isDisaster = (dtMin == HUGE_DT) || sc->nbad > 0;
    bool isBad = false;
    if (sc->ts > 0) {
        if (dtOld / dtMin >= 10.0) isBad = true;
        if (sc->dt0 > TINY && dtMin / sc->dt0 <= sc->limDT0) isBad = true;
        if (dtMin <= TINY) isDisaster = true;
    }
    double dt = dtMin;
    if (sc->t + dt > sc->tFin) dt = fmax(sc->tFin - sc->t, TINY);
    if (sc->dt0 > TINY && dt > 10.0 * sc->dt0) dt = 10.0 * sc->dt0;
    sc->dt = dt;
    if (isDisaster) { sc->status = 5; sc->halted = 1; }
    else if (isBad) { sc->status = 4; sc->halted = 1; }
}

// Boundary kinds: 0 periodic, 1 none, 2 zero-gradient, 3 inner sphere,
// 4 solar wind, 6 uniform inflow (include/gamgpu.h).
enum { BCK_PERIODIC = 0, BCK_NONE = 1, BCK_ZEROGRAD = 2, BCK_SPHIN = 3, BCK_WIND = 4, BCK_HALO = 5, BCK_INFLOW = 6,
       BCK_ION = 7, BCK_LFM = 8 };

// Gather maps of the boundary conditions that copy values (bcs.F90:279-450
// periodic, :799-892 zero-gradient, :934-957 SphIn). x is the box index along
// the BC's direction, n the active count, normal = the value sits on a face
// normal to that direction. Returns the source index (x when untouched).
__device__ __forceinline__ int bmap_lo(int kind, int x, int n) {
    const int G = GAM_NG;
    if (x >= G) return x;
    if (kind == BCK_PERIODIC) return x + n;
    if (kind == BCK_ZEROGRAD || kind == BCK_SPHIN) return G;
    return x;
}
__device__ __forceinline__ int bmap_hi(int kind, int x, int n, bool normal) {
    const int G = GAM_NG;
    if (normal) {
        if (x < G + n + 1 || x > G + n + 4) return x;
        if (kind == BCK_PERIODIC) return x - n;
        if (kind == BCK_ZEROGRAD) return G + n;  // magFlux(je+n+1,JDIR) = magFlux(je+1,JDIR)
        return x;
    }
    if (x < G + n || x > G + n + 3) return x;
    if (kind == BCK_PERIODIC) return x - n;
    if (kind == BCK_ZEROGRAD) return G + n - 1;
    return x;
}
// do25D periodic k: every ghost slab copies ks (bcs.F90:387-394, 423-429)
__device__ __forceinline__ int bmap_25d(int x) {
    const int G = GAM_NG;
    if ((x >= G - 4 && x < G) || (x > G && x <= G + 4)) return G;
    return x;
}

// Source of value (ii,jj,kk) of component comp (-1 cell, 0..2 face normal)
// after the K, then J, then I boundary conditions that are gathers (the
// reference applies INI, OUTI, INJ, OUTJ, INK, OUTK in that order, so a value
// ends up copied from the I-map of the J-map of the K-map of its index). Each
// map applies only over its loop ranges: periodic over the whole box,
// zero-gradient and SphIn over cell ranges of the other two indices. The
// non-periodic I sides (SphIn, wind) were applied before, in place. withB:
// follow only the BCs that also copy Bxyz (periodic and the LFM pole;
// zero-gradient does not). The LFM pole (lfmIn / lfmOut, over the whole
// box) maps a ghost row to its conjugate across the axis and reverses J and
// K fluxes: the return value is the sign of the source.
template <class R>
__device__ __forceinline__ int bc_source(const GamBox& b, const DevParams<R>& P, int comp, bool withB, int& ii,
                                         int& jj, int& kk) {
    int sgn = 1;
    if (P.do25D)
        kk = bmap_25d(kk);
    else if (P.bc[4] == BCK_PERIODIC) {
        kk = bmap_lo(BCK_PERIODIC, kk, b.Nkp);
        kk = bmap_hi(BCK_PERIODIC, kk, b.Nkp, comp == 2);
    }
    if (P.ring.on) {
        sgn = ring_bc_jmap(b, P.ring, comp, jj, kk);
    } else if (P.bc[2] == BCK_PERIODIC || (!withB && ii < b.Ni && kk < b.Nk)) {
        jj = bmap_lo(P.bc[2], jj, b.Njp);
        jj = bmap_hi(P.bc[3], jj, b.Njp, comp == 1);
    }
    if (P.bc[0] == BCK_PERIODIC) {
        ii = bmap_lo(BCK_PERIODIC, ii, b.Nip);
        ii = bmap_hi(BCK_PERIODIC, ii, b.Nip, comp == 0);
    }
    return sgn;
}


// face * (n . B) on face d of box cell c (zeroGrad_obcI, bcs.F90:842-844)
template <class R>
__device__ __forceinline__ R face_proj(const GamBox& b, const Geo<R>& g, int d, long c, const R* B) {
    const long fs = b.fs;
    const R* n = g.Tf + (long)(9 * d) * fs + c;
    return g.face[d * fs + c] * (B[0] * n[0] + B[1] * n[fs] + B[2] * n[2 * fs]);
}

// ---- the solar-wind time series (apps/wind.F90), in FP64 in both forms.
// InterpWgts (:825-868) with doWindInterp = F: the row at or below t (0-based)
__device__ __forceinline__ int wind_row(const WindData& W, double t) {
    if (t >= W.tMax) return W.n - 1;
    if (t <= W.tMin) return 0;
    const int i0 = (int)floor((t - W.tMin) / W.dtW) + 1;  // 1-based, as the reference
    return i0 + 1 <= W.n ? i0 - 1 : W.n - 2;
}
// InterpWind (:766-809) without the spin-up sequence
__device__ __forceinline__ void wind_interp(const WindData& W, double t, double& D, double& P, double* V, double* B) {
    const double* r = W.ts + 12 * wind_row(W, t);
    D = r[1];
    V[0] = r[2]; V[1] = r[3]; V[2] = r[4];
    P = r[5];
    B[1] = r[7];
    B[2] = r[8];
    B[0] = W.Bx0 + W.ByC * B[1] + W.BzC * B[2];
    if (t <= W.tMin) B[0] = B[1] = B[2] = 0.0;
}
// PlaceWind (:812-822) and RefreshWind (:116-157) at time t
__device__ __forceinline__ void wind_refresh(const WindData& W, double t, double* xyzW, double* vFr) {
    const double* r = W.ts + 12 * wind_row(W, t);
    xyzW[0] = r[9]; xyzW[1] = r[10]; xyzW[2] = r[11];
    double D, P, V0[3], B[3];
    wind_interp(W, t, D, P, V0, B);
    const double vSpd = -norm2s3(V0);
    const double bcc = sqrt(W.ByC * W.ByC + W.BzC * W.BzC);
    const double btt = sqrt(1.0 + bcc * bcc);
    if (bcc > TINY) {
        const double CosBp = W.ByC / bcc, SinBp = W.BzC / bcc, CosF = 1.0 / btt, SinF = bcc / btt;
        vFr[0] = vSpd * (CosF * CosF);
        vFr[1] = -(vSpd * CosF * SinF * CosBp);
        vFr[2] = -(vSpd * CosF * SinF * SinBp);
    } else {
        vFr[0] = vSpd; vFr[1] = 0.0; vFr[2] = 0.0;
    }
}
// GetWindAt (:160-176): the wind rewound by the lag time to xyz
__device__ __forceinline__ void wind_at(const WindData& W, const double* xyzW, const double* vFr, const double* xyz,
                                        double t, double& D, double& P, double* V, double* B) {
    const double vMag = norm2s3(vFr);
    const double DelT = ((xyz[0] - xyzW[0]) * vFr[0] + (xyz[1] - xyzW[1]) * vFr[1] + (xyz[2] - xyzW[2]) * vFr[2]) /
                        (vMag * vMag);
    wind_interp(W, t - DelT, D, P, V, B);
}
// wgtWind (:180-203) with RampDown (math.F90:97-111); CUDA's acos and exp
__device__ __forceinline__ double wind_weight(const WindData& W, const double* xyzW, const double* vFr,
                                              const double* xyz, double t) {
    double D, P, V[3], B[3];
    wind_at(W, xyzW, vFr, xyz, t, D, P, V, B);
    const double nA = sqrt(xyz[0] * xyz[0] + xyz[1] * xyz[1] + xyz[2] * xyz[2]);
    const double vA = sqrt(V[0] * V[0] + V[1] * V[1] + V[2] * V[2]);
    double c = 0.0;
#pragma unroll
    for (int x = 0; x < 3; x++) {
        const double nh = nA <= TINY ? 0.0 : xyz[x] / nA;
        const double vh = vA <= TINY ? 0.0 : V[x] / vA;
        c = x == 0 ? (-vh) * nh : c + (-vh) * nh;
    }
    const double dTh = acos(c) * 180.0 / PI_D;
    if (dTh <= 90.0) return 1.0;
    if (dTh >= 180.0) return 0.0;
    const double rScl = (dTh - 90.0) / 90.0;
    return exp(-1.0 / (1.0 - rScl * rScl) + 1.0);
}

// The non-periodic I boundaries, in place: the SphIn copy or the uniform
// inflow on the inner side (bcs.F90:934-957), the solar-wind blend
// (apps/wind.F90:206-300) or zeroGrad_obcI (bcs.F90:820-850) on the outer
// side, for ghost layer n = 1..4 of every (j, k). Writes touch ghost cells and
// ghost faces only; the reads are of the first / last active cell.
template <class R>
__global__ void __launch_bounds__(256) k_bc_iside(GamBox b, DevParams<R> P, Geo<R> g, StateBuf<R> s,
                                                  const GamScalars* sc) {
    if (sc->halted) return;
    const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    const int n = 1 + (int)(t & 3);
    const long q = t >> 2;
    const int jj = (int)(q % (b.Nj + 1)), kk = (int)(q / (b.Nj + 1));
    if (kk > b.Nk) return;
    const long fs = b.fs;
    const int G = GAM_NG;
    const bool cellJK = jj < b.Nj && kk < b.Nk;
    GAM_BOX_CHECK(lidx(b, 0, jj, kk), lidx(b, b.Ni, jj, kk), 14);  // the row this thread writes in
    if (P.bc[0] == BCK_SPHIN && cellJK) {
        const long dst = lidx(b, G - n, jj, kk), src = lidx(b, G, jj, kk);
#pragma unroll
        for (int v = 0; v < 5; v++) s.Gas[v * fs + dst] = s.Gas[v * fs + src];
#pragma unroll
        for (int x = 0; x < 3; x++) s.mf[x * fs + dst] = s.mf[x * fs + src];
#pragma unroll
        for (int x = 0; x < 3; x++) s.B[x * fs + dst] = s.B[x * fs + src];
    }
    if (P.bc[0] == BCK_ION) {
        // IonInner (earthcmi.F90:441-583) with CellPlasmaBC (msphingest.F90:
        // 268-372, single fluid, no ingestion): density and pressure of the
        // mirror cell is+n-1 (k wrapped, lfmIJKcc ringutils.F90:482-518), the
        // velocity of the table; zero flux through the ghost layer's faces
        // (isGoodFaceIJK ranges, gridutils.F90:985-1015)
        const long cg = lidx(b, G - n, jj, kk);
        if (cellJK) {
            int kp = kk, jp = jj;
            if (kk < G) kp = kk + b.Nkp;
            else if (kk >= G + b.Nkp) kp = kk - b.Nkp;
            if (P.ring.on) {  // across the LFM pole: the conjugate's mirror cell
                int kr = kk;
                if (ring_conj_cc(b, P.ring, jp, kr)) kp = kr;
            }
            const long src = lidx(b, G + n - 1, jp, kp);
            GAM_BOX_CHECK(src, src, 14);
            R pU[5], pW[5], gC[5];
#pragma unroll
            for (int v = 0; v < 5; v++) pU[v] = s.Gas[v * fs + src];
            cell_c2p(P, pU, pW);
            const double* V = P.ion.Vg + 3 * ((n - 1) + 4 * ((long)jj + (long)b.Nj * kk));
            const R gW[5] = {pW[0], (R)V[0], (R)V[1], (R)V[2], pW[4]};
            cell_p2c(P, gW, gC);
#pragma unroll
            for (int v = 0; v < 5; v++) s.Gas[v * fs + cg] = gC[v];
        }
        if (jj < b.Nj && kk < b.Nk) s.mf[cg] = (R)0;
        if (jj <= b.Nj && kk < b.Nk) s.mf[fs + cg] = (R)0;
        if (jj < b.Nj && kk <= b.Nk) s.mf[2 * fs + cg] = (R)0;
    }
    if (P.bc[0] == BCK_INFLOW && cellJK) {
        const double* w = P.inflow;
        R gW[5] = {(R)w[0], (R)w[2], (R)w[3], (R)w[4], (R)w[1]}, gC[5];
        cell_p2c(P, gW, gC);
        const R Bin[3] = {(R)w[5], (R)w[6], (R)w[7]};
        const long c = lidx(b, G - n, jj, kk);
#pragma unroll
        for (int v = 0; v < 5; v++) s.Gas[v * fs + c] = gC[v];
#pragma unroll
        for (int d = 0; d < 3; d++) s.mf[d * fs + c] = face_proj(b, g, d, c, Bin);
    }
    if (P.bc[1] == BCK_ZEROGRAD && cellJK) {
        const int ie = G + b.Nip - 1;
        const long cp = lidx(b, ie, jj, kk), cg = lidx(b, ie + n, jj, kk);
        GAM_BOX_CHECK(cp, cp + b.sk, 14);
#pragma unroll
        for (int v = 0; v < 5; v++) s.Gas[v * fs + cg] = s.Gas[v * fs + cp];
        R B[3];
        cell_bxyz(b, g, cp, s.mf[cp], s.mf[cp + 1], s.mf[fs + cp], s.mf[fs + cp + b.sx], s.mf[2 * fs + cp],
                  s.mf[2 * fs + cp + b.sk], B);
        s.mf[cg + 1] = face_proj(b, g, 0, cg + 1, B);
        s.mf[fs + cg] = face_proj(b, g, 1, cg, B);
        s.mf[2 * fs + cg] = face_proj(b, g, 2, cg, B);
    }
    if (P.bc[1] != BCK_WIND) return;
    const WindData& W = P.wind;
    const long wi = (n - 1) + 4 * (jj + (long)(b.Nj + 1) * kk);
    const int ig = G + b.Nip - 1 + n, ip = G + b.Nip - 1;
    // a time series: RefreshWind at Model%t (the time after this step's
    // update), then the wind at each point's lag time (apps/wind.F90:218-223)
    const bool series = W.n > 0;
    const double tnow = sc->t;
    double xyzW[3] = {0.0, 0.0, 0.0}, vFr[3] = {-1.0, 0.0, 0.0};
    if (series) wind_refresh(W, tnow, xyzW, vFr);
    if (cellJK) {
        const double MinMach = 1.0;
        double wSW, Dsw = W.state[0], Psw = W.state[1], Vsw[3] = {W.state[2], W.state[3], W.state[4]};
        if (series) {
            const long cg = lidx(b, ig, jj, kk);
            const double xc[3] = {(double)g.xyzcc[cg], (double)g.xyzcc[fs + cg], (double)g.xyzcc[2 * fs + cg]};
            wSW = wind_weight(W, xyzW, vFr, xc, tnow);
            if (wSW > TINY) {
                double Bsw[3];
                wind_at(W, xyzW, vFr, xc, tnow, Dsw, Psw, Vsw, Bsw);
            }
        } else {
            wSW = W.wC[wi];
        }
        const double wMHD = 1.0 - wSW;
        R gW_sw[5] = {(R)0, (R)0, (R)0, (R)0, (R)0}, gW_in[5] = {(R)0, (R)0, (R)0, (R)0, (R)0};
        if (wSW > TINY) {
            gW_sw[0] = (R)Dsw;
            gW_sw[4] = (R)Psw;
            gW_sw[1] = (R)Vsw[0];
            gW_sw[2] = (R)Vsw[1];
            gW_sw[3] = (R)Vsw[2];
        }
        if (wMHD > TINY) {
            const long cp = lidx(b, ip, jj, kk);
            R gCon[5], Bin[3];
#pragma unroll
            for (int v = 0; v < 5; v++) gCon[v] = s.Gas[v * fs + cp];
#pragma unroll
            for (int x = 0; x < 3; x++) Bin[x] = s.B[x * fs + cp];
            cell_c2p(P, gCon, gW_in);
            // Con2Fast (gamutils.F90:255-269) with CellPress2Cs (:238-253)
            R rho = rmax(gCon[0], P.dFloor);
            R Vx = gCon[1] / rho, Vy = gCon[2] / rho, Vz = gCon[3] / rho;
            R KinE = (R)0.5 * rho * (Vx * Vx + Vy * Vy + Vz * Vz);
            R Pr = rmax(P.gm1 * (gCon[4] - KinE), P.pFloor);
            R Cs = Mth<R>::sqrt_(P.gamma * Pr / rho);
            double Bd[3] = {(double)Bin[0], (double)Bin[1], (double)Bin[2]};
            R MagB = (R)norm2s3(Bd);
            R Va = MagB / Mth<R>::sqrt_(gCon[0]);
            if (P.doBoris) Va = boris_speed((R)P.Ca, Va);
            R Cx = Mth<R>::sqrt_(Cs * Cs + Va * Va);
            const long cf = lidx(b, ip + 1, jj, kk);
            R nH[3] = {g.Tf[0 * fs + cf], g.Tf[1 * fs + cf], g.Tf[2 * fs + cf]};
            R V[3] = {gW_in[1], gW_in[2], gW_in[3]};
            R dn = V[0] * nH[0] + V[1] * nH[1] + V[2] * nH[2];
            if (dn < (R)MinMach * Cx) {
#pragma unroll
                for (int x = 0; x < 3; x++) V[x] = V[x] - dn * nH[x] + (R)MinMach * Cx * nH[x];
            }
            gW_in[1] = V[0];
            gW_in[2] = V[1];
            gW_in[3] = V[2];
        }
        R gW[5], gC[5];
#pragma unroll
        for (int v = 0; v < 5; v++) gW[v] = (R)wSW * gW_sw[v] + (R)wMHD * gW_in[v];
        cell_p2c(P, gW, gC);
        const long cg = lidx(b, ig, jj, kk);
#pragma unroll
        for (int v = 0; v < 5; v++) s.Gas[v * fs + cg] = gC[v];
    }
    // face fluxes: I face ig+1, J and K faces of cell ig
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const long cf = lidx(b, d == 0 ? ig + 1 : ig, jj, kk), cin = lidx(b, d == 0 ? ip + 1 : ip, jj, kk);
        double w, sw;
        if (series) {
            // WindMagFlux (apps/wind.F90:378-391) with Project2Face (bcs.F90:250-263)
            const double xf[3] = {(double)g.xfc[(3 * d) * fs + cf], (double)g.xfc[(3 * d + 1) * fs + cf],
                                  (double)g.xfc[(3 * d + 2) * fs + cf]};
            w = wind_weight(W, xyzW, vFr, xf, tnow);
            double D, Pw, V[3], Bf[3];
            wind_at(W, xyzW, vFr, xf, tnow, D, Pw, V, Bf);
            const R* nh = g.Tf + (long)(9 * d) * fs + cf;
            sw = (double)g.face[d * fs + cf] * ((double)nh[0] * Bf[0] + (double)nh[fs] * Bf[1] + (double)nh[2 * fs] * Bf[2]);
        } else {
            w = W.wF[d * W.nw + wi];
            sw = W.sF[d * W.nw + wi];
        }
        s.mf[d * fs + cf] = (R)w * (R)sw + ((R)1 - (R)w) * s.mf[d * fs + cin];
    }
}
// Bxyz of the wind (apps/wind.F90:341-351) or inflow ghost cells from their
// new fluxes: ig = ie + n (outer) or is - n (inner)
template <class R>
__global__ void __launch_bounds__(256) k_bc_iside_b(GamBox b, Geo<R> g, StateBuf<R> s, const GamScalars* sc,
                                                    int outer, int wrapk = 0) {
    if (sc->halted) return;
    const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    const int n = 1 + (int)(t & 3);
    const long q = t >> 2;
    const int jj = (int)(q % b.Nj), kk = (int)(q / b.Nj);
    if (kk >= b.Nk) return;
    const long fs = b.fs;
    const int ii = outer ? GAM_NG + b.Nip - 1 + n : GAM_NG - n;
    const long c = lidx(b, ii, jj, kk);
    // the ionospheric boundary takes the field of the k-wrapped cell
    // (IonInner's CellBxyz of lfmIJKcc's cell, earthcmi.F90:530-543)
    int kp = kk;
    if (wrapk && kk < GAM_NG) kp = kk + b.Nkp;
    else if (wrapk && kk >= GAM_NG + b.Nkp) kp = kk - b.Nkp;
    const long cs = lidx(b, ii, jj, kp);
    GAM_BOX_CHECK(cs, cs + b.sk, 14);
    R B[3];
    cell_bxyz(b, g, cs, s.mf[cs], s.mf[cs + 1], s.mf[fs + cs], s.mf[fs + cs + b.sx], s.mf[2 * fs + cs],
              s.mf[2 * fs + cs + b.sk], B);
#pragma unroll
    for (int x = 0; x < 3; x++) s.B[x * fs + c] = B[x];
}

// The gather boundary conditions (periodic, zero-gradient J) as one pass over
// the ghost shell, then the final bFlux2Fld of every ghost cell and of every
// cell whose faces changed. copyB: the initial EnforceBCs of CalcGridInfo
// (init.F90:226-238), which copies Bxyz with the BCs instead of recomputing it.
// The launch enumerates the shell outside the deep interior [G+1, G+N-2]^3;
// per dimension the "outer" indices are [0, G] and [G+N-1, Nmax].
struct Shell {
    int nx, ny, nz;         // face-box extents (Ni+1, Nj+1, Nk+1)
    int a[3], bnd[3];       // deep interior [a, bnd] per dimension (empty if bnd < a)
    long nA, nB, nC;        // counts of the three parts
};
static inline Shell make_shell(const GamBox& b) {
    Shell sh;
    sh.nx = b.Ni + 1; sh.ny = b.Nj + 1; sh.nz = b.Nk + 1;
    const int N[3] = {b.Nip, b.Njp, b.Nkp}, M[3] = {sh.nx, sh.ny, sh.nz};
    int nout[3], nin[3];
    for (int d = 0; d < 3; d++) {
        sh.a[d] = GAM_NG + 1;
        sh.bnd[d] = GAM_NG + N[d] - 2;
        nin[d] = sh.bnd[d] >= sh.a[d] ? sh.bnd[d] - sh.a[d] + 1 : 0;
        nout[d] = M[d] - nin[d];
    }
    sh.nA = (long)nout[2] * sh.ny * sh.nx;
    sh.nB = (long)nin[2] * nout[1] * sh.nx;
    sh.nC = (long)nin[2] * nin[1] * nout[0];
    return sh;
}
__device__ __forceinline__ int outer_coord(int o, int a, int bnd) { return (bnd >= a && o >= a) ? o - a + bnd + 1 : o; }
__device__ __forceinline__ bool shell_ijk(const Shell& sh, long t, int& ii, int& jj, int& kk) {
    if (t < sh.nA) {
        ii = (int)(t % sh.nx);
        long q = t / sh.nx;
        jj = (int)(q % sh.ny);
        kk = outer_coord((int)(q / sh.ny), sh.a[2], sh.bnd[2]);
        return true;
    }
    t -= sh.nA;
    if (t < sh.nB) {
        ii = (int)(t % sh.nx);
        long q = t / sh.nx;
        const int nout1 = sh.ny - (sh.bnd[1] >= sh.a[1] ? sh.bnd[1] - sh.a[1] + 1 : 0);
        jj = outer_coord((int)(q % nout1), sh.a[1], sh.bnd[1]);
        kk = sh.a[2] + (int)(q / nout1);
        return true;
    }
    t -= sh.nB;
    if (t < sh.nC) {
        const int nout0 = sh.nx - (sh.bnd[0] >= sh.a[0] ? sh.bnd[0] - sh.a[0] + 1 : 0);
        ii = outer_coord((int)(t % nout0), sh.a[0], sh.bnd[0]);
        long q = t / nout0;
        const int nin1 = sh.bnd[1] - sh.a[1] + 1;
        jj = sh.a[1] + (int)(q % nin1);
        kk = sh.a[2] + (int)(q / nin1);
        return true;
    }
    return false;
}

template <class R>
__global__ void __launch_bounds__(256) k_bc(GamBox b, DevParams<R> P, Geo<R> g, StateBuf<R> s, const GamScalars* sc,
                                            int copyB, Shell sh) {
    if (sc->halted) return;
    int ii, jj, kk;
    const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (!shell_ijk(sh, t, ii, jj, kk)) return;
    const long fs = b.fs;
    const long c = lidx(b, ii, jj, kk);
    GAM_BOX_CHECK(c, c, 14);
    // faces
#pragma unroll
    for (int d = 0; d < 3; d++) {
        int x = ii, y = jj, z = kk;
        const int sg = bc_source(b, P, d, false, x, y, z);
        GAM_BOX_CHECK(lidx(b, x, y, z), lidx(b, x, y, z), 14);
        if (x != ii || y != jj || z != kk) {
            const R v = s.mf[d * fs + lidx(b, x, y, z)];
            s.mf[d * fs + c] = sg < 0 ? -v : v;
        }
    }
    if (ii >= b.Ni || jj >= b.Nj || kk >= b.Nk) return;
    // cell
    {
        int x = ii, y = jj, z = kk;
        bc_source(b, P, -1, false, x, y, z);
        GAM_BOX_CHECK(lidx(b, x, y, z), lidx(b, x, y, z), 14);
        if (x != ii || y != jj || z != kk) {
            const long src = lidx(b, x, y, z);
#pragma unroll
            for (int v = 0; v < 5; v++) s.Gas[v * fs + c] = s.Gas[v * fs + src];
        }
        if (copyB) {
            int xb = ii, yb = jj, zb = kk;
            bc_source(b, P, -1, true, xb, yb, zb);
            GAM_BOX_CHECK(lidx(b, xb, yb, zb), lidx(b, xb, yb, zb), 14);
            if (xb != ii || yb != jj || zb != kk) {
                const long src = lidx(b, xb, yb, zb);
#pragma unroll
                for (int q = 0; q < 3; q++) s.B[q * fs + c] = s.B[q * fs + src];
            }
        }
    }
    if (!P.doMHD || copyB) return;
    // the six faces of this cell after the boundary fill
    auto srcf = [&](int d, int a0, int a1, int a2) -> long {
        int x = a0, y = a1, z = a2;
        bc_source(b, P, d, false, x, y, z);
        return lidx(b, x, y, z);
    };
    // RingFlux2FieldFix: a cell across the LFM pole takes its conjugate's field
    int jb = jj, kb = kk;
    const bool conj = P.ring.on && ring_conj_cc(b, P.ring, jb, kb);
    const long fI = srcf(0, ii, jb, kb), fIp = srcf(0, ii + 1, jb, kb);
    const long fJ = srcf(1, ii, jb, kb), fJp = srcf(1, ii, jb + 1, kb);
    const long fK = srcf(2, ii, jb, kb), fKp = srcf(2, ii, jb, kb + 1);
    {
        long lo = fI, hi = fI;
        for (long v : {fIp, fJ, fJp, fK, fKp}) {
            lo = v < lo ? v : lo;
            hi = v > hi ? v : hi;
        }
        GAM_BOX_CHECK(lo, hi, 14);
    }
    const bool facesMapped = fI != c || fIp != c + 1 || fJ != c || fJp != c + b.sx || fK != c || fKp != c + b.sk;
    const int G = GAM_NG;
    const bool ghost = ii < G || ii >= G + b.Nip || jj < G || jj >= G + b.Njp || kk < G || kk >= G + b.Nkp;
    if (!(ghost || facesMapped)) return;
    R B[3];
    cell_bxyz(b, g, conj ? lidx(b, ii, jb, kb) : c, s.mf[fI], s.mf[fIp], s.mf[fs + fJ], s.mf[fs + fJp],
              s.mf[2 * fs + fK], s.mf[2 * fs + fKp], B);
#pragma unroll
    for (int x = 0; x < 3; x++) s.B[x * fs + c] = B[x];
}

// All boundary conditions of one EnforceBCs (+ final bFlux2Fld unless copyB).
template <class R> void launch_bcs(const Ctx<R>& C, const StateBuf<R>& S, cudaStream_t s, int copyB) {
    const GamBox& b = C.b;
    const bool iside = C.P.bc[0] == BCK_SPHIN || C.P.bc[0] == BCK_INFLOW || C.P.bc[0] == BCK_ION ||
                       C.P.bc[1] == BCK_WIND || C.P.bc[1] == BCK_ZEROGRAD;
    if (iside) {
        const long n = 4L * (b.Nj + 1) * (b.Nk + 1);
        k_bc_iside<R><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(b, C.P, C.g, S, C.sc);
        // the wind's and the inflow's own Bxyz of their ghost cells matter
        // only where no final bFlux2Fld follows (the initial fill); a step
        // recomputes every ghost
        const long m = 4L * b.Nj * b.Nk;
        if (C.P.bc[1] == BCK_WIND && copyB)
            k_bc_iside_b<R><<<(unsigned)((m + 255) / 256), 256, 0, s>>>(b, C.g, S, C.sc, 1);
        if (C.P.bc[0] == BCK_INFLOW && copyB)
            k_bc_iside_b<R><<<(unsigned)((m + 255) / 256), 256, 0, s>>>(b, C.g, S, C.sc, 0);
        if (C.P.bc[0] == BCK_ION && copyB)
            k_bc_iside_b<R><<<(unsigned)((m + 255) / 256), 256, 0, s>>>(b, C.g, S, C.sc, 0, 1);
    }
    const Shell sh = make_shell(b);
    const long nsh = sh.nA + sh.nB + sh.nC;
    k_bc<R><<<(unsigned)((nsh + 255) / 256), 256, 0, s>>>(b, C.P, C.g, S, C.sc, copyB, sh);
}

// CalcDT on a state without changing it (gam_calc_dt): min of CellDT over
// the dt range into sc->dtmin_bits.
template <class R>
__global__ void __launch_bounds__(128) k_dt_only(GamBox b, DevParams<R> P, Geo<R> g, StateBuf<R> s,
                                                 GamScalars* sc, double gamma_d, double gm1_d, int countBad) {
    int ii, jj, kk;
    const int G = GAM_NG;
    Range r{G - P.dtIlo, G + b.Nip - 1 + P.dtIhi, G - P.dtJlo, G + b.Njp - 1 + P.dtJhi, G - P.dtKlo,
            G + b.Nkp - 1 + P.dtKhi};
    double mydt = HUGE_DT;
    if (thread_ijk(r, ii, jj, kk) && GAM_BOX_OK(lidx(b, ii, jj, kk), lidx(b, ii, jj, kk), 13)) {
        const long fs = b.fs;
        const long c = lidx(b, ii, jj, kk);
        double Ud[5], Bt[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int v = 0; v < 5; v++) Ud[v] = (double)s.Gas[v * fs + c];
        if (P.doMHD) {
#pragma unroll
            for (int x = 0; x < 3; x++) {
                Bt[x] = (double)s.B[x * fs + c];
                if (P.doBackground) Bt[x] = Bt[x] + g.B0[x * fs + c];
            }
        }
        double dtc = P.doBoris ? cell_dt<R, true>(P, Ud, Bt, (double)g.dl[c], gamma_d, gm1_d, sc->CFL)
                                : cell_dt<R, false>(P, Ud, Bt, (double)g.dl[c], gamma_d, gm1_d, sc->CFL);
        if (dtc > 0.0 && dtc < 1.0e300) mydt = dtc;
        else if (countBad && !sc->fixedTimestep) atomicAdd(&sc->nbad, 1);
    }
    if (sc->fixedTimestep && countBad) return;
    for (int o = 16; o > 0; o >>= 1) mydt = fmin(mydt, __shfl_xor_sync(0xffffffffu, mydt, o));
    if ((threadIdx.x & 31) == 0 && mydt < HUGE_DT) atomicMin(&sc->dtmin_bits, dbits(mydt));
}


// bFlux2Fld over every cell of a state (gridutils.F90:281-301)
template <class R>
__global__ void __launch_bounds__(128) k_bfield_all(GamBox b, Geo<R> g, StateBuf<R> s, const GamScalars* sc,
                                                    RingData ring) {
    int ii, jj, kk;
    Range r{0, b.Ni - 1, 0, b.Nj - 1, 0, b.Nk - 1};
    if (!thread_ijk(r, ii, jj, kk)) return;
    const long fs = b.fs;
    const long c = lidx(b, ii, jj, kk);
    int jc = jj, kc = kk;
    const long cb = (ring.on && ring_conj_cc(b, ring, jc, kc)) ? lidx(b, ii, jc, kc) : c;
    GAM_BOX_CHECK(cb, cb + b.sk, 16);
    R B[3];
    cell_bxyz(b, g, cb, s.mf[cb], s.mf[cb + 1], s.mf[fs + cb], s.mf[fs + cb + b.sx], s.mf[2 * fs + cb],
              s.mf[2 * fs + cb + b.sk], B);
#pragma unroll
    for (int x = 0; x < 3; x++) s.B[x * fs + c] = B[x];
}

// ----------------------------------------------------------------- launches
static inline dim3 grid_for(const Range& r, dim3 blk) {
    return dim3((unsigned)((r.i1 - r.i0 + 1 + blk.x - 1) / blk.x), (unsigned)((r.j1 - r.j0 + 1 + blk.y - 1) / blk.y),
                (unsigned)((r.k1 - r.k0 + 1 + blk.z - 1) / blk.z));
}

// RingAverage (ringav.F90:26-75) on the updated state: smoothing EMFs of both
// poles, PoleE and FixEFieldLFM on them, E2Flux with dt = 1, CleanLoops,
// bFlux2Fld of the cells around the rings, SmoothGas of both poles
template <class R> void launch_ring_average(const Ctx<R>& C, const StateBuf<R>& O, cudaStream_t s) {
    const GamBox& b = C.b;
    const RingData& Rg = C.P.ring;
    const int G = GAM_NG;
    if (C.P.doMHD) {
        const long nz = 2L * (Rg.NumR + 2) * b.Ni * b.Nk;
        k_ring_zero_e<R><<<(unsigned)((nz + 255) / 256), 256, 0, s>>>(b, Rg, C.sc);
        const long ne = 2L * (b.Nip + 1) * Rg.NumR;
        const size_t smE = (size_t)(2 * Rg.Np + Rg.chunkStride / 5) * sizeof(R);
        k_ring_smooth_e<R><<<(unsigned)ne, 32, smE, s>>>(b, Rg, O, C.sc);
        R* E = (R*)Rg.smoothE;
        const int ni = b.Nip + 1;
        k_ring_pole_e<R><<<(unsigned)(2 * ni), 32, Rg.Np * sizeof(R), s>>>(b, Rg, E, G, G + b.Nip, C.sc);
        // FixEFieldLFM over the rows that can be nonzero (the others hold zeros)
        const int sj1 = std::min(G + Rg.NumR + 1, G + b.Njp), ej0 = std::max(G + b.Njp - 1 - Rg.NumR, G);
        if (Rg.doS)
            k_fix_e_lfm<R><<<(unsigned)(((long)ni * (sj1 - G + 1) + 255) / 256), 256, 0, s>>>(b, E, G, sj1, C.sc);
        if (Rg.doE)
            k_fix_e_lfm<R><<<(unsigned)(((long)ni * (G + b.Njp - ej0 + 1) + 255) / 256), 256, 0, s>>>(
                b, E, ej0, G + b.Njp, C.sc);
        const long nf = 2L * (Rg.NumR + 1) * (b.Nip + 1) * (b.Nkp + 1);
        k_ring_e2flux<R><<<(unsigned)((nf + 255) / 256), 256, 0, s>>>(b, Rg, O, C.sc);
        if (Rg.clean) k_ring_clean_loops<R><<<(unsigned)(2 * ni), 32, Rg.Np * sizeof(R), s>>>(b, Rg, O, C.sc);
        const long nb = 2L * (G + Rg.NumR + 2) * b.Ni * b.Nk;
        k_ring_bfield<R><<<(unsigned)((nb + 127) / 128), 128, 0, s>>>(b, C.g, Rg, O, C.sc);
    }
    const long ng = 2L * b.Nip * Rg.NumR;
    const size_t smG = (size_t)(5 * Rg.Np + Rg.chunkStride) * sizeof(R);
    k_ring_smooth_gas<R><<<(unsigned)ng, 32, smG, s>>>(b, C.P, O, C.sc);
}

// The kernels of one stepGamera in order, each handed to f(id, launch) with
// id: 0 begin, 1 predict, 2/3 mom2face/vxb I, 4/5 J, 6/7 K, 8/9/10 stress
// I/J/K, 11 update_faces, 12 update_cells, 13 dt_finalize, 14 bc.
// st[cur] is State (n); st[1-cur] holds oState (n-1) on entry and State
// (n+1) on exit.
template <class R, class F> void for_each_kernel(const Ctx<R>& C, int cur, cudaStream_t& s, F&& f) {
    const GamBox& b = C.b;
    const int G = GAM_NG;
    const StateBuf<R> S = C.st[cur], O = C.st[1 - cur];
    const dim3 blk(32, 4, 1);
    const dim3 sblk(16, 8, 1);  // flux kernels: 8 rows per block for the J-direction stencil reuse
    const Range all{0, b.Ni, 0, b.Nj, 0, b.Nk};
    const Range cells{0, b.Ni - 1, 0, b.Nj - 1, 0, b.Nk - 1};
    const int kke = C.P.do25D ? G : G + b.Nkp - 1;  // last active k of the stress sweep
    f(0, [&] { k_step_begin<<<1, 1, 0, s>>>(C.sc); });
    const dim3 pblk(32, 8, 1);
    f(1, [&] {
        if (C.P.doAB3)
            k_predict<R, sizeof(R) == 8 ? 3 : 4, true><<<grid_for(all, pblk), pblk, 0, s>>>(b, C.P, C.g, S, O, C.w, C.sc,
                                                                                          C.oomf);
        else if (C.kvar & 8)
            k_predict<R, 1><<<grid_for(all, pblk), pblk, 0, s>>>(b, C.P, C.g, S, O, C.w, C.sc, nullptr);
        else  // FP64: 3 blocks/SM (4 for the strict build, measured); FP32: 4
            k_predict<R, (sizeof(R) == 8 && !GAM_STRICT_KERNELS) ? 3 : 4><<<grid_for(all, pblk), pblk, 0, s>>>(
                b, C.P, C.g, S, O, C.w, C.sc, nullptr);
    });
    if (C.P.doMHD) {
        const Range mf[3] = {{0, b.Ni - 1, G, G + b.Njp, 0, b.Nk - 1},
                             {0, b.Ni - 1, 0, b.Nj - 1, G, G + b.Nkp},
                             {G, G + b.Nip, 0, b.Nj - 1, 0, b.Nk - 1}};
        const Range ed[3] = {{G, G + b.Nip - 1, G, G + b.Njp, G, G + b.Nkp},
                             {G, G + b.Nip, G, G + b.Njp - 1, G, G + b.Nkp},
                             {G, G + b.Nip, G, G + b.Njp, G, G + b.Nkp - 1}};
        for (int eD = 0; eD < 3; eD++) {
            // edge directions whose stencils run along k (Mom2Face of eD = 1, VxB of eD = 0, 1)
            const dim3 mb = (eD == 1 && (C.kvar & 1024)) ? dim3(32, 1, 4) : blk;
            const dim3 vb = (eD < 2 && (C.kvar & 512)) ? dim3(32, 1, 4) : blk;
            f(2 + 2 * eD, [&] { k_mom2face<R><<<grid_for(mf[eD], mb), mb, 0, s>>>(b, C.P, C.g, C.w, eD, mf[eD], C.sc); });
            f(3 + 2 * eD, [&] {
                if (C.kvar & 16)
                    k_vxb<R, 10><<<grid_for(ed[eD], vb), vb, 0, s>>>(b, C.P, C.g, C.w, eD, ed[eD], C.sc);
                else if ((C.kvar & 32) || sizeof(R) == 4)  // FP32: 12 blocks/SM (40 registers) measured best
                    k_vxb<R, 12><<<grid_for(ed[eD], vb), vb, 0, s>>>(b, C.P, C.g, C.w, eD, ed[eD], C.sc);
                else if (C.kvar & 128)
                    k_vxb<R><<<grid_for(ed[eD], vb), vb, 0, s>>>(b, C.P, C.g, C.w, eD, ed[eD], C.sc);
                else  // FP64: 8 blocks/SM (64 registers)
                    k_vxb<R, 8><<<grid_for(ed[eD], vb), vb, 0, s>>>(b, C.P, C.g, C.w, eD, ed[eD], C.sc);
            });
        }
    }
    const Range fr[3] = {{G, G + b.Nip, G, G + b.Njp - 1, G, kke},
                         {G, G + b.Nip - 1, G, G + b.Njp, G, kke},
                         {G, G + b.Nip - 1, G, G + b.Njp - 1, G, G + b.Nkp}};
    const R* Blim = C.P.doLFMLim ? S.B : C.w.Bl;
    auto stress = [&](auto Dc) {
        constexpr int D = decltype(Dc)::value;
        const Range& r = fr[D];
        // K sweep: blocks that extend along k share its 8-point stencil planes
        // in L1 (16x1x8 measured 5 % faster than 16x8x1 on the K sweep)
        const dim3 sbk = D != 2           ? sblk
                         : (C.kvar & 256)  ? sblk
                         : (C.kvar & 2048) ? dim3(32, 1, 4)
                         : (C.kvar & 4096) ? dim3(8, 1, 16)
                                           : dim3(16, 1, 8);
        if (C.P.doBoris) {
            k_stress<R, D, sizeof(R) == 4 ? 8 : 6, true><<<grid_for(r, sbk), sbk, 0, s>>>(b, C.P, C.g, Blim, C.w, r, C.sc,
                                                                                        S.Gas, O.Gas);
            return;
        }
        switch (C.kvar & 3) {
            case 1: k_stress<R, D, 1><<<grid_for(r, sbk), sbk, 0, s>>>(b, C.P, C.g, Blim, C.w, r, C.sc, S.Gas, O.Gas); break;
            case 2: k_stress<R, D, 7><<<grid_for(r, sbk), sbk, 0, s>>>(b, C.P, C.g, Blim, C.w, r, C.sc, S.Gas, O.Gas); break;
            case 3: k_stress<R, D, 8><<<grid_for(r, sbk), sbk, 0, s>>>(b, C.P, C.g, Blim, C.w, r, C.sc, S.Gas, O.Gas); break;
            // FP64: 8 blocks/SM for the I and J sweeps, 7 for K (measured); FP32: 8
            default: k_stress<R, D, (sizeof(R) == 4 || D < 2) ? 8 : 7><<<grid_for(r, sbk), sbk, 0, s>>>(b, C.P, C.g, Blim, C.w, r, C.sc, S.Gas, O.Gas); break;
        }
    };
    f(8, [&] { stress(std::integral_constant<int, 0>()); });
    f(9, [&] { stress(std::integral_constant<int, 1>()); });
    if (!C.P.do25D) f(10, [&] { stress(std::integral_constant<int, 2>()); });
    f(11, [&] {
        if (C.P.ion.on && C.P.doMHD) {  // HackE (EFix, earthcmi.F90:321-354)
            const long ne = (long)b.Nj * b.Nk, nf = (long)(b.Nip + 1) * (b.Njp + 1);
            if (C.P.bc[0] == BCK_ION)  // the inner tile (hasLowerBC(IDIR))
                k_ion_efix<R><<<(unsigned)((ne + 255) / 256), 256, 0, s>>>(b, C.P, C.w, C.sc);
            if (C.P.ion.wind) {
                const long nw = 4L * (b.Njp + 1) * (b.Nkp + 1);
                k_wind_efix<R><<<(unsigned)((nw + 255) / 256), 256, 0, s>>>(b, C.P, C.g, S, C.w, C.sc);
                if (C.P.ring.on)  // WindEFix's touch-up of the pole rows of its shells
                    k_ring_pole_e<R><<<8, 32, C.P.ring.Np * sizeof(R), s>>>(b, C.P.ring, C.w.E, GAM_NG + b.Nip - 3,
                                                                          GAM_NG + b.Nip, C.sc);
            }
            if (C.P.bc[4] != BCK_HALO)
                k_fix_e_lfm<R><<<(unsigned)((nf + 255) / 256), 256, 0, s>>>(b, C.w.E, GAM_NG, GAM_NG + b.Njp, C.sc);
        }
        if (C.P.ring.on && C.P.doMHD) {  // PoleE before E2Flux (mhdgroup.F90:140-142)
            const int ni = b.Nip + 1;
            k_ring_pole_e<R><<<(unsigned)(2 * ni), 32, C.P.ring.Np * sizeof(R), s>>>(b, C.P.ring, C.w.E, GAM_NG,
                                                                                    GAM_NG + b.Nip, C.sc);
            const long nf = (long)ni * (b.Njp + 1);
            k_fix_e_lfm<R><<<(unsigned)((nf + 255) / 256), 256, 0, s>>>(b, C.w.E, GAM_NG, GAM_NG + b.Njp, C.sc);
        }
        k_update_faces<R><<<grid_for(all, blk), blk, 0, s>>>(b, C.P, S, O, C.w, C.sc, C.oomf);
    });
    f(12, [&] {
        if (C.P.ring.on) {  // RingFlux (stress.F90:137-139), before the fluxes become deltas
            const long n = 2L * b.Ni * b.Nk + (long)b.Nip * b.Njp;
            k_ring_flux<R><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(b, C.P, C.w, C.sc);
            if (C.P.bc[0] == BCK_ION && C.P.ion.on)
                k_ion_flux<R><<<16, 32, C.P.ring.Np * sizeof(R), s>>>(b, C.P, C.w, C.sc);
        }
        if (C.P.doBoris)
            k_update_cells<R, sizeof(R) == 8 ? 6 : 8, true><<<grid_for(cells, blk), blk, 0, s>>>(b, C.P, C.g, S, O, C.w, C.sc, C.gamma, C.gm1);
        else if (C.kvar & 4)
            k_update_cells<R, 1><<<grid_for(cells, blk), blk, 0, s>>>(b, C.P, C.g, S, O, C.w, C.sc, C.gamma, C.gm1);
        else
            k_update_cells<R, 8><<<grid_for(cells, blk), blk, 0, s>>>(b, C.P, C.g, S, O, C.w, C.sc, C.gamma, C.gm1);
        if (C.P.ring.on) launch_ring_average(C, O, s);  // mhdgroup.F90:69-74
        if (C.P.ion.push) {  // HackStep (PerStep, earthcmi.F90:224-263): PushIon, before CalcDT
            const long np = (long)C.P.ion.nIonP * b.Njp * b.Nkp;
            if (C.P.doBoris)
                k_ion_push<R, true><<<(unsigned)((np + 127) / 128), 128, 0, s>>>(b, C.P, C.g, O, C.sc, C.gamma, C.gm1);
            else
                k_ion_push<R, false><<<(unsigned)((np + 127) / 128), 128, 0, s>>>(b, C.P, C.g, O, C.sc, C.gamma, C.gm1);
        }
        if (C.P.ion.wind) {  // HackStep, wind part: NudgeSW
            const long nn = (long)b.Njp * b.Nkp;
            if (C.P.doBoris)
                k_nudge_sw<R, true><<<(unsigned)((nn + 127) / 128), 128, 0, s>>>(b, C.P, C.g, O, C.sc, C.gamma, C.gm1);
            else
                k_nudge_sw<R, false><<<(unsigned)((nn + 127) / 128), 128, 0, s>>>(b, C.P, C.g, O, C.sc, C.gamma, C.gm1);
            if (C.P.ring.on && C.P.ring.doE)
                k_ring_nudge_axis<R><<<(unsigned)((2 * b.Nkp + 127) / 128), 128, 0, s>>>(b, C.P, O, C.sc);
        }
        if (C.P.ring.on) {  // CalcDT after the ring average and the hooks (gamapp.F90:78-80)
            const dim3 blk2(32, 4, 1);
            const Range r{GAM_NG - C.P.dtIlo, GAM_NG + b.Nip - 1 + C.P.dtIhi, GAM_NG - C.P.dtJlo,
                          GAM_NG + b.Njp - 1 + C.P.dtJhi, GAM_NG - C.P.dtKlo, GAM_NG + b.Nkp - 1 + C.P.dtKhi};
            k_dt_only<R><<<grid_for(r, blk2), blk2, 0, s>>>(b, C.P, C.g, O, C.sc, C.gamma, C.gm1, 1);
        }
    });
    f(13, [&] { k_dt_finalize<<<1, 1, 0, s>>>(C.sc); });
    f(14, [&] { launch_bcs(C, O, s, 0); });
}

// One step. With side streams (C.aux, C.ev) the independent kernels run as
// parallel branches of the captured graph: the three Mom2Face -> EMF chains
// (then the face update) beside the three flux directions; the cell update
// joins them. Every branch writes its own arrays, so the result is the same
// bits as the sequential order.
template <class R> void launch_step(const Ctx<R>& C, int cur, cudaStream_t s) {
    cudaStream_t cs = s;
    if (!C.aux[0] || (C.kvar & 64)) {
        for_each_kernel(C, cur, cs, [](int, auto&& L) { L(); });
        return;
    }
    for_each_kernel(C, cur, cs, [&](int id, auto&& L) {
        switch (id) {
            case 0:
            case 1:
                cs = s;
                L();
                if (id == 1) {
                    cudaEventRecord(C.ev[0], s);
                    for (int q = 0; q < 5; q++) cudaStreamWaitEvent(C.aux[q], C.ev[0], 0);
                }
                return;
            case 2: case 3: cs = C.aux[0]; break;
            case 4: case 5: cs = C.aux[1]; break;
            case 6: case 7: cs = C.aux[2]; break;
            case 8: cs = s; break;
            case 9: cs = C.aux[3]; break;
            case 10: cs = C.aux[4]; break;
            case 11:
                cudaEventRecord(C.ev[1], C.aux[1]);
                cudaEventRecord(C.ev[2], C.aux[2]);
                cudaStreamWaitEvent(C.aux[0], C.ev[1], 0);
                cudaStreamWaitEvent(C.aux[0], C.ev[2], 0);
                cs = C.aux[0];
                break;
            case 12:
                cudaEventRecord(C.ev[3], C.aux[0]);
                cudaEventRecord(C.ev[4], C.aux[3]);
                cudaEventRecord(C.ev[5], C.aux[4]);
                cudaStreamWaitEvent(s, C.ev[3], 0);
                cudaStreamWaitEvent(s, C.ev[4], 0);
                cudaStreamWaitEvent(s, C.ev[5], 0);
                cs = s;
                break;
            default: cs = s; break;
        }
        L();
    });
}

// Device time of each kernel of a step (ms, average of reps back-to-back
// launches; ms[15]). The kernels after k_step_begin read their inputs and
// write other arrays, so repeating one changes nothing; the time bookkeeping
// kernels are not run.
// The reference's clock label of each kernel id of for_each_kernel
// (gamapp.F90:96-99, mhdgroup.F90, fields.F90, stress.F90, step.F90 Tic/Toc)
inline const char* kernel_label(int id) {
    static const char* L[15] = {"Gamera", "Predictor", "Mom2Face", "VxB", "Mom2Face", "VxB", "Mom2Face", "VxB",
                                "Fluxes", "Fluxes", "Fluxes", "CT-Update", "Maxwell", "DT", "BCs"};
    return (id >= 0 && id < 15) ? L[id] : "Gamera";
}

template <class R> void profile_step(const Ctx<R>& C, int cur, cudaStream_t s, int reps, double* ms) {
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    for (int q = 0; q < 15; q++) ms[q] = 0.0;
    cudaStream_t cs = s;
    for_each_kernel(C, cur, cs, [&](int id, auto&& L) {
        if (id == 0 || id == 13) return;
        L();  // warm
        nvtxRangePushA(kernel_label(id));
        cudaEventRecord(e0, s);
        for (int r = 0; r < reps; r++) L();
        cudaEventRecord(e1, s);
        nvtxRangePop();
        cudaEventSynchronize(e1);
        float t = 0.f;
        cudaEventElapsedTime(&t, e0, e1);
        ms[id] = t / reps;
    });
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
}

// Kernel attributes that must be set before a launch is captured in a graph.
template <class R> void prepare() {}

// CalcDT on st[cur] into sc->dtmin_bits (the caller resets it first).
template <class R> void launch_dt_only(const Ctx<R>& C, int cur, cudaStream_t s) {
    const GamBox& b = C.b;
    const int G = GAM_NG;
    const dim3 blk(32, 4, 1);
    const Range r{G - C.P.dtIlo, G + b.Nip - 1 + C.P.dtIhi, G - C.P.dtJlo, G + b.Njp - 1 + C.P.dtJhi,
                  G - C.P.dtKlo, G + b.Nkp - 1 + C.P.dtKhi};
    k_dt_only<R><<<grid_for(r, blk), blk, 0, s>>>(b, C.P, C.g, C.st[cur], C.sc, C.gamma, C.gm1, 0);
}

// CalcGridInfo after the initial condition (init.F90:217-238): Bxyz from the
// fluxes, first EnforceBCs, oState = State.
// bFlux2Fld of State (st[cur]) over every cell (gridutils.F90:281-301)
template <class R> void launch_bfield(const Ctx<R>& C, int cur, cudaStream_t s) {
    const GamBox& b = C.b;
    const dim3 blk(32, 4, 1);
    const Range cells{0, b.Ni - 1, 0, b.Nj - 1, 0, b.Nk - 1};
    k_bfield_all<R><<<grid_for(cells, blk), blk, 0, s>>>(b, C.g, C.st[cur], C.sc, C.P.ring);
}

template <class R> void launch_init(const Ctx<R>& C, int cur, cudaStream_t s) {
    const GamBox& b = C.b;
    const dim3 blk(32, 4, 1);
    const Range all{0, b.Ni, 0, b.Nj, 0, b.Nk};
    const Range cells{0, b.Ni - 1, 0, b.Nj - 1, 0, b.Nk - 1};
    const StateBuf<R> S = C.st[cur], O = C.st[1 - cur];
    if (C.P.doMHD) k_bfield_all<R><<<grid_for(cells, blk), blk, 0, s>>>(b, C.g, S, C.sc, C.P.ring);
    launch_bcs(C, S, s, 1);
    cudaMemcpyAsync(O.Gas, S.Gas, 5 * b.fs * sizeof(R), cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(O.mf, S.mf, 3 * b.fs * sizeof(R), cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(O.B, S.B, 3 * b.fs * sizeof(R), cudaMemcpyDeviceToDevice, s);
    if (C.oomf) cudaMemcpyAsync(C.oomf, S.mf, 3 * b.fs * sizeof(R), cudaMemcpyDeviceToDevice, s);  // ooState = State
}

// ----------------------------------------------------------------- k-slab tiling
// One step in two phases for a caller that reduces dt over several domains:
// phase 0 = begin .. cell update (the dt candidates in sc->dtmin_bits and
// sc->nbad), phase 1 = dt decision and boundary fill. The caller writes the
// global min / count into sc between them (gamapp_mpi.F90:495-512).
template <class R> void launch_step_phase(const Ctx<R>& C, int cur, cudaStream_t s, int phase) {
    cudaStream_t cs = s;
    for_each_kernel(C, cur, cs, [&](int id, auto&& L) {
        if ((id <= 12) == (phase == 0)) L();
    });
}

// Halo of a tile (the depth-4 exchange of updateMpiBCs/haloUpdate,
// gamapp_mpi.F90:573-782) along direction d (0 I, 1 J, 2 K): 11 components
// (Gas 0-4, magFlux 5-7, Bxyz 8-10) x 4 layers along d x the full ghosted
// face-box extents (u, v) of the other two directions (u the lower of the
// two), element (q, l, v, u) at ((q * 4 + l) * nv + v) * nu + u. Pack side 0
// = what this tile sends down (cells and the other faces at G..G+3 along d,
// d-faces at G+1..G+4: the neighbour's upper ghosts); side 1 = what it sends
// up (everything at Nd..Nd+3: the neighbour's lower ghosts). Unpack side 0
// fills this tile's lower ghosts (0..3), side 1 its upper ghosts (cells and
// the other faces at G+Nd.., d-faces at G+Nd+1..), the indices the periodic
// rules of bcs.F90:279-450 use. Exchanging I, then J, then K with the full
// extents carries the edge and corner ghosts through the earlier exchanges.
// The k-slab API's sides are d = 2.
__device__ __forceinline__ int halo_pos(const GamBox& b, int d, int side, bool unpack, int q, int l) {
    const int G = GAM_NG;
    const int Nd = d == 0 ? b.Nip : (d == 1 ? b.Njp : b.Nkp);
    const bool dface = q == 5 + d;
    if (!unpack) return side == 0 ? G + l + (dface ? 1 : 0) : Nd + l;
    return side == 0 ? l : G + Nd + l + (dface ? 1 : 0);
}
template <class R> __device__ __forceinline__ R* halo_ptr(const StateBuf<R>& S, long fs, int q) {
    return q < 5 ? S.Gas + (long)q * fs : (q < 8 ? S.mf + (long)(q - 5) * fs : S.B + (long)(q - 8) * fs);
}
// face-box extents across direction d: nu (the lower other direction), nv
__host__ __device__ __forceinline__ void halo_extents(const GamBox& b, int d, long& nu, long& nv) {
    nu = d == 0 ? b.Nj + 1 : b.Ni + 1;
    nv = d == 2 ? b.Nj + 1 : b.Nk + 1;
}
__device__ __forceinline__ long halo_cell(const GamBox& b, int d, int pos, int u, int v) {
    return d == 0 ? lidx(b, pos, u, v) : (d == 1 ? lidx(b, u, pos, v) : lidx(b, u, v, pos));
}
template <class R>
__global__ void __launch_bounds__(256) k_halo(GamBox b, StateBuf<R> S, R* __restrict__ buf, int d, int side,
                                              int unpack, int copyB, const GamScalars* sc) {
    if (sc->halted) return;  // a failed step keeps its state, ghosts included
    long nu, nv;
    halo_extents(b, d, nu, nv);
    const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (t >= 4 * nu * nv) return;
    const int u = (int)(t % nu), v = (int)((t / nu) % nv), l = (int)(t / (nu * nv));
    const long fs = b.fs;
    for (int q = 0; q < 11; q++) {
        if (unpack && q >= 8 && !copyB) break;
        const long c = halo_cell(b, d, halo_pos(b, d, side, unpack != 0, q, l), u, v);
        GAM_BOX_CHECK(c, c, 15);
        const long e = ((long)(q * 4 + l) * nv + v) * nu + u;
        R* p = halo_ptr(S, fs, q);
        if (unpack)
            p[c] = buf[e];
        else
            buf[e] = p[c];
    }
}
// Bxyz of the unpacked ghost cells from their faces (the final bFlux2Fld)
template <class R>
__global__ void __launch_bounds__(256) k_halo_bxyz(GamBox b, Geo<R> g, StateBuf<R> S, int d, int side,
                                                   const GamScalars* sc, RingData ring) {
    if (sc->halted) return;
    const long nu = d == 0 ? b.Nj : b.Ni, nv = d == 2 ? b.Nj : b.Nk;  // cell extents
    const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (t >= 4 * nu * nv) return;
    const int u = (int)(t % nu), v = (int)((t / nu) % nv), l = (int)(t / (nu * nv));
    const int Nd = d == 0 ? b.Nip : (d == 1 ? b.Njp : b.Nkp);
    const int pos = side == 0 ? l : GAM_NG + Nd + l;
    const long fs = b.fs, c = halo_cell(b, d, pos, u, v);
    // a ghost across the LFM pole takes its conjugate's field
    const int ic = d == 0 ? pos : u;
    int jc = d == 1 ? pos : (d == 0 ? u : v), kc = d == 2 ? pos : v;
    const long cb = (ring.on && ring_conj_cc(b, ring, jc, kc)) ? lidx(b, ic, jc, kc) : c;
    GAM_BOX_CHECK(cb, cb + b.sk, 15);
    R B[3];
    cell_bxyz(b, g, cb, S.mf[cb], S.mf[cb + 1], S.mf[fs + cb], S.mf[fs + cb + b.sx], S.mf[2 * fs + cb],
              S.mf[2 * fs + cb + b.sk], B);
#pragma unroll
    for (int x = 0; x < 3; x++) S.B[x * fs + c] = B[x];
}
// dside = side + 2 d
template <class R> void launch_halo(const Ctx<R>& C, int cur, cudaStream_t s, int dside, int unpack, int copyB, void* buf) {
    const GamBox& b = C.b;
    const int d = dside >> 1, side = dside & 1;
    const StateBuf<R> S = C.st[cur];
    long nu, nv;
    halo_extents(b, d, nu, nv);
    const long n = 4L * nu * nv;
    k_halo<R><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(b, S, (R*)buf, d, side, unpack, copyB, C.sc);
    if (unpack && !copyB && C.P.doMHD) {
        const long m = 4L * (d == 0 ? b.Nj : b.Ni) * (d == 2 ? b.Nj : b.Nk);
        k_halo_bxyz<R><<<(unsigned)((m + 255) / 256), 256, 0, s>>>(b, C.g, S, d, side, C.sc, C.P.ring);
    }
}

}  // namespace GAM_NS
