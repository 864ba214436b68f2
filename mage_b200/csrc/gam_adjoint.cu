// Flux stage of the step (CalcStress / Fluxes / GasKinFlux / MagKinFlux,
// stress.F90:41-599, with Cen8LRs + pdmLR, recon.F90:125-272) and its
// hand-written reverse mode, on caller-owned device arrays in the unpadded box
// layout (component-major (nc, Nk+1, Nj+1, Ni+1), i fastest). The forward is
// the product step's own flux kernel; the adjoint recomputes each face's
// states and fluxes and runs them backwards:
//   outputs  gF (15: v + 5*d), mF (9: x + 3*d), already times the face area
//   inputs   QW = volume * half-state primitives (5), Wn limiter primitives (5),
//            QB = volume * half-state Bxyz (3), Blim limiter Bxyz (3),
//            Bnf = half-state flux / area (3)
// The adjoint accumulates (atomicAdd) into dQW, dWn, dQB, dBlim, dBnf, which
// the caller zeroes. Non-smooth points follow the forward's branches: a
// max/min passes the adjoint to the operand it selected, |x| and sign(x) have
// a zero derivative at 0, sqrt(Va^2) a zero derivative at 0.
#include <string.h>
#define GAM_NS gam_adj
#define GAM_CUDA_MATH 1
#include "gam_step_impl.cuh"

namespace gam_adj {

__device__ GamScalars g_adj_scalars;  // zero: not halted

// the stage scalars, written on the stream by a kernel from its arguments
// (a copy from host memory would make the host wait for the stream)
__global__ void k_adj_scalars(GamScalars* sc, double dt, double pdt, double odt, int fixedTimestep) {
    *sc = GamScalars{};
    sc->dt = dt;
    sc->pdt = pdt;
    sc->odt = odt;
    sc->fixedTimestep = fixedTimestep;
}

template <class A> __device__ __forceinline__ A sgnz(A x) { return x > (A)0 ? (A)1 : (x < (A)0 ? (A)-1 : (A)0); }

// reverse of lrs_from_qdv (8CENT) for one variable: scatter the adjoints of
// Ql, Qr to the 8-point operand stencil and the 4-point limiter stencil
template <class R, class A>
__device__ void lrs_adj(R pdmb, const R* qdv, const R* v, R Vi, A rVi, A aL, A aR, A* aq,
                        A* av, A* a_scale = nullptr) {
    R s = (R)0;
#pragma unroll
    for (int n = 0; n < 8; n++) s += Rc<R>(w8(n)) * qdv[n];
    const R Qi = s / Vi;
    const R v0 = v[0], v1 = v[1], v2 = v[2], v3 = v[3];
    const R maxV = rmax(v1, v2), minV = rmin(v1, v2);
    const R t = rmin(Qi, maxV);
    const R vN = rmax(minV, t);
    const R dv0 = pdmb * (v1 - v0), dv1 = pdmb * (v2 - v1), dv2 = pdmb * (v3 - v2);
    const R s0 = sgn1(dv0), s1 = sgn1(dv1), s2 = sgn1(dv2);
    const R q0 = fabs(s0 + s1), q1 = fabs(s1 + s2);
    const R dvL = vN - v1, dvR = v2 - vN;
    const R uL = fabs(dvL) - q0 * fabs(dv0), uR = fabs(dvR) - q1 * fabs(dv2);
    A a_vN = aL + aR;
    const A a_mL = -(A)s1 * aL, a_mR = (A)s1 * aR;
    const A a_uL = ((R)0 < uL) ? a_mL : (A)0.0, a_uR = ((R)0 < uR) ? a_mR : (A)0.0;
    const A a_dvL = a_uL * sgnz((A)dvL), a_dv0 = -a_uL * q0 * sgnz((A)dv0);
    const A a_dvR = a_uR * sgnz((A)dvR), a_dv2 = -a_uR * q1 * sgnz((A)dv2);
    A a0 = (A)0.0, a1 = (A)0.0, a2 = (A)0.0, a3 = (A)0.0;
    a_vN += a_dvL;
    a1 -= a_dvL;
    a2 += a_dvR;
    a_vN -= a_dvR;
    a1 += pdmb * a_dv0;
    a0 -= pdmb * a_dv0;
    a3 += pdmb * a_dv2;
    a2 -= pdmb * a_dv2;
    A a_t = (A)0.0, a_minV = (A)0.0, a_maxV = (A)0.0, a_Qi = (A)0.0;
    if (minV < t) a_t = a_vN; else a_minV = a_vN;
    if (maxV < Qi) a_maxV = a_t; else a_Qi = a_t;
    if (v2 < v1) a2 += a_minV; else a1 += a_minV;
    if (v1 < v2) a2 += a_maxV; else a1 += a_maxV;
    const A a_s = a_Qi * rVi;
    if (a_scale) *a_scale = a_s;  // aq[n] = w8(n) * a_s
#pragma unroll
    for (int n = 0; n < 8; n++) aq[n] = (A)w8(n) * a_s;
    av[0] = a0; av[1] = a1; av[2] = a2; av[3] = a3;
}

// reverse of mag_kin_flux for one side: adjoints aM (of the mF sums) and aVaD
// (of the VaD sum) -> a_W (5), a_B (3), a_Bn
template <class R, class A>
__device__ void mag_adj(const DevParams<R>& P, A sgn, const R* W, const R* Bm, R Bn, const R* T, const double* B0d,
                        double B0nd, const A* aM, A aVaD, A* aW, A* aB, A& aBn) {
    const A B0[3] = {(A)B0d[0], (A)B0d[1], (A)B0d[2]}, B0n = (A)B0nd;
    const A D = W[0], Pr = W[4];
    const A Bx = Bm[0], By = Bm[1], Bz = Bm[2];
    const A N[3] = {T[0], T[1], T[2]};
    const A dPb = (A)0.5 * (Bx * Bx + By * By + Bz * Bz);
    const A rD = (A)1.0 / D;
    A S[3] = {Bx, By, Bz};
    A Va2;
    if (P.doBackground) {
        S[0] += B0[0]; S[1] += B0[1]; S[2] += B0[2];
        Va2 = (S[0] * S[0] + S[1] * S[1] + S[2] * S[2]) * rD;
    } else {
        Va2 = (A)2.0 * dPb * rD;
    }
    const A Vn = N[0] * W[1] + N[1] * W[2] + N[2] * W[3];
    const A den = (A)2.0 * Pr * rD + Va2;
    const A lam = (A)1.0 / den;
    const A s = Mth<A>::sqrt_(lam);
    const A rs = Mth<A>::sqrt_(den);  // 1 / s
    const A z = sgn * s * Vn;
    const A Vn0 = (A)0.5 * Mth<A>::erfc_(z);
    const A B[3] = {Bx, By, Bz};
    A C[3];
    for (int x = 0; x < 3; x++) C[x] = dPb * N[x] - B[x] * (A)Bn;
    A BdB0 = (A)0.0;
    if (P.doBackground) {
        BdB0 = B0[0] * Bx + B0[1] * By + B0[2] * Bz;
        for (int x = 0; x < 3; x++) C[x] += -(B0[x] * (A)Bn) - B[x] * B0n + BdB0 * N[x];
    }
    A a_Vn0 = (A)0.0, a_dPb = (A)0.0, a_Va2 = (A)0.0, a_Vn = (A)0.0, sumCN = (A)0.0;
    for (int x = 0; x < 3; x++) {
        a_Vn0 += aM[x] * C[x];
        const A aC = aM[x] * Vn0;
        a_dPb += aC * N[x];
        aB[x] += -aC * (A)Bn;
        aBn += -aC * B[x];
        if (P.doBackground) {
            aB[x] += -aC * B0n;
            aBn += -aC * B0[x];
            sumCN += aC * N[x];
        }
    }
    if (P.doBackground)
        for (int x = 0; x < 3; x++) aB[x] += sumCN * B0[x];
    if (Va2 > (A)0.0) a_Va2 += aVaD * (A)0.25 / Mth<A>::sqrt_(Va2);
    const A a_z = a_Vn0 * (-Mth<A>::exp_(-z * z) * ((A)1.0 / Mth<A>::sqrt_((A)PI_D)));
    const A a_s = a_z * sgn * Vn;
    a_Vn += a_z * sgn * s;
    const A a_lam = a_s * (A)0.5 * rs;
    const A a_den = -a_lam * lam * lam;
    aW[4] += a_den * (A)2.0 * rD;
    aW[0] += -a_den * (A)2.0 * Pr * rD * rD;
    a_Va2 += a_den;
    if (P.doBackground) {
        for (int x = 0; x < 3; x++) aB[x] += a_Va2 * (A)2.0 * S[x] * rD;
        aW[0] += -a_Va2 * (S[0] * S[0] + S[1] * S[1] + S[2] * S[2]) * rD * rD;
    } else {
        a_dPb += a_Va2 * (A)2.0 * rD;
        aW[0] += -a_Va2 * (A)2.0 * dPb * rD * rD;
    }
    for (int x = 0; x < 3; x++) {
        aW[1 + x] += a_Vn * N[x];
        aB[x] += a_dPb * B[x];
    }
}

// reverse of gas_kin_flux for one side: adjoints aG (of the gF sums) and aD
// (of the dW sums) -> a_W (5)
template <class R, class A>
__device__ void gas_adj(const DevParams<R>& P, A sgn, const R* W, const R* T, const A* aG, const A* aDW,
                        A* aW) {
    const A D = W[0], Pr = W[4], V[3] = {W[1], W[2], W[3]};
    const A gm1 = P.gm1, rgm1 = (A)1.0 / gm1;
    const A V2 = V[0] * V[0] + V[1] * V[1] + V[2] * V[2];
    const A E = (A)0.5 * D * V2 + Pr * rgm1;
    const A r2P = (A)1.0 / ((A)2.0 * Pr);
    const A lam = D * r2P;
    A N[3], T1[3], T2[3];
    for (int x = 0; x < 3; x++) { N[x] = T[x]; T1[x] = T[3 + x]; T2[x] = T[6 + x]; }
    const A Vn = N[0] * V[0] + N[1] * V[1] + N[2] * V[2];
    const A Vt1 = T1[0] * V[0] + T1[1] * V[1] + T1[2] * V[2];
    const A Vt2 = T2[0] * V[0] + T2[1] * V[1] + T2[2] * V[2];
    const A s = Mth<A>::sqrt_(lam);
    const A rs = (A)1.0 / s;
    const A z = sgn * s * Vn;
    const A Vn0 = (A)0.5 * Mth<A>::erfc_(z);
    const A ex = Mth<A>::exp_(-(lam * Vn * Vn));
    const A sq = Mth<A>::sqrt_((A)PI_D) * s;
    const A rsq = rs * ((A)1.0 / Mth<A>::sqrt_((A)PI_D));
    const A Vn1 = Vn * Vn0 - (A)0.5 * sgn * ex * rsq;
    A a_fMn = (A)0.0, a_fMt1 = (A)0.0, a_fMt2 = (A)0.0;
    for (int x = 0; x < 3; x++) {
        a_fMn += aG[1 + x] * N[x];
        a_fMt1 += aG[1 + x] * T1[x];
        a_fMt2 += aG[1 + x] * T2[x];
    }
    A a_Vn1 = aG[0] * D + aG[4] * (E + (A)0.5 * Pr) + a_fMn * D * Vn + a_fMt1 * D * Vt1 + a_fMt2 * D * Vt2;
    A a_Vn0 = aG[4] * (A)0.5 * Pr * Vn + a_fMn * Pr;
    A a_D = aG[0] * Vn1 + a_fMn * Vn * Vn1 + a_fMt1 * Vt1 * Vn1 + a_fMt2 * Vt2 * Vn1 + aDW[0] * sgn;
    for (int x = 0; x < 3; x++) a_D += aDW[1 + x] * sgn * V[x];
    const A a_E = aG[4] * Vn1 + aDW[4] * sgn;
    A a_Pr = aG[4] * ((A)0.5 * Vn1 + (A)0.5 * Vn0 * Vn) + a_fMn * Vn0;
    A a_Vn = aG[4] * (A)0.5 * Pr * Vn0 + a_fMn * D * Vn1;
    const A a_Vt1 = a_fMt1 * D * Vn1, a_Vt2 = a_fMt2 * D * Vn1;
    A a_V[3];
    for (int x = 0; x < 3; x++) a_V[x] = aDW[1 + x] * sgn * D;
    // Vn1 = Vn Vn0 - (A)0.5 sgn ex / sq
    a_Vn += a_Vn1 * Vn0;
    a_Vn0 += a_Vn1 * Vn;
    const A a_ex = -a_Vn1 * (A)0.5 * sgn * rsq;
    const A a_sq = a_Vn1 * (A)0.5 * sgn * ex * rsq * rsq;
    A a_lam = a_sq * (A)PI_D * (A)0.5 * rsq;
    a_lam += -a_ex * ex * Vn * Vn;
    a_Vn += -a_ex * ex * (A)2.0 * lam * Vn;
    const A a_z = a_Vn0 * (-Mth<A>::exp_(-z * z) * ((A)1.0 / Mth<A>::sqrt_((A)PI_D)));
    const A a_s = a_z * sgn * Vn;
    a_Vn += a_z * sgn * s;
    a_lam += a_s * (A)0.5 * rs;
    a_D += a_lam * r2P;
    a_Pr += -a_lam * D * (A)2.0 * r2P * r2P;
    a_D += a_E * (A)0.5 * V2;
    for (int x = 0; x < 3; x++) a_V[x] += a_E * D * V[x];
    a_Pr += a_E * rgm1;
    for (int x = 0; x < 3; x++) a_V[x] += a_Vn * N[x] + a_Vt1 * T1[x] + a_Vt2 * T2[x];
    aW[0] += a_D;
    aW[1] += a_V[0];
    aW[2] += a_V[1];
    aW[3] += a_V[2];
    aW[4] += a_Pr;
}

// Adjoint of the face fluxes of direction D over the range r (one face per
// thread): recompute (SAVED: load the face states the forward stored in
// w.fsv), then reverse. 4 (FP64) / 6 (FP32) blocks per SM: the unbounded
// recomputing kernel took 214-240 registers (2 blocks); bounded it spills
// (local memory, L1-resident) but hides more load latency (measured on
// 128^3: 3 -> 4 FP64 blocks took the adjoint step from 5.9 to 5.7 ms; with
// the saved states, 5 -> 6 FP32 blocks about 1 %).
template <class R, int D, bool SAVED = false>
__global__ void __launch_bounds__(128, (sizeof(R) == 8 ? 4 : 6)) k_stress_adj(GamBox b, DevParams<R> P, Geo<R> g, const R* __restrict__ Blim,
                                                    Work<R> w, Range r, const R* __restrict__ dgF,
                                                    const R* __restrict__ dmF, R* dQW, R* dWn, R* dQB, R* dBlim,
                                                    R* dBnf, R* __restrict__ rs) {
    int ii, jj, kk;
    if (!thread_ijk(r, ii, jj, kk)) return;
    const long fs = b.fs;
    const long c = lidx(b, ii, jj, kk);
    const long s = D == 0 ? 1L : (D == 1 ? (long)b.sx : b.sk);
    R T[9];
    for (int n = 0; n < 9; n++) T[n] = g.Tf[(n + 9 * D) * fs + c];
    const R fa = g.face[D * fs + c];
    R vol[8];
    for (int n = 0; n < 8; n++) vol[n] = g.vol[c + (n - 4) * s];
    const R Vi = central8(vol);
    R WL[5], WR[5], MagL[3] = {(R)0, (R)0, (R)0}, MagR[3] = {(R)0, (R)0, (R)0};
    R Bn = (R)0;
    double B0[3] = {0.0, 0.0, 0.0}, B0n = 0.0;
    if (P.doMHD) {
        Bn = w.Bnf[D * fs + c];
        if (P.doBackground) {
            for (int x = 0; x < 3; x++) B0[x] = g.fcB0[(x + 3 * D) * fs + c];
            B0n = g.bFlux0[D * fs + c] / (double)fa;
        }
    }
    R VaD = (R)0, dW[5] = {(R)0, (R)0, (R)0, (R)0, (R)0};
    if constexpr (SAVED) {
        const R* o = w.fsv + (long)(GAM_FSV_NC * D) * fs + c;
        for (int v = 0; v < 5; v++) {
            WL[v] = o[v * fs];
            WR[v] = o[(5 + v) * fs];
            dW[v] = o[(17 + v) * fs];
        }
        for (int x = 0; x < 3; x++) {
            MagL[x] = o[(10 + x) * fs];
            MagR[x] = o[(13 + x) * fs];
        }
        VaD = o[16 * fs];
    } else {
        // forward states; the stencils are loaded again for the reverse of
        // the reconstruction rather than kept live (fewer registers, more warps)
        const Quot<R> qVi(Vi);  // the 8 reconstructions share the divisor
        for (int v = 0; v < 5; v++) {
            R qW[8], nW[4];
            for (int n = 0; n < 8; n++) qW[n] = w.QW[v * fs + c + (n - 4) * s];
            for (int m = 0; m < 4; m++) nW[m] = w.Wn[v * fs + c + (m - 2) * s];
            lrs_from_qdv(P, qW, nW, qVi, WL[v], WR[v]);
        }
        if (P.doMHD) {
            for (int x = 0; x < 3; x++) {
                R qB[8], nB[4];
                for (int n = 0; n < 8; n++) qB[n] = w.QB[x * fs + c + (n - 4) * s];
                for (int m = 0; m < 4; m++) nB[m] = Blim[x * fs + c + (m - 2) * s];
                lrs_from_qdv(P, qB, nB, qVi, MagL[x], MagR[x]);
            }
            R mFs[3] = {(R)0, (R)0, (R)0}, bbD = (R)0;
            mag_kin_flux(P, (R)-1, WL, MagL, Bn, T, B0, B0n, mFs, bbD, VaD);
            mag_kin_flux(P, (R)1, WR, MagR, Bn, T, B0, B0n, mFs, bbD, VaD);
        }
        R gFs[5] = {(R)0, (R)0, (R)0, (R)0, (R)0};
        gas_kin_flux(P, (R)-1, WL, T, gFs, dW);
        gas_kin_flux(P, (R)1, WR, T, gFs, dW);
    }
    // reverse of the outputs gF = fa (gFs - cHogH VaD dW), mF = fa mFs
    // in the form's precision (A = R): FP64 for the drop-in, FP32 for the FP32 form
    using A = R;
    A aG[5], aDW[5], aVaD = (A)0, aM[3] = {(A)0, (A)0, (A)0};
    for (int v = 0; v < 5; v++) {
        const A Gv = dgF[(v + 5 * D) * fs + c];
        aG[v] = (A)fa * Gv;
        aDW[v] = -(A)fa * (A)P.cHogH * (A)VaD * Gv;
        aVaD += -(A)fa * (A)P.cHogH * Gv * (A)dW[v];
    }
    A aWL[5] = {0, 0, 0, 0, 0}, aWR[5] = {0, 0, 0, 0, 0}, aBL[3] = {0, 0, 0}, aBR[3] = {0, 0, 0}, aBn = (A)0;
    gas_adj(P, (A)-1, WL, T, aG, aDW, aWL);
    gas_adj(P, (A)1, WR, T, aG, aDW, aWR);
    if (P.doMHD) {
        for (int x = 0; x < 3; x++) aM[x] = (A)fa * dmF[(x + 3 * D) * fs + c];
        mag_adj(P, (A)-1, WL, MagL, Bn, T, B0, B0n, aM, aVaD, aWL, aBL, aBn);
        mag_adj(P, (A)1, WR, MagR, Bn, T, B0, B0n, aM, aVaD, aWR, aBR, aBn);
        dBnf[D * fs + c] += (R)aBn;
    }
    // reverse of the reconstruction: scatter to the stencils
    A aq[8], av[4];
    const A rVi = (A)1 / (A)Vi;
    for (int v = 0; v < 5; v++) {
        R qW[8], nW[4];
        for (int n = 0; n < 8; n++) qW[n] = w.QW[v * fs + c + (n - 4) * s];
        for (int m = 0; m < 4; m++) nW[m] = w.Wn[v * fs + c + (m - 2) * s];
        A as;
        lrs_adj(P.pdmb, qW, nW, Vi, rVi, aWL[v], aWR[v], aq, av, &as);
        if (rs) {  // per face: the stencil weight scale and the 4 limiter adjoints
            rs[(5 * v) * fs + c] = (R)as;
            for (int m = 0; m < 4; m++) rs[(5 * v + 1 + m) * fs + c] = (R)av[m];
            continue;
        }
        for (int n = 0; n < 8; n++) atomicAdd(&dQW[v * fs + c + (n - 4) * s], (R)aq[n]);
        for (int m = 0; m < 4; m++) atomicAdd(&dWn[v * fs + c + (m - 2) * s], (R)av[m]);
    }
    if (P.doMHD)
        for (int x = 0; x < 3; x++) {
            R qB[8], nB[4];
            for (int n = 0; n < 8; n++) qB[n] = w.QB[x * fs + c + (n - 4) * s];
            for (int m = 0; m < 4; m++) nB[m] = Blim[x * fs + c + (m - 2) * s];
            A as;
            lrs_adj(P.pdmb, qB, nB, Vi, rVi, aBL[x], aBR[x], aq, av, &as);
            if (rs) {
                rs[(5 * (5 + x)) * fs + c] = (R)as;
                for (int m = 0; m < 4; m++) rs[(5 * (5 + x) + 1 + m) * fs + c] = (R)av[m];
                continue;
            }
            for (int n = 0; n < 8; n++) atomicAdd(&dQB[x * fs + c + (n - 4) * s], (R)aq[n]);
            for (int m = 0; m < 4; m++) atomicAdd(&dBlim[x * fs + c + (m - 2) * s], (R)av[m]);
        }
}


// The stencil adjoints of the faces of all three directions gathered per
// cell, in a fixed order (deterministic, no atomics), and stored: cell c is
// point n of the 8-point operand stencil of face c + (4 - n) e_D (adjoint
// w8(n) * scale of that face) and point m of the 4-point limiter stencil of
// face c + (2 - m) e_D; faces outside the range r[D] carry nothing. rs holds
// per direction D (40 components from 40 D) per face and variable (0-4
// QW/Wn, 5-7 QB/Blim) the scale and the 4 limiter adjoints. The sums run
// over n (m) per direction, then I, J, K, as three passes adding into a
// zeroed array would.
template <class R>
__global__ void __launch_bounds__(256) k_stress_adj_gather3(GamBox b, Range r0, Range r1, Range r2,
                                                            const R* __restrict__ rs, int nvar, R* __restrict__ dQW,
                                                            R* __restrict__ dWn, R* __restrict__ dQB,
                                                            R* __restrict__ dBlim) {
    using A = R;
    int ii, jj, kk;
    const Range all{0, b.Ni - 1, 0, b.Nj - 1, 0, b.Nk - 1};
    if (!thread_ijk(all, ii, jj, kk)) return;
    const int p[3] = {ii, jj, kk};
    const Range rr[3] = {r0, r1, r2};
    bool line[3];
#pragma unroll
    for (int D = 0; D < 3; D++) {
        const int lo[3] = {rr[D].i0, rr[D].j0, rr[D].k0}, hi[3] = {rr[D].i1, rr[D].j1, rr[D].k1};
        bool ok = p[D] >= lo[D] - 4 && p[D] <= hi[D] + 3;
        for (int a = 0; a < 3; a++)
            if (a != D && (p[a] < lo[a] || p[a] > hi[a])) ok = false;
        line[D] = ok;
    }
    const long fs = b.fs;
    const long c = lidx(b, ii, jj, kk);
    for (int v = 0; v < nvar; v++) {
        A qs[3], ls[3];
#pragma unroll
        for (int D = 0; D < 3; D++) {
            const long s = D == 0 ? 1L : (D == 1 ? (long)b.sx : b.sk);
            const int lo = D == 0 ? rr[D].i0 : (D == 1 ? rr[D].j0 : rr[D].k0);
            const int hi = D == 0 ? rr[D].i1 : (D == 1 ? rr[D].j1 : rr[D].k1);
            const R* q0 = rs + (40 * D + 5 * v) * fs + c;
            A q = (A)0, l = (A)0;
            if (line[D] && p[D] - 3 >= lo && p[D] + 4 <= hi) {
                // every face of both stencils in range: loads first, then the sums
                R x[8], y[4];
#pragma unroll
                for (int n = 0; n < 8; n++) x[n] = q0[(4 - n) * s];
#pragma unroll
                for (int m = 0; m < 4; m++) y[m] = q0[(1 + m) * fs + (2 - m) * s];
#pragma unroll
                for (int n = 0; n < 8; n++) q += (A)w8(n) * (A)x[n];
#pragma unroll
                for (int m = 0; m < 4; m++) l += (A)y[m];
            } else if (line[D]) {
#pragma unroll
                for (int n = 0; n < 8; n++) {
                    const int f = p[D] + 4 - n;
                    if (f >= lo && f <= hi) q += (A)w8(n) * (A)q0[(4 - n) * s];
                }
#pragma unroll
                for (int m = 0; m < 4; m++) {
                    const int f = p[D] + 2 - m;
                    if (f >= lo && f <= hi) l += (A)q0[(1 + m) * fs + (2 - m) * s];
                }
            }
            qs[D] = q;
            ls[D] = l;
        }
        A q = (A)0, l = (A)0;
#pragma unroll
        for (int D = 0; D < 3; D++)
            if (line[D]) {
                q += qs[D];
                l += ls[D];
            }
        R* dq = v < 5 ? dQW + v * fs : dQB + (v - 5) * fs;
        R* dl = v < 5 ? dWn + v * fs : dBlim + (v - 5) * fs;
        dq[c] = (R)q;
        dl[c] = (R)l;
    }
}


// reverse of edge_lrs (EdgeLRs for faces of direction a along bd): adjoints of
// bL*Vi, bR*Vi -> the abh (8) and bn (4) stencils
template <class R, class A>
__device__ void edge_lrs_adj(const GamBox& b, const DevParams<R>& P, const Geo<R>& g, const Work<R>& w, long c, int a,
                             int bd, A aBL, A aBR, R* dabh, R* dbn, R* es = nullptr) {
    const long fs = b.fs;
    const long s = dstride(b, bd);
    R qdv[8], area[8], nmag[4];
    for (int n = 0; n < 8; n++) {
        area[n] = g.face[a * fs + c + (n - 4) * s];
        qdv[n] = w.abh[a * fs + c + (n - 4) * s];
    }
    for (int m = 0; m < 4; m++) nmag[m] = w.bn[a * fs + c + (m - 2) * s];
    const R Vi = central8(area);
    A aq[8], av[4], as;
    lrs_adj<R, A>(P.pdmb, qdv, nmag, Vi, (A)1.0 / (A)Vi, aBL * (A)Vi, aBR * (A)Vi, aq, av, &as);
    if (es) {  // per edge: the stencil weight scale and the 4 limiter adjoints (es[0..4 fs])
        es[c] = (R)as;
        for (int m = 0; m < 4; m++) es[(1 + m) * fs + c] = (R)av[m];
        return;
    }
    for (int n = 0; n < 8; n++) atomicAdd(&dabh[a * fs + c + (n - 4) * s], (R)aq[n]);
    for (int m = 0; m < 4; m++) atomicAdd(&dbn[a * fs + c + (m - 2) * s], (R)av[m]);
}

// Adjoint of the edge EMF of direction eD (k_vxb) over the range r: dE ->
// dDh, dabh, dbn, dAVf (the AVf of this eD, 3 components, caller-zeroed) by
// atomics, or, with es, the edge's own adjoints stored per edge (14
// components: 0-4 and 5-9 the scale and limiter adjoints of the EdgeLRs of
// dT1 and dT2 faces, 10-12 the velocity adjoint aVC, 13 the corner density's)
// for a gather in a fixed order. SAVED: the corner values come from w.esv
// (stored by the forward) instead of being recomputed.
template <class R, bool SAVED = false>
__global__ void __launch_bounds__(128, 6) k_vxb_adj(GamBox b, DevParams<R> P, Geo<R> g, Work<R> w, int eD, Range r,
                                                 double dt, const R* __restrict__ dE, R* dDh, R* dabh, R* dbn,
                                                 R* dAVf, R* __restrict__ es) {
    int ii, jj, kk;
    if (!thread_ijk(r, ii, jj, kk)) return;
    int dT1, dT2;
    edge_dirs(eD, dT1, dT2);
    const long fs = b.fs;
    const long c = lidx(b, ii, jj, kk);
    const int e1 = eD == 0 ? 1 : 0, e2 = eD == 2 ? 1 : 2;
    const long s1 = dstride(b, e1), s2 = dstride(b, e2);
    // forward recompute (k_vxb), or its saved corner values
    R Dc, bT1L, bT1R, fA1, bT2L, bT2R, fA2, VC[3];
    const long s2v = dstride(b, dT2);
    if constexpr (SAVED) {
        const R* o = w.esv + (long)(GAM_ESV_NC * eD) * fs + c;
        Dc = o[0];
        bT1L = o[fs];
        bT1R = o[2 * fs];
        fA1 = o[3 * fs];
        bT2L = o[4 * fs];
        bT2R = o[5 * fs];
        fA2 = o[6 * fs];
        for (int x = 0; x < 3; x++) VC[x] = o[(7 + x) * fs];
    } else {
        Dc = (R)0.25 * (w.Dh[c] + w.Dh[c - s1] + w.Dh[c - s2] + w.Dh[c - s1 - s2]);
        R area1[8], area2[8];
        edge_lrs(b, P, g, w, c, dT1, dT2, area1, bT1L, bT1R, fA1);
        edge_lrs(b, P, g, w, c, dT2, dT1, area2, bT2L, bT2R, fA2);
        const R dA0 = rmax(fA1, (R)TINY);
        for (int x = 0; x < 3; x++) {
            R acc = (R)0;
            for (int n = 0; n < 8; n++) acc += Rc<R>(w8(n)) * w.AVf[(x + 3 * eD) * fs + c + (n - 4) * s2v];
            VC[x] = acc / dA0;
        }
    }
    const R dA = rmax(fA1, (R)TINY);
    const R* Te = g.Te;
    R T1[3], T2[3];
    for (int x = 0; x < 3; x++) {
        T1[x] = Te[(3 + x + 9 * eD) * fs + c];
        T2[x] = Te[(6 + x + 9 * eD) * fs + c];
    }
    const R v1 = VC[0] * T1[0] + VC[1] * T1[1] + VC[2] * T1[2];
    const R v2 = VC[0] * T2[0] + VC[1] * T2[1] + VC[2] * T2[2];
    const R vD0 = Mth<R>::sqrt_(v1 * v1 + v2 * v2);
    const R xni = g.Teb[(0 + 4 * eD) * fs + c], yni = g.Teb[(1 + 4 * eD) * fs + c];
    const R xnj = g.Teb[(2 + 4 * eD) * fs + c], ynj = g.Teb[(3 + 4 * eD) * fs + c];
    const R detT = (R)1 / (xni * ynj - xnj * yni);
    const R bT1 = (R)0.5 * (bT1L + bT1R) / fA1;
    const R bT2 = (R)0.5 * (bT2L + bT2R) / fA2;
    const R db1 = (bT1R - bT1L) / fA1;
    const R db2 = (bT2R - bT2L) / fA2;
    const R Jd = db2 - db1;
    R b1 = detT * (ynj * bT1 - yni * bT2);
    R b2 = detT * (-(xnj * bT1) + xni * bT2);
    if (P.doBackground) {
        b1 = b1 + (R)g.edgB0[(0 + 2 * eD) * fs + c];
        b2 = b2 + (R)g.edgB0[(1 + 2 * eD) * fs + c];
    }
    const R m = Mth<R>::sqrt_(b1 * b1 + b2 * b2), q = Mth<R>::sqrt_(Dc);
    const R vA = m / q;
    const R vDp = vD0 + vA;
    const R edge = g.edge[eD * fs + c];
    const R cap = P.CFL * edge / (R)dt;
    const R vDiff = rmin(vDp, cap);
    // reverse, in the form's precision
    using A = R;
    const A a_e = (A)dE[eD * fs + c] * (A)edge;
    const A a_v1 = -a_e * b2, a_b2e = -a_e * v1, a_v2 = a_e * b1, a_b1e = a_e * v2;
    const A a_vDiff = a_e * P.Vd0 * Jd, a_Jd = a_e * P.Vd0 * vDiff;
    const A a_vDp = (cap < vDp) ? (A)0.0 : a_vDiff;
    A a_b1 = a_b1e, a_b2 = a_b2e, a_v1t = a_v1, a_v2t = a_v2;
    const A rq = (A)1.0 / (A)q;
    const A a_m = a_vDp * rq;
    const A a_q = -a_vDp * (A)m * rq * rq;
    const A a_Dc = a_q * (A)0.5 * rq;
    if (m > (R)0) {
        const A rm = (A)1.0 / (A)m;
        a_b1 += a_m * b1 * rm;
        a_b2 += a_m * b2 * rm;
    }
    if (vD0 > (R)0) {
        const A rv = (A)1.0 / (A)vD0;
        a_v1t += a_vDp * v1 * rv;
        a_v2t += a_vDp * v2 * rv;
    }
    const A a_bT1 = a_b1 * detT * ynj - a_b2 * detT * xnj;
    const A a_bT2 = -a_b1 * detT * yni + a_b2 * detT * xni;
    const A a_db2 = a_Jd, a_db1 = -a_Jd;
    const A rA1 = (A)1.0 / (A)fA1, rA2 = (A)1.0 / (A)fA2;
    const A aT1R = (a_db1 + a_bT1 * (A)0.5) * rA1, aT1L = (-a_db1 + a_bT1 * (A)0.5) * rA1;
    const A aT2R = (a_db2 + a_bT2 * (A)0.5) * rA2, aT2L = (-a_db2 + a_bT2 * (A)0.5) * rA2;
    edge_lrs_adj<R, A>(b, P, g, w, c, dT1, dT2, aT1L, aT1R, dabh, dbn, es);
    edge_lrs_adj<R, A>(b, P, g, w, c, dT2, dT1, aT2L, aT2R, dabh, dbn, es ? es + 5 * fs : nullptr);
    const A rdA = (A)1.0 / (A)dA;
    for (int x = 0; x < 3; x++) {
        const A aVC = (a_v1t * T1[x] + a_v2t * T2[x]) * rdA;
        if (es) {
            es[(10 + x) * fs + c] = (R)aVC;
            continue;
        }
        for (int n = 0; n < 8; n++) atomicAdd(&dAVf[x * fs + c + (n - 4) * s2v], (R)((A)w8(n) * aVC));
    }
    if (es) {
        es[13 * fs + c] = (R)a_Dc;
        return;
    }
    const long cc[4] = {c, c - s1, c - s2, c - s1 - s2};
    for (int n = 0; n < 4; n++) atomicAdd(&dDh[cc[n]], (R)((A)0.25 * a_Dc));
}

struct Range3 {
    Range r[3];
};

// The adjoints the edges of the three directions hold in es (k_vxb_adj; 14
// components from es + 14 eD fs), gathered per position in a fixed order
// (deterministic, no atomics) and stored: for the faces of each direction fa
// their operand and limiter stencil adjoints (dabh, dbn) from the edges
// whose EdgeLRs run over them, for the cells the corner densities' dDh and,
// per edge direction, the velocity stencil's dAVf times face area /
// interpolated volume of Mom2Face (aS + 3 eD fs; zero outside the Mom2Face
// range mf[eD]). Edges outside their range ed[eD] carry nothing. The sums
// run over the stencil, then eD = I, J, K, as three passes adding into a
// zeroed array would.
template <class R>
__global__ void __launch_bounds__(256) k_vxb_adj_gather3(GamBox b, Geo<R> g, Range3 ed, Range3 mf,
                                                         const R* __restrict__ es, R* __restrict__ dDh,
                                                         R* __restrict__ dabh, R* __restrict__ dbn,
                                                         R* __restrict__ aS) {
    using A = R;
    int ii, jj, kk;
    const Range all{0, b.Ni, 0, b.Nj, 0, b.Nk};
    if (!thread_ijk(all, ii, jj, kk)) return;
    const long fs = b.fs;
    const long c = lidx(b, ii, jj, kk);
    const int p[3] = {ii, jj, kk};
    A fq[3] = {(A)0, (A)0, (A)0}, fl[3] = {(A)0, (A)0, (A)0};
    const bool isCell = ii < b.Ni && jj < b.Nj && kk < b.Nk;
    A d = (A)0;
#pragma unroll
    for (int eD = 0; eD < 3; eD++) {
        const Range r = ed.r[eD];
        const int lo[3] = {r.i0, r.j0, r.k0}, hi[3] = {r.i1, r.j1, r.k1};
        // is the edge at p + k e_dd inside the range?
        auto in_r = [&](int dd, int k) {
            bool ok = true;
#pragma unroll
            for (int a = 0; a < 3; a++) {
                const int q = p[a] + (a == dd ? k : 0);
                ok = ok && q >= lo[a] && q <= hi[a];
            }
            return ok;
        };
        int dT1, dT2;
        edge_dirs(eD, dT1, dT2);
        const R* e = es + 14L * eD * fs + c;
        // every edge within -3..4 of p along dT1 and along dT2 in range
        const bool full = in_r(dT1, -3) && in_r(dT1, 4) && in_r(dT2, -3) && in_r(dT2, 4);
#pragma unroll
        for (int side = 0; side < 2; side++) {
            const int fa = side == 0 ? dT1 : dT2, bd = side == 0 ? dT2 : dT1;
            const R* e0 = e + (5 * side) * fs;
            const long sb = dstride(b, bd);
            A q = (A)0, l = (A)0;
            bool any = false;
            if (full) {
                R x[8], y[4];
#pragma unroll
                for (int n = 0; n < 8; n++) x[n] = e0[(4 - n) * sb];
#pragma unroll
                for (int m = 0; m < 4; m++) y[m] = e0[(1 + m) * fs + (2 - m) * sb];
#pragma unroll
                for (int n = 0; n < 8; n++) q += (A)w8(n) * (A)x[n];
#pragma unroll
                for (int m = 0; m < 4; m++) l += (A)y[m];
                any = true;
            } else {
#pragma unroll
                for (int n = 0; n < 8; n++)
                    if (in_r(bd, 4 - n)) {
                        q += (A)w8(n) * (A)e0[(4 - n) * sb];
                        any = true;
                    }
#pragma unroll
                for (int m = 0; m < 4; m++)
                    if (in_r(bd, 2 - m)) {
                        l += (A)e0[(1 + m) * fs + (2 - m) * sb];
                        any = true;
                    }
            }
            if (any) {
                fq[fa] += q;
                fl[fa] += l;
            }
        }
        if (!isCell) continue;
        // the velocity stencil along dT2, scaled as Mom2Face's adjoint
        const Range rm = mf.r[eD];
        const bool inm = ii >= rm.i0 && ii <= rm.i1 && jj >= rm.j0 && jj <= rm.j1 && kk >= rm.k0 && kk <= rm.k1;
        const long s2 = dstride(b, dT2);
        double AdV = 0.0;
        if (inm) {
            const long s1 = dstride(b, dT1);
            R vol[8];
            for (int n = 0; n < 8; n++) vol[n] = g.vol[c + (n - 4) * s1];
            const R dV = rmax(central8(vol), (R)TINY);
            AdV = (double)g.face[dT1 * fs + c] / (double)dV;
        }
#pragma unroll
        for (int x = 0; x < 3; x++) {
            A v = (A)0;
            if (inm && full) {
                R y[8];
#pragma unroll
                for (int n = 0; n < 8; n++) y[n] = e[(10 + x) * fs + (4 - n) * s2];
#pragma unroll
                for (int n = 0; n < 8; n++) v += (A)w8(n) * (A)y[n];
            } else if (inm) {
#pragma unroll
                for (int n = 0; n < 8; n++)
                    if (in_r(dT2, 4 - n)) v += (A)w8(n) * (A)e[(10 + x) * fs + (4 - n) * s2];
            }
            aS[(3 * eD + x) * fs + c] = inm ? (R)((double)(R)v * AdV) : (R)0;
        }
        // the 4 corners of GetCornerD: edges c, c + s1, c + s2, c + s1 + s2
        const int e1 = eD == 0 ? 1 : 0, e2 = eD == 2 ? 1 : 2;
        const long t1 = dstride(b, e1), t2 = dstride(b, e2);
        A dd = (A)0;
        bool anyd = false;
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int o1 = q & 1, o2 = q >> 1;
            bool ok = true;
#pragma unroll
            for (int a = 0; a < 3; a++) {
                const int v = p[a] + (a == e1 ? o1 : 0) + (a == e2 ? o2 : 0);
                ok = ok && v >= lo[a] && v <= hi[a];
            }
            if (ok) {
                dd += (A)0.25 * (A)e[13 * fs + o1 * t1 + o2 * t2];
                anyd = true;
            }
        }
        if (anyd) d += dd;
    }
#pragma unroll
    for (int fa = 0; fa < 3; fa++) {
        dabh[fa * fs + c] = (R)fq[fa];
        dbn[fa * fs + c] = (R)fl[fa];
    }
    if (isCell) dDh[c] = (R)d;
}

// Mom2Face's adjoint gathered per cell: dVdV = sum over eD of the 8-point
// stencil along dT1 of the scaled dAVf (aS + 3 eD fs) over the faces of the
// Mom2Face range mf[eD], in FP64 per eD, then eD = I, J, K; stored.
template <class R>
__global__ void __launch_bounds__(256) k_m2f_adj_gather3(GamBox b, Range3 mf, const R* __restrict__ aS,
                                                         R* __restrict__ dVdV) {
    int ii, jj, kk;
    const Range all{0, b.Ni - 1, 0, b.Nj - 1, 0, b.Nk - 1};
    if (!thread_ijk(all, ii, jj, kk)) return;
    const long fs = b.fs, c = lidx(b, ii, jj, kk);
    const int p[3] = {ii, jj, kk};
    R out[3] = {(R)0, (R)0, (R)0};
#pragma unroll
    for (int eD = 0; eD < 3; eD++) {
        int dT1, dT2;
        edge_dirs(eD, dT1, dT2);
        const Range r = mf.r[eD];
        const int lo[3] = {r.i0, r.j0, r.k0}, hi[3] = {r.i1, r.j1, r.k1};
        bool line = true;
#pragma unroll
        for (int a = 0; a < 3; a++)
            if (a != dT1 && (p[a] < lo[a] || p[a] > hi[a])) line = false;
        if (!line) continue;
        const long s = dstride(b, dT1);
        const R* a0 = aS + 3L * eD * fs + c;
        double acc[3] = {0.0, 0.0, 0.0};
        bool any = false;
#pragma unroll
        for (int n = 0; n < 8; n++) {
            const int f = p[dT1] + 4 - n;
            if (f >= lo[dT1] && f <= hi[dT1]) {
                any = true;
#pragma unroll
                for (int x = 0; x < 3; x++) acc[x] += w8(n) * (double)a0[x * fs + (4 - n) * s];
            }
        }
        if (any)
            for (int x = 0; x < 3; x++) out[x] += (R)acc[x];
    }
    for (int x = 0; x < 3; x++) dVdV[x * fs + c] = out[x];
}

// Adjoint of Mom2Face for edge direction eD over the range r: dAVf -> dVdV
template <class R>
__global__ void __launch_bounds__(256) k_m2f_adj(GamBox b, Geo<R> g, int eD, Range r, const R* __restrict__ dAVf,
                                                 R* dVdV) {
    int ii, jj, kk;
    if (!thread_ijk(r, ii, jj, kk)) return;
    int dT1, dT2;
    edge_dirs(eD, dT1, dT2);
    const long fs = b.fs;
    const long c = lidx(b, ii, jj, kk);
    const long s = dstride(b, dT1);
    R vol[8];
    for (int n = 0; n < 8; n++) vol[n] = g.vol[c + (n - 4) * s];
    const R dV = rmax(central8(vol), (R)TINY);
    const R A = g.face[dT1 * fs + c];
    const double AdV = (double)A / (double)dV;
    for (int x = 0; x < 3; x++) {
        const double a = (double)dAVf[x * fs + c] * AdV;
        if (a == 0.0) continue;
        for (int n = 0; n < 8; n++) atomicAdd(&dVdV[x * fs + c + (n - 4) * s], (R)(w8(n) * a));
    }
}

// ----------------------------------------------------------------- predictor and update
// reverse of cell_c2p (CellC2P): aW (5) -> aU (5)
template <class A>
__device__ void c2p_adj(A dF, A pF, A gm1, const A* U, const A* aW, A* aU) {
    const A rho = U[0], rr = (A)1.0 / rho;
    const A V[3] = {U[1] * rr, U[2] * rr, U[3] * rr};
    const A KinE = (A)0.5 * rho * (V[0] * V[0] + V[1] * V[1] + V[2] * V[2]);
    const A p = gm1 * (U[4] - KinE);
    A a_rho = (rho < dF) ? (A)0.0 : aW[0];
    A a_V[3] = {aW[1], aW[2], aW[3]};
    A a_E = (A)0.0, a_KinE = (A)0.0;
    if (!(p < pF)) { a_E = aW[4] * gm1; a_KinE = -aW[4] * gm1; }
    a_rho += a_KinE * (A)0.5 * (V[0] * V[0] + V[1] * V[1] + V[2] * V[2]);
    for (int x = 0; x < 3; x++) a_V[x] += a_KinE * rho * V[x];
    for (int x = 0; x < 3; x++) {
        aU[1 + x] += a_V[x] * rr;
        a_rho += -a_V[x] * V[x] * rr;
    }
    aU[0] += a_rho;
    aU[4] += a_E;
}
// reverse of cell_p2c (CellP2C): aU (5) -> aW (5)
template <class A>
__device__ void p2c_adj(A dF, A pF, A gm1, const A* W, const A* aU, A* aW) {
    const A rho = W[0] < dF ? dF : W[0];
    const A V[3] = {W[1], W[2], W[3]};
    const A V2 = V[0] * V[0] + V[1] * V[1] + V[2] * V[2];
    A a_rho = aU[0] + aU[4] * (A)0.5 * V2;
    for (int x = 0; x < 3; x++) {
        a_rho += aU[1 + x] * V[x];
        aW[1 + x] += aU[1 + x] * rho + aU[4] * rho * V[x];
    }
    aW[4] += (W[4] < pF) ? (A)0.0 : aU[4] / gm1;
    aW[0] += (W[0] < dF) ? (A)0.0 : a_rho;
}
// reverse of block_c2p (BlockCon2Prim): aW (5) -> aU (5)
template <class A>
__device__ void bc2p_adj(A dF, A pF, A gm1, const A* U, const A* aW, A* aU) {
    const A D = U[0] < dF ? dF : U[0], rD = (A)1.0 / D;
    const A M[3] = {U[1], U[2], U[3]};
    const A M2 = M[0] * M[0] + M[1] * M[1] + M[2] * M[2];
    const A KinE = (A)0.5 * M2 * rD;
    const A p = gm1 * (U[4] - KinE);
    A a_D = aW[0], a_M[3];
    for (int x = 0; x < 3; x++) {
        a_M[x] = aW[1 + x] * rD;
        a_D += -aW[1 + x] * M[x] * rD * rD;
    }
    A a_E = (A)0.0, a_KinE = (A)0.0;
    if (!(p < pF)) { a_E = aW[4] * gm1; a_KinE = -aW[4] * gm1; }
    for (int x = 0; x < 3; x++) a_M[x] += a_KinE * M[x] * rD;
    a_D += -a_KinE * (A)0.5 * M2 * rD * rD;
    aU[0] += (U[0] < dF) ? (A)0.0 : a_D;
    for (int x = 0; x < 3; x++) aU[1 + x] += a_M[x];
    aU[4] += a_E;
}

// V d B_x / d (flux of face f of cell c), f = 0..5 (I-, I+, J-, J+, K-, K+),
// as in gamCellBxyz: xfc - xyzcc with the sign of the face
template <class R>
__device__ __forceinline__ R dbdf(const GamBox& b, const Geo<R>& g, long c, int f, int x) {
    const long fs = b.fs;
    const int d = f >> 1, up = f & 1;
    double off;
    if constexpr (std::is_same<R, float>::value) {
        off = g.dxf[(x + 3 * f) * fs + c];
    } else {
        const long cf = c + (up ? dstride(b, d) : 0L);
        off = (double)g.xfc[(x + 3 * d) * fs + cf] - (double)g.xyzcc[x * fs + c];
    }
    return up ? off : -off;
}

// predictor adjoint, cells: dQW, dWn, dDh, dVdV, dQB -> dGas, doGas; writes
// aB = volume * dQB (the adjoint of the half-state Bxyz) for the face pass
template <class R>
__global__ void __launch_bounds__(128) k_predict_adj_cells(GamBox b, DevParams<R> P, Geo<R> g, StateBuf<R> cur,
                                                           StateBuf<R> old, double pdt, double odt, Work<R> dw,
                                                           R* dGas, R* doGas, R* aB) {
    using A = R;  // accumulation in the form's precision
    int ii, jj, kk;
    Range r{0, b.Ni - 1, 0, b.Nj - 1, 0, b.Nk - 1};
    if (!thread_ijk(r, ii, jj, kk)) return;
    const long fs = b.fs, c = lidx(b, ii, jj, kk);
    const A dF = P.dFloor, pF = P.pFloor, gm1 = P.gm1;
    A Q[5], oQ[5], W[5], oW[5], pW[5], pWf[5], pQ[5];
    for (int v = 0; v < 5; v++) { Q[v] = cur.Gas[v * fs + c]; oQ[v] = old.Gas[v * fs + c]; }
    auto c2p = [&](const A* U, A* Wo) {
        const A rho = U[0], rr = (A)1.0 / rho;
        const A Vx = U[1] * rr, Vy = U[2] * rr, Vz = U[3] * rr;
        const A KinE = (A)0.5 * rho * (Vx * Vx + Vy * Vy + Vz * Vz);
        Wo[0] = rho < dF ? dF : rho; Wo[1] = Vx; Wo[2] = Vy; Wo[3] = Vz;
        const A pp = gm1 * (U[4] - KinE);
        Wo[4] = pp < pF ? pF : pp;
    };
    c2p(Q, W);
    c2p(oQ, oW);
    const A rodt = (A)1.0 / odt, pr = pdt * rodt;
    for (int v = 0; v < 5; v++) pW[v] = W[v] + pdt * ((W[v] - oW[v]) * rodt);
    for (int v = 0; v < 5; v++) pWf[v] = pW[v];
    pWf[0] = pW[0] < dF ? dF : pW[0];
    pWf[4] = pW[4] < pF ? pF : pW[4];
    {
        const A rho = pWf[0] < dF ? dF : pWf[0];
        const A IntE = (pWf[4] < pF ? pF : pWf[4]) * ((A)1.0 / gm1);
        const A KinE = (A)0.5 * rho * (pWf[1] * pWf[1] + pWf[2] * pWf[2] + pWf[3] * pWf[3]);
        pQ[0] = rho; pQ[1] = rho * pWf[1]; pQ[2] = rho * pWf[2]; pQ[3] = rho * pWf[3]; pQ[4] = IntE + KinE;
    }
    const A vol = g.vol[c];
    A aWh[5], apQ[5] = {0, 0, 0, 0, 0};
    for (int v = 0; v < 5; v++) aWh[v] = vol * (A)dw.QW[v * fs + c];
    aWh[0] += dw.Dh[c];
    const A Dm = pQ[0] < dF ? dF : pQ[0], rDm = (A)1.0 / Dm;
    A aDm = (A)0.0;
    for (int x = 0; x < 3; x++) {
        const A a = dw.VdV[x * fs + c];
        apQ[1 + x] += vol * a * rDm;
        aDm += -vol * pQ[1 + x] * a * rDm * rDm;
    }
    if (!(pQ[0] < dF)) apQ[0] += aDm;
    bc2p_adj(dF, pF, gm1, pQ, aWh, apQ);
    A apWf[5] = {0, 0, 0, 0, 0};
    p2c_adj(dF, pF, gm1, pWf, apQ, apWf);
    A apW[5];
    for (int v = 0; v < 5; v++) apW[v] = apWf[v];
    apW[0] = (pW[0] < dF) ? (A)0.0 : apWf[0];
    apW[4] = (pW[4] < pF) ? (A)0.0 : apWf[4];
    A aW[5], aoW[5];
    for (int v = 0; v < 5; v++) {
        aW[v] = apW[v] + apW[v] * pr;
        aoW[v] = -apW[v] * pr;
    }
    A aQ[5] = {0, 0, 0, 0, 0}, aoQ[5] = {0, 0, 0, 0, 0};
    c2p_adj(dF, pF, gm1, Q, aW, aQ);
    c2p_adj(dF, pF, gm1, oQ, aoW, aoQ);
    A aWn[5];
    for (int v = 0; v < 5; v++) aWn[v] = dw.Wn[v * fs + c];
    bc2p_adj(dF, pF, gm1, Q, aWn, aQ);
    for (int v = 0; v < 5; v++) {
        dGas[v * fs + c] += (R)aQ[v];
        doGas[v * fs + c] += (R)aoQ[v];
    }
    if (P.doMHD)
        for (int x = 0; x < 3; x++) aB[x * fs + c] = (R)(vol * (A)dw.QB[x * fs + c]);
}

// predictor adjoint, faces: dabh, dBnf, dbn and the Bxyz adjoints of the two
// cells sharing the face -> dmf, domf
template <class R>
__global__ void __launch_bounds__(256) k_predict_adj_faces(GamBox b, DevParams<R> P, Geo<R> g, double pdt, double odt,
                                                           Work<R> dw, const R* __restrict__ aB, R* dmf, R* domf) {
    using A = R;
    int ii, jj, kk;
    Range r{0, b.Ni, 0, b.Nj, 0, b.Nk};
    if (!thread_ijk(r, ii, jj, kk)) return;
    const long fs = b.fs, c = lidx(b, ii, jj, kk);
    if (!P.doMHD) return;
    const int ijk[3] = {ii, jj, kk}, n[3] = {b.Ni, b.Nj, b.Nk};
    const A pr = pdt / odt;
    A rv = (A)0.0;
    if (ii < b.Ni && jj < b.Nj && kk < b.Nk) rv = (A)1.0 / (A)g.vol[c];
    for (int d = 0; d < 3; d++) {
        const A Af = g.face[d * fs + c];
        const A Am = Af < (A)TINY ? (A)TINY : Af, rAm = (A)1.0 / Am;
        A ahm = (A)dw.abh[d * fs + c] * Af * rAm + (A)dw.Bnf[d * fs + c] / Af;
        // cells c (this is its lower face d) and c - s_d (its upper face)
        bool inLo = true, inUp = true;
        for (int e = 0; e < 3; e++) {
            const int lo = ijk[e] - (e == d ? 1 : 0);
            if (ijk[e] >= n[e]) inLo = false;
            if (lo < 0 || lo >= n[e]) inUp = false;
        }
        if (inLo)
            for (int x = 0; x < 3; x++) ahm += (A)aB[x * fs + c] * rv * dbdf(b, g, c, 2 * d, x);
        if (inUp) {
            const long cu = c - dstride(b, d);
            const A rvu = (A)1.0 / (A)g.vol[cu];
            for (int x = 0; x < 3; x++) ahm += (A)aB[x * fs + cu] * rvu * dbdf(b, g, cu, 2 * d + 1, x);
        }
        dmf[d * fs + c] += (R)(ahm + ahm * pr + (A)dw.bn[d * fs + c] * rAm);
        domf[d * fs + c] += (R)(-ahm * pr);
    }
}

// update adjoint, cells: dnxtGas -> dcurGas, and the scaled adjoints
// sU = dt aU / V, sM = dt aM / V of the active cells for the face pass
template <class R>
__global__ void __launch_bounds__(128) k_update_adj_cells(GamBox b, DevParams<R> P, Geo<R> g, StateBuf<R> cur,
                                                          Work<R> w, double dt, const R* __restrict__ dnGas, R* dGas,
                                                          R* sU, R* sM) {
    using A = R;
    int ii, jj, kk;
    Range r{0, b.Ni - 1, 0, b.Nj - 1, 0, b.Nk - 1};
    if (!thread_ijk(r, ii, jj, kk)) return;
    const long fs = b.fs, c = lidx(b, ii, jj, kk);
    const int G = GAM_NG;
    const bool active = ii >= G && ii < G + b.Nip && jj >= G && jj < G + b.Njp && kk >= G && kk < G + b.Nkp;
    if (!active) {
        for (int v = 0; v < 5; v++) dGas[v * fs + c] += dnGas[v * fs + c];
        return;
    }
    const A dF = P.dFloor, pF = P.pFloor, gm1 = P.gm1;
    const A dV = g.vol[c], rdV = (A)1.0 / dV;
    const long sj = b.sx, sk = b.sk;
    A U[5], dGasM[3] = {0, 0, 0};
    for (int v = 0; v < 5; v++) {
        const R* gI = w.gF + (v + 0) * fs;
        const R* gJ = w.gF + (v + 5) * fs;
        const R* gK = w.gF + (v + 10) * fs;
        const A dGasH = ((A)gI[c] - gI[c + 1] + gJ[c] - gJ[c + sj] + gK[c] - gK[c + sk]) * rdV;
        U[v] = (A)cur.Gas[v * fs + c] + dt * dGasH;
    }
    A aU[5], aM3[3] = {0, 0, 0};
    A ao[5];
    for (int v = 0; v < 5; v++) ao[v] = dnGas[v * fs + c];
    if (P.doMHD) {
        for (int x = 0; x < 3; x++) {
            const R* mI = w.mF + (x + 0) * fs;
            const R* mJ = w.mF + (x + 3) * fs;
            const R* mK = w.mF + (x + 6) * fs;
            dGasM[x] = ((A)mI[c] - mI[c + 1] + mJ[c] - mJ[c + sj] + mK[c] - mK[c + sk]) * rdV;
            if (P.doBackground) dGasM[x] += g.dpB0[x * fs + c];
        }
        // CellMaxwell (mhdgroup.F90:299-329) backwards
        const A D = U[0] < dF ? dF : U[0], rD = (A)1.0 / D;
        const A M[3] = {U[1], U[2], U[3]};
        const A KinE = (A)0.5 * (M[0] * M[0] + M[1] * M[1] + M[2] * M[2]) * rD;
        const A p = gm1 * (U[4] - KinE);
        A Mn[3];
        for (int x = 0; x < 3; x++) Mn[x] = M[x] + dt * dGasM[x];
        const A Mn2 = Mn[0] * Mn[0] + Mn[1] * Mn[1] + Mn[2] * Mn[2];
        A a_D = ao[0], a_Mn[3];
        const A a_KinEn = ao[4], a_Pr = ao[4] * ((A)1.0 / gm1);
        for (int x = 0; x < 3; x++) a_Mn[x] = ao[1 + x] + a_KinEn * Mn[x] * rD;
        a_D += -a_KinEn * (A)0.5 * Mn2 * rD * rD;
        A a_M[3];
        for (int x = 0; x < 3; x++) {
            a_M[x] = a_Mn[x];
            aM3[x] = a_Mn[x] * dt;
        }
        A a_U4 = (A)0.0, a_KinE = (A)0.0;
        if (!(p < pF)) { a_U4 = a_Pr * gm1; a_KinE = -a_Pr * gm1; }
        for (int x = 0; x < 3; x++) a_M[x] += a_KinE * M[x] * rD;
        a_D += -a_KinE * (A)0.5 * (M[0] * M[0] + M[1] * M[1] + M[2] * M[2]) * rD * rD;
        aU[0] = (U[0] < dF) ? (A)0.0 : a_D;
        for (int x = 0; x < 3; x++) aU[1 + x] = a_M[x];
        aU[4] = a_U4;
    } else {
        for (int v = 0; v < 5; v++) aU[v] = ao[v];
    }
    for (int v = 0; v < 5; v++) {
        dGas[v * fs + c] += (R)aU[v];
        sU[v * fs + c] = (R)(dt * aU[v] * rdV);
    }
    for (int x = 0; x < 3; x++) sM[x * fs + c] = (R)(aM3[x] * rdV);
}

// update adjoint, faces: face fluxes gF/mF from the two cells, E2Flux -> dE,
// and dcurmf = dnxtmf (copied or updated faces alike)
template <class R>
__global__ void __launch_bounds__(256) k_update_adj_faces(GamBox b, DevParams<R> P, double dt,
                                                          const R* __restrict__ sU, const R* __restrict__ sM,
                                                          const R* __restrict__ dnmf, R* dmf, R* dgF, R* dmF, R* dE,
                                                          int assign) {
    using A = R;
    int ii, jj, kk;
    Range r{0, b.Ni, 0, b.Nj, 0, b.Nk};
    if (!thread_ijk(r, ii, jj, kk)) return;
    const long fs = b.fs, c = lidx(b, ii, jj, kk);
    const int G = GAM_NG;
    const int lo[3] = {G, G, G}, hi[3] = {G + b.Nip - 1, G + b.Njp - 1, G + b.Nkp - 1};
    auto act = [&](int a0, int a1, int a2) {
        return a0 >= lo[0] && a0 <= hi[0] && a1 >= lo[1] && a1 <= hi[1] && a2 >= lo[2] && a2 <= hi[2];
    };
    for (int d = 0; d < 3; d++) {
        const bool inLo = act(ii, jj, kk);
        const bool inUp = act(ii - (d == 0), jj - (d == 1), kk - (d == 2));
        const long cu = c - dstride(b, d);
        for (int v = 0; v < 5; v++) {
            A a = (A)0.0;
            if (inLo) a += sU[v * fs + c];
            if (inUp) a -= sU[v * fs + cu];
            if (assign)
                dgF[(v + 5 * d) * fs + c] = (R)a;
            else
                dgF[(v + 5 * d) * fs + c] += (R)a;
        }
        if (P.doMHD)
            for (int x = 0; x < 3; x++) {
                A a = (A)0.0;
                if (inLo) a += sM[x * fs + c];
                if (inUp) a -= sM[x * fs + cu];
                if (assign)
                    dmF[(x + 3 * d) * fs + c] = (R)a;
                else
                    dmF[(x + 3 * d) * fs + c] += (R)a;
            }
        dmf[d * fs + c] += dnmf[d * fs + c];
    }
    if (!P.doMHD) return;
    // E2Flux on the faces [G, G+Nip] x [G, G+Njp] x [G, G+Nkp] (k_update_faces)
    auto inr = [&](int a0, int a1, int a2) {
        return a0 >= G && a0 <= G + b.Nip && a1 >= G && a1 <= G + b.Njp && a2 >= G && a2 <= G + b.Nkp;
    };
    const long sj = b.sx, sk = b.sk;
    auto An = [&](int q, int a0, int a1, int a2) -> A {
        return inr(a0, a1, a2) ? (A)dnmf[q * fs + c + (a0 - ii) + (long)(a1 - jj) * sj + (long)(a2 - kk) * sk] : (A)0.0;
    };
    const A a0c = An(0, ii, jj, kk), a1c = An(1, ii, jj, kk), a2c = An(2, ii, jj, kk);
    // mf0 -= dt (E2[+j] - E2 - E1[+k] + E1); mf1 -= dt (E0[+k] - E0 - E2[+i] + E2); mf2 -= dt (E1[+i] - E1 - E0[+j] + E0)
    const A aE2 = -dt * (An(0, ii, jj - 1, kk) - a0c - An(1, ii - 1, jj, kk) + a1c);
    const A aE1 = -dt * (-An(0, ii, jj, kk - 1) + a0c + An(2, ii - 1, jj, kk) - a2c);
    const A aE0 = -dt * (An(1, ii, jj, kk - 1) - a1c - An(2, ii, jj - 1, kk) + a2c);
    if (assign) {
        dE[c] = (R)aE0;
        dE[fs + c] = (R)aE1;
        dE[2 * fs + c] = (R)aE2;
    } else {
        dE[c] += (R)aE0;
        dE[fs + c] += (R)aE1;
        dE[2 * fs + c] += (R)aE2;
    }
}
// ----------------------------------------------------------------- I-side boundaries
// The non-periodic I boundaries of the differentiation form, as the step
// restatement writes them (mage_b200/diffstep.py, _iside_bcs): the uniform
// inflow or the SphIn copy (bcs.F90:934-957) on the inner side, the constant
// solar wind (apps/wind.F90:206-374, MinMach = 1) or zeroGrad_obcI
// (bcs.F90:820-850) on the outer side, on ghost layers n = 1..4. One thread
// per (j, k) of the face box; a thread writes its own row only, and reads the
// first / last active cell and its faces, which no fill writes.
template <class R>
struct ISideDev {
    R inflow[8], wind[8];   // rho, P, Vx, Vy, Vz, Bx, By, Bz
    const R* wC;            // (Nk, Nj, 4) blend weights of the ghost cells
    const R* wF[3];         // (Nk+1, Nj+1, 4) face blend weights
    const R* sF[3];         // (Nk+1, Nj+1, 4) wind face fluxes
};

template <class R>
__device__ __forceinline__ R iside_proj(const GamBox& b, const R* face, const R* Tf, int d, long c, const R* B) {
    const long fs = b.fs;
    const R* n = Tf + (long)(9 * d) * fs + c;
    return face[d * fs + c] * (B[0] * n[0] + B[1] * n[fs] + B[2] * n[2 * fs]);
}

// the wind's MHD-side primitives of the last active cell: CellC2P, then the
// MinMach fix of the normal velocity with the fast speed of Con2Fast
template <class R>
struct WindEdge {
    R gC[5], Bin[3], gWin[5], V[3], nH[3];
    R rho, Vf[3], KinE, Pv, Pr, Cs, S, MagB, sq, Va, Cx, dn;
    bool fix;
    __device__ void eval(const DevParams<R>& P, const R* Gas, const R* B, const R* Tf, long fs, long cp) {
        for (int v = 0; v < 5; v++) gC[v] = Gas[v * fs + cp];
        for (int x = 0; x < 3; x++) Bin[x] = B[x * fs + cp];
        cell_c2p(P, gC, gWin);
        rho = rmax(gC[0], P.dFloor);
        for (int x = 0; x < 3; x++) Vf[x] = gC[1 + x] / rho;
        KinE = (R)0.5 * rho * (Vf[0] * Vf[0] + Vf[1] * Vf[1] + Vf[2] * Vf[2]);
        Pv = P.gm1 * (gC[4] - KinE);
        Pr = rmax(Pv, P.pFloor);
        Cs = Mth<R>::sqrt_(P.gamma * Pr / rho);
        S = Bin[0] * Bin[0] + Bin[1] * Bin[1] + Bin[2] * Bin[2];
        MagB = S > (R)0 ? Mth<R>::sqrt_(S) : (R)0;
        sq = Mth<R>::sqrt_(gC[0]);
        Va = MagB / sq;
        Cx = Mth<R>::sqrt_(Cs * Cs + Va * Va);
        const long cf = cp + 1;  // the I face ip + 1
        for (int x = 0; x < 3; x++) nH[x] = Tf[x * fs + cf];
        for (int x = 0; x < 3; x++) V[x] = gWin[1 + x];
        dn = V[0] * nH[0] + V[1] * nH[1] + V[2] * nH[2];
        fix = dn < Cx;
        if (fix)
            for (int x = 0; x < 3; x++) V[x] = V[x] - dn * nH[x] + Cx * nH[x];
    }
    // the blended primitives of ghost layer n (weight wSW of the wind)
    __device__ void blend(const ISideDev<R>& is, R wSW, R* gW) const {
        const R wMHD = (R)1 - wSW;
        const R sw = wSW > (R)TINY ? (R)1 : (R)0, mh = wMHD > (R)TINY ? (R)1 : (R)0;
        const R gW_sw[5] = {sw * is.wind[0], sw * is.wind[2], sw * is.wind[3], sw * is.wind[4], sw * is.wind[1]};
        const R gWi[5] = {mh * gWin[0], mh * V[0], mh * V[1], mh * V[2], mh * gWin[4]};
        for (int v = 0; v < 5; v++) gW[v] = wSW * gW_sw[v] + wMHD * gWi[v];
    }
};

template <class R>
__global__ void __launch_bounds__(256) k_iside_fill(GamBox b, DevParams<R> P, const R* __restrict__ face,
                                                    const R* __restrict__ Tf, ISideDev<R> is,
                                                    const R* __restrict__ B, R* Gas, R* mf) {
    const int jj = blockIdx.x * blockDim.x + threadIdx.x, kk = blockIdx.y * blockDim.y + threadIdx.y;
    if (jj > b.Nj || kk > b.Nk) return;
    const bool cellJK = jj < b.Nj && kk < b.Nk;
    const long fs = b.fs;
    const int G = GAM_NG, ip = G + b.Nip - 1;
    auto at = [&](int i) { return lidx(b, i, jj, kk); };
    if (P.bc[0] == BCK_INFLOW && cellJK) {
        const R gW[5] = {is.inflow[0], is.inflow[2], is.inflow[3], is.inflow[4], is.inflow[1]};
        R gC[5];
        cell_p2c(P, gW, gC);
        const R Bw[3] = {is.inflow[5], is.inflow[6], is.inflow[7]};
        for (int n = 1; n <= 4; n++) {
            const long c = at(G - n);
            for (int v = 0; v < 5; v++) Gas[v * fs + c] = gC[v];
            for (int d = 0; d < 3; d++) mf[d * fs + c] = iside_proj(b, face, Tf, d, c, Bw);
        }
    }
    if (P.bc[1] == BCK_ZEROGRAD && cellJK) {
        const long cp = at(ip);
        const R Bc[3] = {B[cp], B[fs + cp], B[2 * fs + cp]};
        R g0[5];
        for (int v = 0; v < 5; v++) g0[v] = Gas[v * fs + cp];
        for (int n = 1; n <= 4; n++) {
            const long cg = at(ip + n);
            for (int v = 0; v < 5; v++) Gas[v * fs + cg] = g0[v];
            mf[cg + 1] = iside_proj(b, face, Tf, 0, cg + 1, Bc);
            mf[fs + cg] = iside_proj(b, face, Tf, 1, cg, Bc);
            mf[2 * fs + cg] = iside_proj(b, face, Tf, 2, cg, Bc);
        }
    }
    if (P.bc[0] == BCK_SPHIN && cellJK) {
        const long src = at(G);
        R g0[5], f0[3];
        for (int v = 0; v < 5; v++) g0[v] = Gas[v * fs + src];
        for (int x = 0; x < 3; x++) f0[x] = mf[x * fs + src];
        for (int n = 1; n <= 4; n++) {
            const long dst = at(G - n);
            for (int v = 0; v < 5; v++) Gas[v * fs + dst] = g0[v];
            for (int x = 0; x < 3; x++) mf[x * fs + dst] = f0[x];
        }
    }
    if (P.bc[1] != BCK_WIND) return;
    const R fin[3] = {mf[at(ip + 1)], mf[fs + at(ip)], mf[2 * fs + at(ip)]};
    const long tf = ((long)kk * (b.Nj + 1) + jj) * 4;
    if (cellJK) {
        WindEdge<R> we;
        we.eval(P, Gas, B, Tf, fs, at(ip));
        const long tc = ((long)kk * b.Nj + jj) * 4;
        for (int n = 1; n <= 4; n++) {
            R gW[5], gC[5];
            we.blend(is, is.wC[tc + n - 1], gW);
            cell_p2c(P, gW, gC);
            const long cg = at(ip + n);
            for (int v = 0; v < 5; v++) Gas[v * fs + cg] = gC[v];
        }
    }
    for (int n = 1; n <= 4; n++)
        for (int d = 0; d < 3; d++) {
            const R w = is.wF[d][tf + n - 1];
            const long cf = d == 0 ? at(ip + n + 1) : at(ip + n);
            mf[d * fs + cf] = w * is.sF[d][tf + n - 1] + ((R)1 - w) * fin[d];
        }
}

// Adjoint of k_iside_fill: Gas and B as the fill found them at the first /
// last active cell (the fill leaves those unchanged), dGas and dMf the
// adjoints of the filled arrays. In place: every ghost the fill wrote passes
// its adjoint to what it was computed from and is zeroed; dB (the field of
// the update's fluxes) is added into at the last active cells. Follows the
// forward's branches (floors, the MinMach switch, sqrt at 0 with a zero
// derivative).
template <class R>
__global__ void __launch_bounds__(256) k_iside_adj(GamBox b, DevParams<R> P, const R* __restrict__ face,
                                                   const R* __restrict__ Tf, ISideDev<R> is,
                                                   const R* __restrict__ Gas, const R* __restrict__ B, R* dG, R* dM,
                                                   R* dB) {
    using A = R;
    const int jj = blockIdx.x * blockDim.x + threadIdx.x, kk = blockIdx.y * blockDim.y + threadIdx.y;
    if (jj > b.Nj || kk > b.Nk) return;
    const bool cellJK = jj < b.Nj && kk < b.Nk;
    const long fs = b.fs;
    const int G = GAM_NG, ip = G + b.Nip - 1;
    auto at = [&](int i) { return lidx(b, i, jj, kk); };
    const long cp = at(ip);
    if (P.bc[1] == BCK_WIND) {
        const long tf = ((long)kk * (b.Nj + 1) + jj) * 4;
        A afin[3] = {(A)0, (A)0, (A)0};
        for (int n = 1; n <= 4; n++)
            for (int d = 0; d < 3; d++) {
                const long cf = d == 0 ? at(ip + n + 1) : at(ip + n);
                afin[d] += ((A)1 - (A)is.wF[d][tf + n - 1]) * (A)dM[d * fs + cf];
                dM[d * fs + cf] = (R)0;
            }
        dM[at(ip + 1)] += (R)afin[0];
        dM[fs + cp] += (R)afin[1];
        dM[2 * fs + cp] += (R)afin[2];
        if (cellJK) {
            WindEdge<R> we;
            we.eval(P, Gas, B, Tf, fs, cp);
            const long tc = ((long)kk * b.Nj + jj) * 4;
            A aWin0 = (A)0, aWin4 = (A)0, aVn[3] = {(A)0, (A)0, (A)0};
            for (int n = 1; n <= 4; n++) {
                const R wSW = is.wC[tc + n - 1];
                R gW[5];
                we.blend(is, wSW, gW);
                const long cg = at(ip + n);
                A aU[5], aW[5] = {(A)0, (A)0, (A)0, (A)0, (A)0};
                for (int v = 0; v < 5; v++) {
                    aU[v] = dG[v * fs + cg];
                    dG[v * fs + cg] = (R)0;
                }
                p2c_adj<A>(P.dFloor, P.pFloor, P.gm1, gW, aU, aW);
                const A wMHD = (A)1 - (A)wSW;
                const A mh = wMHD > (A)TINY ? (A)1 : (A)0;
                aWin0 += mh * wMHD * aW[0];
                for (int x = 0; x < 3; x++) aVn[x] += mh * wMHD * aW[1 + x];
                aWin4 += mh * wMHD * aW[4];
            }
            // the MinMach fix: V' = V - dn nH + Cx nH, dn = V . nH
            A aV[3] = {aVn[0], aVn[1], aVn[2]}, aCx = (A)0;
            if (we.fix) {
                A s = (A)0;
                for (int x = 0; x < 3; x++) s += aVn[x] * (A)we.nH[x];
                aCx = s;
                for (int x = 0; x < 3; x++) aV[x] += -s * (A)we.nH[x];
            }
            // CellC2P of the edge cell
            const A aWc[5] = {aWin0, aV[0], aV[1], aV[2], aWin4};
            A aG[5] = {(A)0, (A)0, (A)0, (A)0, (A)0};
            c2p_adj<A>(P.dFloor, P.pFloor, P.gm1, we.gC, aWc, aG);
            // Con2Fast: Cx = sqrt(Cs^2 + Va^2), Va = MagB / sqrt(rho_c),
            // MagB = |B|, Cs = sqrt(gamma Pr / rho)
            A aB[3] = {(A)0, (A)0, (A)0};
            if (aCx != (A)0 && we.Cx > (R)0) {
                const A aCs = aCx * (A)we.Cs / (A)we.Cx, aVa = aCx * (A)we.Va / (A)we.Cx;
                const A aMagB = aVa / (A)we.sq;
                aG[0] += -aVa * (A)we.Va * (A)0.5 / (A)we.gC[0];
                if (we.S > (R)0)
                    for (int x = 0; x < 3; x++) aB[x] = aMagB * (A)we.Bin[x] / (A)we.MagB;
                A arho = (A)0;
                if (we.Cs > (R)0) {
                    const A aX = aCs * (A)0.5 / (A)we.Cs;
                    const A aPr = aX * (A)P.gamma / (A)we.rho;
                    arho += -aX * (A)P.gamma * (A)we.Pr / ((A)we.rho * (A)we.rho);
                    if (!(we.Pv < P.pFloor)) {
                        aG[4] += aPr * (A)P.gm1;
                        const A aKinE = -aPr * (A)P.gm1;
                        arho += aKinE * (A)0.5 *
                                ((A)we.Vf[0] * (A)we.Vf[0] + (A)we.Vf[1] * (A)we.Vf[1] + (A)we.Vf[2] * (A)we.Vf[2]);
                        for (int x = 0; x < 3; x++) {
                            const A aVf = aKinE * (A)we.rho * (A)we.Vf[x];
                            aG[1 + x] += aVf / (A)we.rho;
                            arho += -aVf * (A)we.Vf[x] / (A)we.rho;
                        }
                    }
                }
                if (!(we.gC[0] < P.dFloor)) aG[0] += arho;
            }
            for (int v = 0; v < 5; v++) dG[v * fs + cp] += (R)aG[v];
            for (int x = 0; x < 3; x++) dB[x * fs + cp] += (R)aB[x];
        }
    }
    if (P.bc[1] == BCK_ZEROGRAD && cellJK) {
        A ag[5] = {(A)0, (A)0, (A)0, (A)0, (A)0}, aB[3] = {(A)0, (A)0, (A)0};
        for (int n = 1; n <= 4; n++) {
            const long cg = at(ip + n);
            for (int v = 0; v < 5; v++) {
                ag[v] += (A)dG[v * fs + cg];
                dG[v * fs + cg] = (R)0;
            }
            const long cf[3] = {cg + 1, cg, cg};
            for (int d = 0; d < 3; d++) {
                const A a = (A)dM[d * fs + cf[d]] * (A)face[d * fs + cf[d]];
                dM[d * fs + cf[d]] = (R)0;
                for (int x = 0; x < 3; x++) aB[x] += a * (A)Tf[(9 * d + x) * fs + cf[d]];
            }
        }
        for (int v = 0; v < 5; v++) dG[v * fs + cp] += (R)ag[v];
        for (int x = 0; x < 3; x++) dB[x * fs + cp] += (R)aB[x];
    }
    if (P.bc[0] == BCK_SPHIN && cellJK) {
        const long src = at(G);
        A ag[5] = {(A)0, (A)0, (A)0, (A)0, (A)0}, af[3] = {(A)0, (A)0, (A)0};
        for (int n = 1; n <= 4; n++) {
            const long dst = at(G - n);
            for (int v = 0; v < 5; v++) {
                ag[v] += (A)dG[v * fs + dst];
                dG[v * fs + dst] = (R)0;
            }
            for (int x = 0; x < 3; x++) {
                af[x] += (A)dM[x * fs + dst];
                dM[x * fs + dst] = (R)0;
            }
        }
        for (int v = 0; v < 5; v++) dG[v * fs + src] += (R)ag[v];
        for (int x = 0; x < 3; x++) dM[x * fs + src] += (R)af[x];
    }
    if (P.bc[0] == BCK_INFLOW && cellJK)
        for (int n = 1; n <= 4; n++) {
            const long c = at(G - n);
            for (int v = 0; v < 5; v++) dG[v * fs + c] = (R)0;
            for (int d = 0; d < 3; d++) dM[d * fs + c] = (R)0;
        }
}

// Adjoint of the inflow state (rho, P, Vx, Vy, Vz, Bx, By, Bz) from the
// adjoints of the inflow's ghost cells and faces (before k_iside_adj zeroes
// them): one block, each thread a fixed set of (j, k) rows, then a fixed
// tree over the threads, in FP64 (deterministic); added into dw.
template <class R>
__global__ void __launch_bounds__(256) k_inflow_adj(GamBox b, DevParams<R> P, const R* __restrict__ face,
                                                    const R* __restrict__ Tf, ISideDev<R> is,
                                                    const R* __restrict__ dG, const R* __restrict__ dM, R* dw) {
    __shared__ double red[8][256];
    const int t = threadIdx.x;
    const long fs = b.fs;
    const int G = GAM_NG;
    const R gW[5] = {is.inflow[0], is.inflow[2], is.inflow[3], is.inflow[4], is.inflow[1]};
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    const long rows = (long)b.Nj * b.Nk;
    for (long q = t; q < rows; q += 256) {
        const int jj = (int)(q % b.Nj), kk = (int)(q / b.Nj);
        for (int n = 1; n <= 4; n++) {
            const long c = lidx(b, G - n, jj, kk);
            R aU[5], aW[5] = {(R)0, (R)0, (R)0, (R)0, (R)0};
            for (int v = 0; v < 5; v++) aU[v] = dG[v * fs + c];
            p2c_adj<R>(P.dFloor, P.pFloor, P.gm1, gW, aU, aW);
            acc[0] += (double)aW[0];
            acc[1] += (double)aW[4];
            for (int x = 0; x < 3; x++) acc[2 + x] += (double)aW[1 + x];
            for (int d = 0; d < 3; d++) {
                const double a = (double)dM[d * fs + c] * (double)face[d * fs + c];
                for (int x = 0; x < 3; x++) acc[5 + x] += a * (double)Tf[(9 * d + x) * fs + c];
            }
        }
    }
    for (int q = 0; q < 8; q++) red[q][t] = acc[q];
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
        if (t < h)
            for (int q = 0; q < 8; q++) red[q][t] += red[q][t + h];
        __syncthreads();
    }
    if (t < 8) dw[t] += (R)red[t][0];
}

}  // namespace gam_adj

// ------------------------------------------------------------ C ABI
#include "../../include/gamgpu.h"

namespace {
GamBox torch_box(int Nip, int Njp, int Nkp) {
    GamBox b;
    b.Nip = Nip; b.Njp = Njp; b.Nkp = Nkp;
    b.Ni = Nip + 2 * GAM_NG; b.Nj = Njp + 2 * GAM_NG; b.Nk = Nkp + 2 * GAM_NG;
    b.sx = b.Ni + 1;
    b.sk = (long)b.sx * (b.Nj + 1);
    b.nbox = b.sk * (b.Nk + 1);
    b.fs = b.nbox;
    return b;
}
template <class R> DevParams<R> dev_params(const gam_params* p) {
    DevParams<R> P;
    memset(&P, 0, sizeof(P));
    P.gamma = (R)p->gamma; P.gm1 = (R)(p->gamma - 1); P.CFL = (R)p->CFL; P.pdmb = (R)p->pdmb; P.Vd0 = (R)p->Vd0;
    P.cHogH = (R)p->cHogH; P.dFloor = (R)p->dFloor; P.pFloor = (R)p->pFloor;
    P.doMHD = p->doMHD; P.doLFMLim = p->doLFMLim; P.do25D = p->do25D; P.doBackground = p->doBackground;
    P.up7 = p->rmeth == GAM_RECON_7UP;
    for (int n = 0; n < 6; n++) P.bc[n] = p->bc[n];
    P.dtKlo = P.dtKhi = 1;
    P.dtIlo = P.dtIhi = P.dtJlo = P.dtJhi = 1;
    return P;
}
template <class R>
int flux_call(const gam_params* p, const void* QW, const void* Wn, const void* QB, const void* Blim, const void* Bnf,
              const void* vol, const void* face, const void* Tf, const double* fcB0, const double* bFlux0, void* gF,
              void* mF, const void* dgF, const void* dmF, void* dQW, void* dWn, void* dQB, void* dBlim, void* dBnf,
              cudaStream_t s, void* rscratch = nullptr, void* fstates = nullptr) {
    using namespace gam_adj;
    const GamBox b = torch_box(p->Nip, p->Njp, p->Nkp);
    const DevParams<R> P = dev_params<R>(p);
    Geo<R> g;
    memset(&g, 0, sizeof(g));
    g.vol = (const R*)vol; g.face = (const R*)face; g.Tf = (const R*)Tf;
    g.fcB0 = fcB0; g.bFlux0 = bFlux0;
    Work<R> w;
    memset(&w, 0, sizeof(w));
    w.QW = (R*)QW; w.Wn = (R*)Wn; w.QB = (R*)QB; w.Bnf = (R*)Bnf; w.gF = (R*)gF; w.mF = (R*)mF;
    w.fsv = (R*)fstates;  // non-null: the forward stores the face states, the adjoint loads them
    GamScalars* sc = nullptr;
    if (cudaGetSymbolAddress((void**)&sc, g_adj_scalars) != cudaSuccess) return GAM_ECUDA;
    const int G = GAM_NG;
    const Range fr[3] = {{G, G + b.Nip, G, G + b.Njp - 1, G, G + b.Nkp - 1},
                         {G, G + b.Nip - 1, G, G + b.Njp, G, G + b.Nkp - 1},
                         {G, G + b.Nip - 1, G, G + b.Njp - 1, G, G + b.Nkp}};
    const dim3 blk(16, 8, 1);
    auto grid = [&](const Range& r) {
        return dim3((unsigned)((r.i1 - r.i0 + 1 + blk.x - 1) / blk.x), (unsigned)((r.j1 - r.j0 + 1 + blk.y - 1) / blk.y),
                    (unsigned)((r.k1 - r.k0 + 1 + blk.z - 1) / blk.z));
    };
    const R* Bl = (const R*)Blim;
    if (!dgF && fstates) {
        k_stress<R, 0, 1, false, true><<<grid(fr[0]), blk, 0, s>>>(b, P, g, Bl, w, fr[0], sc, nullptr, nullptr);
        k_stress<R, 1, 1, false, true><<<grid(fr[1]), blk, 0, s>>>(b, P, g, Bl, w, fr[1], sc, nullptr, nullptr);
        k_stress<R, 2, 1, false, true><<<grid(fr[2]), blk, 0, s>>>(b, P, g, Bl, w, fr[2], sc, nullptr, nullptr);
    } else if (!dgF) {
        k_stress<R, 0, 1><<<grid(fr[0]), blk, 0, s>>>(b, P, g, Bl, w, fr[0], sc, nullptr, nullptr);
        k_stress<R, 1, 1><<<grid(fr[1]), blk, 0, s>>>(b, P, g, Bl, w, fr[1], sc, nullptr, nullptr);
        k_stress<R, 2, 1><<<grid(fr[2]), blk, 0, s>>>(b, P, g, Bl, w, fr[2], sc, nullptr, nullptr);
    } else if (fstates) {
        R* rs = (R*)rscratch;
        const long fs40 = 40L * b.fs;
        const R* a = (const R*)dgF;
        const R* m = (const R*)dmF;
        k_stress_adj<R, 0, true><<<grid(fr[0]), blk, 0, s>>>(b, P, g, Bl, w, fr[0], a, m, (R*)dQW, (R*)dWn, (R*)dQB,
                                                              (R*)dBlim, (R*)dBnf, rs);
        k_stress_adj<R, 1, true><<<grid(fr[1]), blk, 0, s>>>(b, P, g, Bl, w, fr[1], a, m, (R*)dQW, (R*)dWn, (R*)dQB,
                                                              (R*)dBlim, (R*)dBnf, rs ? rs + fs40 : nullptr);
        k_stress_adj<R, 2, true><<<grid(fr[2]), blk, 0, s>>>(b, P, g, Bl, w, fr[2], a, m, (R*)dQW, (R*)dWn, (R*)dQB,
                                                              (R*)dBlim, (R*)dBnf, rs ? rs + 2 * fs40 : nullptr);
        if (rs) {
            const dim3 gblk(32, 8, 1);
            const dim3 ggrid((unsigned)((b.Ni + gblk.x - 1) / gblk.x), (unsigned)((b.Nj + gblk.y - 1) / gblk.y),
                             (unsigned)b.Nk);
            k_stress_adj_gather3<R><<<ggrid, gblk, 0, s>>>(b, fr[0], fr[1], fr[2], rs, p->doMHD ? 8 : 5, (R*)dQW,
                                                           (R*)dWn, (R*)dQB, (R*)dBlim);
        }
    } else {
        const R* a = (const R*)dgF;
        const R* m = (const R*)dmF;
        // rs null: scatter with atomics; else each direction stores per face
        // (40 components from rs + 40 D fs), then one gather per cell stores
        // dQW, dWn, dQB and dBlim
        R* rs = (R*)rscratch;
        const long fs40 = 40L * b.fs;
        k_stress_adj<R, 0><<<grid(fr[0]), blk, 0, s>>>(b, P, g, Bl, w, fr[0], a, m, (R*)dQW, (R*)dWn, (R*)dQB,
                                                        (R*)dBlim, (R*)dBnf, rs);
        k_stress_adj<R, 1><<<grid(fr[1]), blk, 0, s>>>(b, P, g, Bl, w, fr[1], a, m, (R*)dQW, (R*)dWn, (R*)dQB,
                                                        (R*)dBlim, (R*)dBnf, rs ? rs + fs40 : nullptr);
        k_stress_adj<R, 2><<<grid(fr[2]), blk, 0, s>>>(b, P, g, Bl, w, fr[2], a, m, (R*)dQW, (R*)dWn, (R*)dQB,
                                                        (R*)dBlim, (R*)dBnf, rs ? rs + 2 * fs40 : nullptr);
        if (rs) {
            const dim3 gblk(32, 8, 1);
            const dim3 ggrid((unsigned)((b.Ni + gblk.x - 1) / gblk.x), (unsigned)((b.Nj + gblk.y - 1) / gblk.y),
                             (unsigned)b.Nk);
            k_stress_adj_gather3<R><<<ggrid, gblk, 0, s>>>(b, fr[0], fr[1], fr[2], rs, p->doMHD ? 8 : 5, (R*)dQW,
                                                           (R*)dWn, (R*)dQB, (R*)dBlim);
        }
    }
    return cudaGetLastError() == cudaSuccess ? GAM_OK : GAM_ECUDA;
}
int check(const gam_params* p, int32_t fp32) {
    if (!p) return GAM_EINVAL;
    if (p->rmeth != GAM_RECON_8CENT) return GAM_EINVAL;  // the adjoint covers 8CENT
    if (p->doBoris || p->doAB3) return GAM_EINVAL;      // and the step without Boris, with AB2
    if (p->nG != 4 || p->Nip < 1 || p->Njp < 1 || p->Nkp < 1 || p->do25D) return GAM_EBADDIM;
    (void)fp32;
    return GAM_OK;
}
}  // namespace

extern "C" int gam_flux_forward(const gam_params* p, int32_t fp32, const void* QW, const void* Wn, const void* QB,
                                const void* Blim, const void* Bnf, const void* volume, const void* face,
                                const void* Tf, const double* fcB0, const double* bFlux0, void* gF, void* mF,
                                void* stream) {
    int rc = check(p, fp32);
    if (rc) return rc;
    if (!QW || !Wn || !QB || !Blim || !Bnf || !volume || !face || !Tf || !gF || !mF) return GAM_EINVAL;
    if (p->doBackground && (!fcB0 || !bFlux0)) return GAM_EINVAL;
    cudaStream_t s = (cudaStream_t)stream;
    return fp32 ? flux_call<float>(p, QW, Wn, QB, Blim, Bnf, volume, face, Tf, fcB0, bFlux0, gF, mF, nullptr, nullptr,
                                   nullptr, nullptr, nullptr, nullptr, nullptr, s)
                : flux_call<double>(p, QW, Wn, QB, Blim, Bnf, volume, face, Tf, fcB0, bFlux0, gF, mF, nullptr, nullptr,
                                    nullptr, nullptr, nullptr, nullptr, nullptr, s);
}

extern "C" int gam_flux_adjoint(const gam_params* p, int32_t fp32, const void* QW, const void* Wn, const void* QB,
                                const void* Blim, const void* Bnf, const void* volume, const void* face,
                                const void* Tf, const double* fcB0, const double* bFlux0, const void* dgF,
                                const void* dmF, void* dQW, void* dWn, void* dQB, void* dBlim, void* dBnf,
                                void* stream) {
    int rc = check(p, fp32);
    if (rc) return rc;
    if (!QW || !Wn || !QB || !Blim || !Bnf || !volume || !face || !Tf || !dgF || !dmF || !dQW || !dWn || !dQB ||
        !dBlim || !dBnf)
        return GAM_EINVAL;
    if (p->doBackground && (!fcB0 || !bFlux0)) return GAM_EINVAL;
    cudaStream_t s = (cudaStream_t)stream;
    return fp32 ? flux_call<float>(p, QW, Wn, QB, Blim, Bnf, volume, face, Tf, fcB0, bFlux0, nullptr, nullptr, dgF,
                                   dmF, dQW, dWn, dQB, dBlim, dBnf, s)
                : flux_call<double>(p, QW, Wn, QB, Blim, Bnf, volume, face, Tf, fcB0, bFlux0, nullptr, nullptr, dgF,
                                    dmF, dQW, dWn, dQB, dBlim, dBnf, s);
}

namespace {
template <class R>
int efield_call(const gam_params* p, const void* Dh, const void* abh, const void* bn, const void* VdV, const void* vol,
                const void* face, const void* edge, const void* Te, const void* Teb, const double* edgB0, double dt,
                void* AVf, void* E, const void* dE, void* dDh, void* dabh, void* dbn, void* dVdV, void* dAVf,
                cudaStream_t s, bool avf_saved = false, void* escratch = nullptr, void* estates = nullptr) {
    using namespace gam_adj;
    const GamBox b = torch_box(p->Nip, p->Njp, p->Nkp);
    const DevParams<R> P = dev_params<R>(p);
    Geo<R> g;
    memset(&g, 0, sizeof(g));
    g.vol = (const R*)vol; g.face = (const R*)face; g.edge = (const R*)edge; g.Te = (const R*)Te; g.Teb = (const R*)Teb;
    g.edgB0 = edgB0;
    Work<R> w;
    memset(&w, 0, sizeof(w));
    w.Dh = (R*)Dh; w.abh = (R*)abh; w.bn = (R*)bn; w.VdV = (R*)VdV; w.AVf = (R*)AVf; w.E = (R*)E;
    w.esv = (R*)estates;  // non-null: the forward stores the corner values, the adjoint loads them
    GamScalars* sc = nullptr;
    if (cudaGetSymbolAddress((void**)&sc, g_adj_scalars) != cudaSuccess) return GAM_ECUDA;
    // the forward kernels read dt from the scalars; the adjoint with AVf kept
    // launches none of them
    if (!(dE && avf_saved)) k_adj_scalars<<<1, 1, 0, s>>>(sc, dt, 0.0, 0.0, 0);
    const int G = GAM_NG;
    const Range mf[3] = {{0, b.Ni - 1, G, G + b.Njp, 0, b.Nk - 1},
                         {0, b.Ni - 1, 0, b.Nj - 1, G, G + b.Nkp},
                         {G, G + b.Nip, 0, b.Nj - 1, 0, b.Nk - 1}};
    const Range ed[3] = {{G, G + b.Nip - 1, G, G + b.Njp, G, G + b.Nkp},
                         {G, G + b.Nip, G, G + b.Njp - 1, G, G + b.Nkp},
                         {G, G + b.Nip, G, G + b.Njp, G, G + b.Nkp - 1}};
    const dim3 blk(32, 4, 1);
    auto grid = [&](const Range& r) {
        return dim3((unsigned)((r.i1 - r.i0 + 1 + blk.x - 1) / blk.x), (unsigned)((r.j1 - r.j0 + 1 + blk.y - 1) / blk.y),
                    (unsigned)((r.k1 - r.k0 + 1 + blk.z - 1) / blk.z));
    };
    for (int eD = 0; eD < 3; eD++) {
        // the adjoint of a whole step finds AVf as its forward left it
        if (!(dE && avf_saved)) k_mom2face<R><<<grid(mf[eD]), blk, 0, s>>>(b, P, g, w, eD, mf[eD], sc);
        if (!dE && estates) {
            k_vxb<R, 1, true><<<grid(ed[eD]), blk, 0, s>>>(b, P, g, w, eD, ed[eD], sc);
        } else if (!dE) {
            k_vxb<R><<<grid(ed[eD]), blk, 0, s>>>(b, P, g, w, eD, ed[eD], sc);
        } else if (escratch) {
            // deterministic: the edges store their adjoints (14 components
            // from escratch + 14 eD fs), gathered per position after the third
            if (estates)
                k_vxb_adj<R, true><<<grid(ed[eD]), blk, 0, s>>>(b, P, g, w, eD, ed[eD], dt, (const R*)dE, (R*)dDh,
                                                                 (R*)dabh, (R*)dbn, (R*)dAVf,
                                                                 (R*)escratch + 14L * eD * b.fs);
            else
                k_vxb_adj<R><<<grid(ed[eD]), blk, 0, s>>>(b, P, g, w, eD, ed[eD], dt, (const R*)dE, (R*)dDh,
                                                           (R*)dabh, (R*)dbn, (R*)dAVf, (R*)escratch + 14L * eD * b.fs);
            if (eD == 2) {
                R* es = (R*)escratch;
                R* aS = es + 42L * b.fs;  // the scaled dAVf of the three edge directions
                const Range allF{0, b.Ni, 0, b.Nj, 0, b.Nk}, allC{0, b.Ni - 1, 0, b.Nj - 1, 0, b.Nk - 1};
                const Range3 ed3{{ed[0], ed[1], ed[2]}}, mf3{{mf[0], mf[1], mf[2]}};
                k_vxb_adj_gather3<R><<<grid(allF), blk, 0, s>>>(b, g, ed3, mf3, es, (R*)dDh, (R*)dabh, (R*)dbn, aS);
                k_m2f_adj_gather3<R><<<grid(allC), blk, 0, s>>>(b, mf3, aS, (R*)dVdV);
            }
        } else {
            if (cudaMemsetAsync(dAVf, 0, 3 * b.fs * sizeof(R), s) != cudaSuccess) return GAM_ECUDA;
            k_vxb_adj<R><<<grid(ed[eD]), blk, 0, s>>>(b, P, g, w, eD, ed[eD], dt, (const R*)dE, (R*)dDh, (R*)dabh,
                                                       (R*)dbn, (R*)dAVf, nullptr);
            k_m2f_adj<R><<<grid(mf[eD]), blk, 0, s>>>(b, g, eD, mf[eD], (const R*)dAVf, (R*)dVdV);
        }
    }
    return cudaGetLastError() == cudaSuccess ? GAM_OK : GAM_ECUDA;
}
}  // namespace

extern "C" int gam_efield_forward(const gam_params* p, int32_t fp32, const void* Dh, const void* abh, const void* bn,
                                  const void* VdV, const void* volume, const void* face, const void* edge,
                                  const void* Te, const void* Teb, const double* edgB0, double dt, void* AVf, void* E,
                                  void* stream) {
    int rc = check(p, fp32);
    if (rc) return rc;
    if (!Dh || !abh || !bn || !VdV || !volume || !face || !edge || !Te || !Teb || !AVf || !E || !(dt > 0.0))
        return GAM_EINVAL;
    if (p->doBackground && !edgB0) return GAM_EINVAL;
    cudaStream_t s = (cudaStream_t)stream;
    return fp32 ? efield_call<float>(p, Dh, abh, bn, VdV, volume, face, edge, Te, Teb, edgB0, dt, AVf, E, nullptr,
                                     nullptr, nullptr, nullptr, nullptr, nullptr, s)
                : efield_call<double>(p, Dh, abh, bn, VdV, volume, face, edge, Te, Teb, edgB0, dt, AVf, E, nullptr,
                                      nullptr, nullptr, nullptr, nullptr, nullptr, s);
}

extern "C" int gam_efield_adjoint(const gam_params* p, int32_t fp32, const void* Dh, const void* abh, const void* bn,
                                  const void* VdV, const void* volume, const void* face, const void* edge,
                                  const void* Te, const void* Teb, const double* edgB0, double dt, void* AVf,
                                  const void* dE, void* dDh, void* dabh, void* dbn, void* dVdV, void* dAVf,
                                  void* stream) {
    int rc = check(p, fp32);
    if (rc) return rc;
    if (!Dh || !abh || !bn || !VdV || !volume || !face || !edge || !Te || !Teb || !AVf || !dE || !dDh || !dabh ||
        !dbn || !dVdV || !dAVf || !(dt > 0.0))
        return GAM_EINVAL;
    if (p->doBackground && !edgB0) return GAM_EINVAL;
    cudaStream_t s = (cudaStream_t)stream;
    return fp32 ? efield_call<float>(p, Dh, abh, bn, VdV, volume, face, edge, Te, Teb, edgB0, dt, AVf, nullptr, dE,
                                     dDh, dabh, dbn, dVdV, dAVf, s)
                : efield_call<double>(p, Dh, abh, bn, VdV, volume, face, edge, Te, Teb, edgB0, dt, AVf, nullptr, dE,
                                      dDh, dabh, dbn, dVdV, dAVf, s);
}

// ------------------------------------------------------------ predictor and update stages
namespace {
template <class R> Geo<R> geo_of(const void* vol, const void* face, const void* xfc, const void* xyzcc, const void* dxf,
                                 const double* dpB0) {
    Geo<R> g;
    memset(&g, 0, sizeof(g));
    g.vol = (const R*)vol; g.face = (const R*)face; g.xfc = (const R*)xfc; g.xyzcc = (const R*)xyzcc;
    g.dxf = (const R*)dxf; g.dpB0 = dpB0;
    return g;
}
int set_scalars(double dt, double pdt, double odt, cudaStream_t s, GamScalars** sc) {
    if (cudaGetSymbolAddress((void**)sc, gam_adj::g_adj_scalars) != cudaSuccess) return GAM_ECUDA;
    gam_adj::k_adj_scalars<<<1, 1, 0, s>>>(*sc, dt, pdt, odt, 1);
    return cudaGetLastError() == cudaSuccess ? GAM_OK : GAM_ECUDA;
}
dim3 grid3(const Range& r, dim3 blk) {
    return dim3((unsigned)((r.i1 - r.i0 + 1 + blk.x - 1) / blk.x), (unsigned)((r.j1 - r.j0 + 1 + blk.y - 1) / blk.y),
                (unsigned)((r.k1 - r.k0 + 1 + blk.z - 1) / blk.z));
}
template <class R>
int predict_call(const gam_params* p, const void* const* st, const void* const* geo, double pdt, double odt,
                 void* const* out, const void* const* din, void* aB, void* const* dst, cudaStream_t s) {
    using namespace gam_adj;
    const GamBox b = torch_box(p->Nip, p->Njp, p->Nkp);
    const DevParams<R> P = dev_params<R>(p);
    const Geo<R> g = geo_of<R>(geo[0], geo[1], geo[2], geo[3], geo[4], nullptr);
    StateBuf<R> cur{(R*)st[0], (R*)st[1], nullptr}, old{(R*)st[2], (R*)st[3], nullptr};
    GamScalars* sc = nullptr;  // the forward kernels read pdt, odt from the scalars; the adjoint takes them as arguments
    if (out && set_scalars(0.0, pdt, odt, s, &sc)) return GAM_ECUDA;
    const Range all{0, b.Ni, 0, b.Nj, 0, b.Nk}, cells{0, b.Ni - 1, 0, b.Nj - 1, 0, b.Nk - 1};
    if (out) {
        Work<R> w;
        memset(&w, 0, sizeof(w));
        w.QW = (R*)out[0]; w.Wn = (R*)out[1]; w.Dh = (R*)out[2]; w.VdV = (R*)out[3]; w.QB = (R*)out[4];
        w.abh = (R*)out[5]; w.Bnf = (R*)out[6]; w.bn = (R*)out[7];
        const dim3 blk(32, 8, 1);
        k_predict<R, 1><<<grid3(all, blk), blk, 0, s>>>(b, P, g, cur, old, w, sc, nullptr);
    } else {
        Work<R> dw;
        memset(&dw, 0, sizeof(dw));
        dw.QW = (R*)din[0]; dw.Wn = (R*)din[1]; dw.Dh = (R*)din[2]; dw.VdV = (R*)din[3]; dw.QB = (R*)din[4];
        dw.abh = (R*)din[5]; dw.Bnf = (R*)din[6]; dw.bn = (R*)din[7];
        const dim3 blk(32, 4, 1);
        k_predict_adj_cells<R><<<grid3(cells, blk), blk, 0, s>>>(b, P, g, cur, old, pdt, odt, dw, (R*)dst[0],
                                                                  (R*)dst[2], (R*)aB);
        k_predict_adj_faces<R><<<grid3(all, blk), blk, 0, s>>>(b, P, g, pdt, odt, dw, (const R*)aB, (R*)dst[1],
                                                                (R*)dst[3]);
    }
    return cudaGetLastError() == cudaSuccess ? GAM_OK : GAM_ECUDA;
}
template <class R>
int update_call(const gam_params* p, const void* const* in, const void* const* geo, const double* dpB0, double dt,
                void* const* out, const void* const* din, void* sU, void* sM, void* const* dst, cudaStream_t s,
                bool assign = false) {
    using namespace gam_adj;
    const GamBox b = torch_box(p->Nip, p->Njp, p->Nkp);
    const DevParams<R> P = dev_params<R>(p);
    const Geo<R> g = geo_of<R>(geo[0], nullptr, geo[1], geo[2], geo[3], dpB0);
    // in: curGas, curMf, E, gF, mF
    StateBuf<R> cur{(R*)in[0], (R*)in[1], nullptr};
    Work<R> w;
    memset(&w, 0, sizeof(w));
    w.E = (R*)in[2]; w.gF = (R*)in[3]; w.mF = (R*)in[4];
    GamScalars* sc = nullptr;  // the forward kernels read dt from the scalars; the adjoint takes it as an argument
    if (out && set_scalars(dt, 0.0, 0.0, s, &sc)) return GAM_ECUDA;
    const Range all{0, b.Ni, 0, b.Nj, 0, b.Nk}, cells{0, b.Ni - 1, 0, b.Nj - 1, 0, b.Nk - 1};
    const dim3 blk(32, 4, 1);
    if (out) {
        StateBuf<R> nxt{(R*)out[0], (R*)out[1], (R*)out[2]};
        k_update_faces<R><<<grid3(all, blk), blk, 0, s>>>(b, P, cur, nxt, w, sc, nullptr);
        const double gamma = p->gamma, gm1 = p->gamma - 1;
        k_update_cells<R, 1><<<grid3(cells, blk), blk, 0, s>>>(b, P, g, cur, nxt, w, sc, gamma, gm1);
    } else {
        k_update_adj_cells<R><<<grid3(cells, blk), blk, 0, s>>>(b, P, g, cur, w, dt, (const R*)din[0], (R*)dst[0],
                                                                 (R*)sU, (R*)sM);
        k_update_adj_faces<R><<<grid3(all, blk), blk, 0, s>>>(b, P, dt, (const R*)sU, (const R*)sM, (const R*)din[1],
                                                               (R*)dst[1], (R*)dst[3], (R*)dst[4], (R*)dst[2],
                                                               assign ? 1 : 0);
    }
    return cudaGetLastError() == cudaSuccess ? GAM_OK : GAM_ECUDA;
}
}  // namespace

// st: curGas, curMf, oldGas, oldMf; geo: volume, face, xfc, xyzcc, dxf (FP32 only, else NULL)
// out (forward): QW, Wn, Dh, VdV, QB, abh, Bnf, bn
// din (adjoint): their adjoints; dst: dcurGas, dcurMf, doldGas, doldMf (added to); aB: 3-component scratch
extern "C" int gam_predict_stage(const gam_params* p, int32_t fp32, const void* const* st, const void* const* geo,
                                 double pdt, double odt, void* const* out, const void* const* din, void* aB,
                                 void* const* dst, void* stream) {
    int rc = check(p, fp32);
    if (rc) return rc;
    if (!st || !geo || (!out && (!din || !aB || !dst)) || !p->doLFMLim) return GAM_EINVAL;
    cudaStream_t s = (cudaStream_t)stream;
    return fp32 ? predict_call<float>(p, st, geo, pdt, odt, out, din, aB, dst, s)
                : predict_call<double>(p, st, geo, pdt, odt, out, din, aB, dst, s);
}
// in: curGas, curMf, E, gF, mF; geo: volume, xfc, xyzcc, dxf; dpB0 (FP64) when doBackground
// out (forward): nxtGas, nxtMf, nxtB (scratch); din (adjoint): dnxtGas, dnxtMf
// dst: dcurGas, dcurMf, dE, dgF, dmF (added to); sU (5) and sM (3) scratch
extern "C" int gam_update_stage(const gam_params* p, int32_t fp32, const void* const* in, const void* const* geo,
                                const double* dpB0, double dt, void* const* out, const void* const* din, void* sU,
                                void* sM, void* const* dst, void* stream) {
    int rc = check(p, fp32);
    if (rc) return rc;
    if (!in || !geo || (!out && (!din || !sU || !sM || !dst))) return GAM_EINVAL;
    if (p->doBackground && !dpB0) return GAM_EINVAL;
    cudaStream_t s = (cudaStream_t)stream;
    return fp32 ? update_call<float>(p, in, geo, dpB0, dt, out, din, sU, sM, dst, s)
                : update_call<double>(p, in, geo, dpB0, dt, out, din, sU, sM, dst, s);
}

// For the whole-step adjoint (gam_stepadj.cu), which owns its work area: the
// update stage's adjoint stores the face, flux and edge adjoints (dst[2..4])
// instead of adding into caller-zeroed arrays; the E-field adjoint finds AVf
// as the step's forward left it instead of recomputing Mom2Face; the flux and
// E-field adjoints store their stencil adjoints per face and per edge in
// scratch (120 and 51 box-sized components) and gather them per position in a
// fixed order, so that every call gives the same bits, and store (not add)
// dQW, dWn, dQB, dBlim, dDh, dabh, dbn and dVdV.
int gam_update_adjoint_store(const gam_params* p, int32_t fp32, const void* const* in, const void* const* geo,
                             const double* dpB0, double dt, const void* const* din, void* sU, void* sM,
                             void* const* dst, void* stream) {
    int rc = check(p, fp32);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    return fp32 ? update_call<float>(p, in, geo, dpB0, dt, nullptr, din, sU, sM, dst, s, true)
                : update_call<double>(p, in, geo, dpB0, dt, nullptr, din, sU, sM, dst, s, true);
}
int gam_efield_adjoint_saved(const gam_params* p, int32_t fp32, const void* Dh, const void* abh, const void* bn,
                             const void* VdV, const void* volume, const void* face, const void* edge, const void* Te,
                             const void* Teb, const double* edgB0, double dt, void* AVf, const void* dE, void* dDh,
                             void* dabh, void* dbn, void* dVdV, void* dAVf, void* scratch, const void* estates,
                             void* stream) {
    int rc = check(p, fp32);
    if (rc) return rc;
    if (!scratch || !estates) return GAM_EINVAL;
    cudaStream_t s = (cudaStream_t)stream;
    void* esv = const_cast<void*>(estates);
    return fp32 ? efield_call<float>(p, Dh, abh, bn, VdV, volume, face, edge, Te, Teb, edgB0, dt, AVf, nullptr, dE,
                                     dDh, dabh, dbn, dVdV, dAVf, s, true, scratch, esv)
                : efield_call<double>(p, Dh, abh, bn, VdV, volume, face, edge, Te, Teb, edgB0, dt, AVf, nullptr, dE,
                                      dDh, dabh, dbn, dVdV, dAVf, s, true, scratch, esv);
}
// CalcElecField into AVf, E that also stores the corner values (GAM_ESV_NC
// per edge and direction) for gam_efield_adjoint_saved
int gam_efield_forward_save(const gam_params* p, int32_t fp32, const void* Dh, const void* abh, const void* bn,
                            const void* VdV, const void* volume, const void* face, const void* edge, const void* Te,
                            const void* Teb, const double* edgB0, double dt, void* AVf, void* E, void* estates,
                            void* stream) {
    int rc = check(p, fp32);
    if (rc) return rc;
    if (!AVf || !E || !estates || !(dt > 0.0)) return GAM_EINVAL;
    cudaStream_t s = (cudaStream_t)stream;
    return fp32 ? efield_call<float>(p, Dh, abh, bn, VdV, volume, face, edge, Te, Teb, edgB0, dt, AVf, E, nullptr,
                                     nullptr, nullptr, nullptr, nullptr, nullptr, s, false, nullptr, estates)
                : efield_call<double>(p, Dh, abh, bn, VdV, volume, face, edge, Te, Teb, edgB0, dt, AVf, E, nullptr,
                                      nullptr, nullptr, nullptr, nullptr, nullptr, s, false, nullptr, estates);
}
int gam_flux_adjoint_gather(const gam_params* p, int32_t fp32, const void* QW, const void* Wn, const void* QB,
                            const void* Blim, const void* Bnf, const void* volume, const void* face, const void* Tf,
                            const double* fcB0, const double* bFlux0, const void* dgF, const void* dmF, void* dQW,
                            void* dWn, void* dQB, void* dBlim, void* dBnf, void* scratch, const void* fstates,
                            void* stream) {
    int rc = check(p, fp32);
    if (rc) return rc;
    if (!scratch || !fstates) return GAM_EINVAL;
    cudaStream_t s = (cudaStream_t)stream;
    void* fsv = const_cast<void*>(fstates);
    return fp32 ? flux_call<float>(p, QW, Wn, QB, Blim, Bnf, volume, face, Tf, fcB0, bFlux0, nullptr, nullptr, dgF,
                                   dmF, dQW, dWn, dQB, dBlim, dBnf, s, scratch, fsv)
                : flux_call<double>(p, QW, Wn, QB, Blim, Bnf, volume, face, Tf, fcB0, bFlux0, nullptr, nullptr, dgF,
                                    dmF, dQW, dWn, dQB, dBlim, dBnf, s, scratch, fsv);
}
// CalcStress into gF, mF that also stores the face states (GAM_FSV_NC per
// face and direction) for gam_flux_adjoint_gather
int gam_flux_forward_save(const gam_params* p, int32_t fp32, const void* QW, const void* Wn, const void* QB,
                          const void* Blim, const void* Bnf, const void* volume, const void* face, const void* Tf,
                          const double* fcB0, const double* bFlux0, void* gF, void* mF, void* fstates, void* stream) {
    int rc = check(p, fp32);
    if (rc) return rc;
    if (!gF || !mF || !fstates) return GAM_EINVAL;
    cudaStream_t s = (cudaStream_t)stream;
    return fp32 ? flux_call<float>(p, QW, Wn, QB, Blim, Bnf, volume, face, Tf, fcB0, bFlux0, gF, mF, nullptr, nullptr,
                                   nullptr, nullptr, nullptr, nullptr, nullptr, s, nullptr, fstates)
                : flux_call<double>(p, QW, Wn, QB, Blim, Bnf, volume, face, Tf, fcB0, bFlux0, gF, mF, nullptr, nullptr,
                                    nullptr, nullptr, nullptr, nullptr, nullptr, s, nullptr, fstates);
}

// ------------------------------------------------------------ I-side boundaries (C ABI)
namespace {
int iside_check(const gam_params* p) {
    const int a = p->bc[0], c = p->bc[1];
    const bool pin = a == GAM_BC_PERIODIC, pout = c == GAM_BC_PERIODIC;
    if (pin != pout) return GAM_EINVAL;
    if (!pin && a != GAM_BC_SPHIN && a != GAM_BC_INFLOW) return GAM_EINVAL;
    if (!pout && c != GAM_BC_ZEROGRAD && c != GAM_BC_WIND) return GAM_EINVAL;
    return GAM_OK;
}
template <class R>
int iside_dev(const gam_params* p, const gam_iside* is, gam_adj::ISideDev<R>& d) {
    memset(&d, 0, sizeof(d));
    const bool inflow = p->bc[0] == GAM_BC_INFLOW, wind = p->bc[1] == GAM_BC_WIND;
    if ((inflow || wind) && !is) return GAM_EINVAL;
    if (is)
        for (int q = 0; q < 8; q++) {
            d.inflow[q] = (R)is->inflow[q];
            d.wind[q] = (R)is->wind[q];
        }
    if (wind) {
        if (!is->wC) return GAM_EINVAL;
        d.wC = (const R*)is->wC;
        for (int x = 0; x < 3; x++) {
            if (!is->wF[x] || !is->sF[x]) return GAM_EINVAL;
            d.wF[x] = (const R*)is->wF[x];
            d.sF[x] = (const R*)is->sF[x];
        }
    }
    return GAM_OK;
}
template <class R>
int iside_call(const gam_params* p, const void* const* geo, const gam_iside* is, const void* Gas, const void* B,
               void* oGas, void* omf, void* dG, void* dM, void* dB, void* dw, cudaStream_t s) {
    using namespace gam_adj;
    ISideDev<R> d;
    int rc = iside_dev<R>(p, is, d);
    if (rc) return rc;
    const GamBox b = torch_box(p->Nip, p->Njp, p->Nkp);
    const DevParams<R> P = dev_params<R>(p);
    const R* face = (const R*)geo[0];
    const R* Tf = (const R*)geo[1];
    const dim3 blk(32, 8, 1), grd((unsigned)((b.Nj + 1 + 31) / 32), (unsigned)((b.Nk + 1 + 7) / 8), 1);
    if (oGas) {
        k_iside_fill<R><<<grd, blk, 0, s>>>(b, P, face, Tf, d, (const R*)B, (R*)oGas, (R*)omf);
    } else {
        if (dw && p->bc[0] == GAM_BC_INFLOW)
            k_inflow_adj<R><<<1, 256, 0, s>>>(b, P, face, Tf, d, (const R*)dG, (const R*)dM, (R*)dw);
        k_iside_adj<R><<<grd, blk, 0, s>>>(b, P, face, Tf, d, (const R*)Gas, (const R*)B, (R*)dG, (R*)dM, (R*)dB);
    }
    return cudaGetLastError() == cudaSuccess ? GAM_OK : GAM_ECUDA;
}
}  // namespace

extern "C" int gam_iside_fill(const gam_params* p, int32_t fp32, const void* const* geo, const gam_iside* is,
                              const void* B, void* Gas, void* mf, void* stream) {
    int rc = check(p, fp32);
    if (rc) return rc;
    if ((rc = iside_check(p))) return rc;
    if (!geo || !geo[0] || !geo[1] || !B || !Gas || !mf) return GAM_EINVAL;
    cudaStream_t s = (cudaStream_t)stream;
    return fp32 ? iside_call<float>(p, geo, is, nullptr, B, Gas, mf, nullptr, nullptr, nullptr, nullptr, s)
                : iside_call<double>(p, geo, is, nullptr, B, Gas, mf, nullptr, nullptr, nullptr, nullptr, s);
}

extern "C" int gam_iside_adjoint(const gam_params* p, int32_t fp32, const void* const* geo, const gam_iside* is,
                                 const void* Gas, const void* B, void* dGas, void* dMf, void* dB, void* dinflow,
                                 void* stream) {
    int rc = check(p, fp32);
    if (rc) return rc;
    if ((rc = iside_check(p))) return rc;
    if (!geo || !geo[0] || !geo[1] || !Gas || !B || !dGas || !dMf || !dB) return GAM_EINVAL;
    cudaStream_t s = (cudaStream_t)stream;
    return fp32 ? iside_call<float>(p, geo, is, Gas, B, nullptr, nullptr, dGas, dMf, dB, dinflow, s)
                : iside_call<double>(p, geo, is, Gas, B, nullptr, nullptr, dGas, dMf, dB, dinflow, s);
}
