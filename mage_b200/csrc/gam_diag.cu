// Diagnostics over the active cells with deterministic FP64 reductions:
// DivB (gridutils.F90:717-770), volume-weighted conserved totals, and the
// min(di,dj,dk) CFL length used by CellDT.
//
// Reduction order is fixed: NB blocks each stride over the active cells in a
// fixed pattern and reduce in shared memory by a fixed tree, then one block
// sums the NB partials by the same tree. Results do not depend on timing.
#include <cuda_runtime.h>
#include "gam_layout.cuh"

namespace {
constexpr int NB = 1024;  // blocks of the first pass
constexpr int NT = 256;   // threads per block

__device__ __forceinline__ long lidx(const GamBox& b, int ii, int jj, int kk) {
    return (long)ii + (long)b.sx * jj + b.sk * kk;
}
__device__ __forceinline__ void active_ijk(const GamBox& b, long n, int& ii, int& jj, int& kk) {
    ii = GAM_NG + (int)(n % b.Nip);
    long r = n / b.Nip;
    jj = GAM_NG + (int)(r % b.Njp);
    kk = GAM_NG + (int)(r / b.Njp);
}
template <int NV> __device__ void block_sum(double (*sh)[NT], double* acc, double* out) {
    for (int v = 0; v < NV; v++) sh[v][threadIdx.x] = acc[v];
    __syncthreads();
    for (int w = NT / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            for (int v = 0; v < NV; v++) sh[v][threadIdx.x] = sh[v][threadIdx.x] + sh[v][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int v = 0; v < NV; v++) out[v] = sh[v][0];
}

// bFlux0: background face fluxes (Model%doBackground) or null
template <class R> __global__ void k_divb(GamBox b, const R* __restrict__ mf, const double* __restrict__ bFlux0,
                                          double* partial) {
    __shared__ double sh[1][NT];
    const long n = (long)b.Nip * b.Njp * b.Nkp;
    const long fs = b.fs;
    double acc[1] = {0.0};
    for (long q = blockIdx.x * (long)NT + threadIdx.x; q < n; q += (long)NB * NT) {
        int ii, jj, kk;
        active_ijk(b, q, ii, jj, kk);
        long c = lidx(b, ii, jj, kk);
        double dFi = (double)mf[c] - (double)mf[c + 1];
        double dFj = (double)mf[fs + c] - (double)mf[fs + c + b.sx];
        double dFk = (double)mf[2 * fs + c] - (double)mf[2 * fs + c + b.sk];
        double dFi0 = 0.0, dFj0 = 0.0, dFk0 = 0.0;
        if (bFlux0) {
            dFi0 = bFlux0[c] - bFlux0[c + 1];
            dFj0 = bFlux0[fs + c] - bFlux0[fs + c + b.sx];
            dFk0 = bFlux0[2 * fs + c] - bFlux0[2 * fs + c + b.sk];
        }
        acc[0] += fabs(dFi + dFj + dFk + dFi0 + dFj0 + dFk0);
    }
    block_sum<1>(sh, acc, partial + blockIdx.x);
}
template <class R> __global__ void k_totals(GamBox b, const R* __restrict__ Gas, const R* __restrict__ vol, double* partial) {
    __shared__ double sh[5][NT];
    const long n = (long)b.Nip * b.Njp * b.Nkp;
    const long fs = b.fs;
    double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    for (long q = blockIdx.x * (long)NT + threadIdx.x; q < n; q += (long)NB * NT) {
        int ii, jj, kk;
        active_ijk(b, q, ii, jj, kk);
        long c = lidx(b, ii, jj, kk);
        double dV = (double)vol[c];
        for (int v = 0; v < 5; v++) acc[v] += (double)Gas[v * fs + c] * dV;
    }
    double o[5];
    block_sum<5>(sh, acc, o);
    if (threadIdx.x == 0)
        for (int v = 0; v < 5; v++) partial[v * NB + blockIdx.x] = o[v];
}
template <int NV> __global__ void k_final(const double* partial, double* out) {
    __shared__ double sh[NV][NT];
    double acc[NV];
    for (int v = 0; v < NV; v++) {
        acc[v] = 0.0;
        for (int q = threadIdx.x; q < NB; q += NT) acc[v] += partial[v * NB + q];
    }
    block_sum<NV>(sh, acc, out);
}
__global__ void k_min3(GamBox b, const double* __restrict__ dijk, double* dl) {
    long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (t >= b.nbox) return;
    double di = dijk[t], dj = dijk[b.fs + t], dk = dijk[2 * b.fs + t];
    double m = di;
    if (dj < m) m = dj;
    if (dk < m) m = dk;
    dl[t] = m;
}
}  // namespace

int gam_diag_partials(const GamBox&) { return NB; }

void gam_diag_divb(const GamBox& b, const double* mf, const double* bFlux0, double* partial, double* out,
                   cudaStream_t s) {
    k_divb<double><<<NB, NT, 0, s>>>(b, mf, bFlux0, partial);
    k_final<1><<<1, NT, 0, s>>>(partial, out);
}
void gam_diag_divb_f(const GamBox& b, const float* mf, const double* bFlux0, double* partial, double* out,
                     cudaStream_t s) {
    k_divb<float><<<NB, NT, 0, s>>>(b, mf, bFlux0, partial);
    k_final<1><<<1, NT, 0, s>>>(partial, out);
}
void gam_diag_totals(const GamBox& b, const double* Gas, const double* vol, double* partial, double* out,
                     cudaStream_t s) {
    k_totals<double><<<NB, NT, 0, s>>>(b, Gas, vol, partial);
    k_final<5><<<1, NT, 0, s>>>(partial, out);
}
void gam_diag_totals_f(const GamBox& b, const float* Gas, const float* vol, double* partial, double* out,
                       cudaStream_t s) {
    k_totals<float><<<NB, NT, 0, s>>>(b, Gas, vol, partial);
    k_final<5><<<1, NT, 0, s>>>(partial, out);
}
void gam_diag_min3(const GamBox& b, const double* dijk, double* dl, cudaStream_t s) {
    k_min3<<<(unsigned)((b.nbox + 255) / 256), 256, 0, s>>>(b, dijk, dl);
}
