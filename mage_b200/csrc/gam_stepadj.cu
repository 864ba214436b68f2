// One whole stepGamera of the differentiation form and its adjoint behind two
// C entry points (gam_step_fwd_save, gam_step_adj), on caller-owned device
// arrays in the unpadded box layout of the stage entry points
// (component-major (nc, Nk+1, Nj+1, Ni+1), i fastest). The stages are the
// ones gam_predict_stage, gam_efield_*, gam_flux_* and gam_update_stage run;
// this file adds what lies between them in the step:
//   * bFlux2Fld / gamCellBxyz (gridutils.F90:281-301, 648-680) on every cell
//     of the box, for the limiter field of the step's start and the field of
//     its end, and the adjoint of that linear map;
//   * the boundary conditions that copy values (periodic, bcs.F90:279-450;
//     zero-gradient J, bcs.F90:853-892), which EnforceBCs (step.F90:17-55)
//     applies I, then J, then K, composed into one source index per box
//     position (the K rule acts on the position first, then J, then I), as a gather from the update's result, and the adjoint of that
//     gather: every source position sums the adjoints of the positions copied
//     from it in ascending index order (deterministic, no atomics). With a
//     zero-gradient J the composed map is not a projection (the upper ghost
//     faces of I copy J-ghost faces that the map itself fills), so the gather
//     reads the update's result, never its own output.
// Compiled with -fmad=false: the cell-field map evaluates in the same order
// and rounding as the element-wise PyTorch restatement of the step, so both
// give the same bits.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <stdint.h>
#include <string.h>

#include "../../include/gamgpu.h"
#include "gam_bcmap.cuh"
#include "gam_ctx.cuh"
#include "gam_quot.cuh"

// stage adjoints for a whole step (gam_adjoint.cu)
int gam_update_adjoint_store(const gam_params* p, int32_t fp32, const void* const* in, const void* const* geo,
                             const double* dpB0, double dt, const void* const* din, void* sU, void* sM,
                             void* const* dst, void* stream);
int gam_efield_adjoint_saved(const gam_params* p, int32_t fp32, const void* Dh, const void* abh, const void* bn,
                             const void* VdV, const void* volume, const void* face, const void* edge, const void* Te,
                             const void* Teb, const double* edgB0, double dt, void* AVf, const void* dE, void* dDh,
                             void* dabh, void* dbn, void* dVdV, void* dAVf, void* scratch, const void* estates,
                             void* stream);
int gam_efield_forward_save(const gam_params* p, int32_t fp32, const void* Dh, const void* abh, const void* bn,
                            const void* VdV, const void* volume, const void* face, const void* edge, const void* Te,
                            const void* Teb, const double* edgB0, double dt, void* AVf, void* E, void* estates,
                            void* stream);
int gam_flux_adjoint_gather(const gam_params* p, int32_t fp32, const void* QW, const void* Wn, const void* QB,
                            const void* Blim, const void* Bnf, const void* volume, const void* face, const void* Tf,
                            const double* fcB0, const double* bFlux0, const void* dgF, const void* dmF, void* dQW,
                            void* dWn, void* dQB, void* dBlim, void* dBnf, void* scratch, const void* fstates,
                            void* stream);
int gam_flux_forward_save(const gam_params* p, int32_t fp32, const void* QW, const void* Wn, const void* QB,
                          const void* Blim, const void* Bnf, const void* volume, const void* face, const void* Tf,
                          const double* fcB0, const double* bFlux0, void* gF, void* mF, void* fstates, void* stream);

namespace gam_stepadj {

// out[c][t] = in[c][src(t)] for the nc components of a field
template <class R>
__global__ void k_bc_gather(Box b, int comp, int nc, const R* __restrict__ in, R* __restrict__ out) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    int i, j, k;
    if (!pos_of(b, t, i, j, k)) return;
    const long s = bc_source(b, comp, i, j, k);
    for (int c = 0; c < nc; c++) out[c * b.n + t] = in[c * b.n + s];
}

// adjoint of the four gathers of EnforceBCs (the gas, 5 components, and the
// flux of each direction) in one launch, blockIdx.y = the field f (0 gas,
// 1 + d flux d), from the tables of bc_adj_tables: out[s] = (g[s] where the
// map fixes s, else 0) + the sum of g over the positions that copy s, in
// ascending order
struct BcAdjDev {
    const int* code[4];
    const int* rowStart[4];
    const int* src[4];
};
template <class R>
__global__ void __launch_bounds__(256) k_bc_gather_adj_tab(Box b, BcAdjDev tab, const R* __restrict__ gG,
                                                           R* __restrict__ oG, const R* __restrict__ gM,
                                                           R* __restrict__ oM) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= b.n) return;
    const int f = blockIdx.y;
    const long n = b.n;
    const int nc = f == 0 ? 5 : 1;
    const R* g = f == 0 ? gG : gM + (long)(f - 1) * n;
    R* out = f == 0 ? oG : oM + (long)(f - 1) * n;
    const int code = tab.code[f][t];
    const int row = (code >> 1) - 1;
    int q0 = 0, q1 = 0;
    if (row >= 0) {
        q0 = tab.rowStart[f][row];
        q1 = tab.rowStart[f][row + 1];
    }
    const int* src = tab.src[f];
    for (int c = 0; c < nc; c++) {
        const R own = (code & 1) ? g[c * n + t] : (R)0;
        if (q1 > q0) {
            R acc = g[c * n + src[q0]];
            for (int q = q0 + 1; q < q1; q++) acc = acc + g[c * n + src[q]];
            out[c * n + t] = own + acc;
        } else {
            out[c * n + t] = own;
        }
    }
}

// gamCellBxyz on every cell of the box: B = (sum over faces of +-flux x face
// centroid)/V - div * cell centroid / V in FP64; in FP32 with the face-minus-
// cell centroid offsets dxf (x + 6 d: lower face of direction d, x + 3 + 6 d:
// upper face)
template <class R>
__global__ void k_box_bxyz(Box b, const R* __restrict__ vol, const R* __restrict__ xfc, const R* __restrict__ xyzcc,
                           const R* __restrict__ dxf, const R* __restrict__ mf, R* __restrict__ B) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    int i, j, k;
    if (!pos_of(b, t, i, j, k) || i >= b.Ni || j >= b.Nj || k >= b.Nk) return;
    const long n = b.n, sj = b.nx, sk = (long)b.nx * b.ny;
    const R fI = mf[t], fIp = mf[t + 1], fJ = mf[n + t], fJp = mf[n + t + sj], fK = mf[2 * n + t],
            fKp = mf[2 * n + t + sk];
    const R dV = vol[t];
    if (dxf) {
        for (int x = 0; x < 3; x++) {
            const R s = fIp * dxf[(x + 3) * n + t] + fJp * dxf[(x + 9) * n + t] + fKp * dxf[(x + 15) * n + t] -
                        fI * dxf[x * n + t] - fJ * dxf[(x + 6) * n + t] - fK * dxf[(x + 12) * n + t];
            B[x * n + t] = s / dV;
        }
        return;
    }
    const R Div = fIp - fI + fJp - fJ + fKp - fK;
    for (int x = 0; x < 3; x++) {
        const R s = fIp * xfc[x * n + t + 1] + fJp * xfc[(x + 3) * n + t + sj] + fKp * xfc[(x + 6) * n + t + sk] -
                    fI * xfc[x * n + t] - fJ * xfc[(x + 3) * n + t] - fK * xfc[(x + 6) * n + t];
        const R tt = s / dV;
        B[x * n + t] = tt - Div * xyzcc[x * n + t] / dV;
    }
}

// adjoint of k_box_bxyz: every face of direction d adds the adjoints of the
// two cells it bounds (the cell below as its upper face, the cell at its own
// index as its lower face)
// quotients by one divisor, equal to the IEEE quotient (FP64: gam::QuotExact,
// one division per divisor; FP32: the division)
template <class R>
struct DivBy {
    R d;
    __device__ explicit DivBy(R dd) : d(dd) {}
    __device__ R operator()(R a) const { return a / d; }
};
template <>
struct DivBy<double> {
    gam::QuotExact q;
    __device__ explicit DivBy(double dd) : q(dd) {}
    __device__ double operator()(double a) const { return q(a); }
};

template <class R>
__global__ void k_box_bxyz_adj(Box b, const R* __restrict__ vol, const R* __restrict__ xfc,
                               const R* __restrict__ xyzcc, const R* __restrict__ dxf, const R* __restrict__ gB,
                               R* __restrict__ dmf) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    int i, j, k;
    if (!pos_of(b, t, i, j, k)) return;
    const long n = b.n;
    const long st[3] = {1, (long)b.nx, (long)b.nx * b.ny};
    const int p[3] = {i, j, k};
    const int N[3] = {b.Ni, b.Nj, b.Nk};
    const bool inCell = i < b.Ni && j < b.Nj && k < b.Nk;
    const DivBy<R> byV(inCell ? vol[t] : (R)1);
#pragma unroll
    for (int d = 0; d < 3; d++) {
        bool below = p[d] >= 1;
        for (int a = 0; a < 3; a++)
            if (p[a] >= N[a] + (a == d ? 1 : 0)) below = false;
        R acc = (R)0;
        if (below) {
            const long c = t - st[d];
            const DivBy<R> byVc(vol[c]);
            for (int x = 0; x < 3; x++) {
                const R w = dxf ? dxf[(x + 3 + 6 * d) * n + c] : xfc[(x + 3 * d) * n + t] - xyzcc[x * n + c];
                acc = acc + byVc(gB[x * n + c] * w);
            }
        }
        if (inCell) {
            for (int x = 0; x < 3; x++) {
                const R w = dxf ? dxf[(x + 6 * d) * n + t] : xfc[(x + 3 * d) * n + t] - xyzcc[x * n + t];
                acc = acc - byV(gB[x * n + t] * w);
            }
        }
        dmf[d * n + t] += acc;
    }
}

unsigned blocks(long n, int blk) { return (unsigned)((n + blk - 1) / blk); }

// Side streams of the adjoint step (created once per device, non-blocking):
// independent stages run on them between a fork and a join by events, on
// the caller's stream or inside a graph captured from it.
constexpr int NSIDE = 1;
struct SideStreams {
    cudaStream_t s[NSIDE];
    cudaEvent_t fork, join[NSIDE];
    bool ok;
};
SideStreams* side_streams() {
    static std::mutex mu;
    static SideStreams per[64];
    static bool made[64];
    static unsigned long long ctx[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> lock(mu);
    SideStreams& t = per[dev];
    // made again in a new context of the device (after cudaDeviceReset); the
    // old handles died with their context
    const unsigned long long id = gam_current_ctx_id();
    if (!made[dev] || id != ctx[dev]) {
        made[dev] = true;
        ctx[dev] = id;
        t.ok = cudaEventCreateWithFlags(&t.fork, cudaEventDisableTiming) == cudaSuccess;
        for (int i = 0; i < NSIDE && t.ok; i++)
            t.ok = cudaStreamCreateWithFlags(&t.s[i], cudaStreamNonBlocking) == cudaSuccess &&
                   cudaEventCreateWithFlags(&t.join[i], cudaEventDisableTiming) == cudaSuccess;
    }
    return t.ok ? &t : nullptr;
}
// the side streams i < n wait for the work issued so far on s
int fork(const SideStreams* t, int n, cudaStream_t s) {
    if (cudaEventRecord(t->fork, s) != cudaSuccess) return GAM_ECUDA;
    for (int i = 0; i < n; i++)
        if (cudaStreamWaitEvent(t->s[i], t->fork, 0) != cudaSuccess) return GAM_ECUDA;
    return GAM_OK;
}
// s waits for the work issued so far on the side streams i < n
int join(const SideStreams* t, int n, cudaStream_t s) {
    for (int i = 0; i < n; i++)
        if (cudaEventRecord(t->join[i], t->s[i]) != cudaSuccess || cudaStreamWaitEvent(s, t->join[i], 0) != cudaSuccess)
            return GAM_ECUDA;
    return GAM_OK;
}

// work arrays, each of nc components; a start on 64 elements
enum Slot {
    QW, Wn, Dh, VdV, QB, abh, Bnf, bn, AVf, E, Blim, gF, mF,                                      // forward
    FSV, ESV,  // the flux kernels' face states and the edge kernels' corner values per direction
               // (written before they are read: not zeroed)
    dQW, dWn, dDh, dVdV, dQB, dabh, dBnf, dbn, dAVf, dE, dgF, dmF, dBlim, sU, sM, aB, dnG, dnM, tM,  // adjoint
    RS,  // scratch of the deterministic gathers: the flux adjoint's per-face reconstruction adjoints
         // (3 directions x 8 variables x 5), after them the edge adjoints (3 x 14) and the scaled dAVf
         // (3 x 3), apart so that the two adjoints run at the same time
    UG, UM, UB, aBm,  // non-periodic I only: the update's result after the I-side fills, the field of its
                      // fluxes before them, and that field's adjoint
    NSLOT
};
constexpr int slot_nc[NSLOT] = {5, 5, 1, 3, 3, 3, 3, 3, 9, 3, 3, 15, 9, 66, 30,  // 3 x GAM_FSV_NC, 3 x GAM_ESV_NC
                                5, 5, 1, 3, 3, 3, 3, 3, 3, 3, 15, 9, 3, 5, 3, 3, 5, 3, 3, 171,
                                5, 3, 3, 3};
bool has_iside(const gam_params* p) { return p->bc[0] != GAM_BC_PERIODIC; }

struct Work {
    void* p[NSLOT];
    size_t fwd_bytes, bytes;
};
Work layout(const Box& b, int fp32, void* base, bool iside) {
    const size_t es = fp32 ? 4 : 8;
    Work w;
    size_t off = 0;
    for (int s = 0; s < NSLOT; s++) {
        if (s == FSV) w.fwd_bytes = off;
        w.p[s] = base ? (void*)((char*)base + off) : nullptr;
        const size_t bytes = (s >= UG && !iside) ? 0 : (size_t)slot_nc[s] * (size_t)b.n * es;
        off += (bytes + 255) / 256 * 256;
    }
    w.bytes = off;
    return w;
}

int check(const gam_params* p) {
    if (!p) return GAM_EINVAL;
    if (p->rmeth != GAM_RECON_8CENT || p->doBoris || p->doAB3 || !p->doLFMLim || !p->doMHD) return GAM_EINVAL;
    if (p->nG != 4 || p->Nip < 1 || p->Njp < 4 || p->Nkp < 1 || p->do25D) return GAM_EBADDIM;
    if ((double)(p->Nip + 9) * (p->Njp + 9) * (p->Nkp + 9) >= 2147483648.0) return GAM_EBADDIM;  // 32-bit indexing
    // boundaries: periodic I, or SphIn / inflow inside and zero-gradient /
    // wind outside; periodic K; periodic or zero-gradient J
    const bool ip = p->bc[0] == GAM_BC_PERIODIC && p->bc[1] == GAM_BC_PERIODIC;
    const bool is = (p->bc[0] == GAM_BC_SPHIN || p->bc[0] == GAM_BC_INFLOW) &&
                    (p->bc[1] == GAM_BC_ZEROGRAD || p->bc[1] == GAM_BC_WIND);
    if (!ip && !is) return GAM_EINVAL;
    if (p->bc[4] != GAM_BC_PERIODIC || p->bc[5] != GAM_BC_PERIODIC) return GAM_EINVAL;
    const bool jp = p->bc[2] == GAM_BC_PERIODIC && p->bc[3] == GAM_BC_PERIODIC;
    const bool jz = p->bc[2] == GAM_BC_ZEROGRAD && p->bc[3] == GAM_BC_ZEROGRAD;
    if (!jp && !jz) return GAM_EINVAL;
    return GAM_OK;
}

template <class R>
int launch_bxyz(const Box& b, const void* const* geo, const void* mf, void* B, cudaStream_t s) {
    k_box_bxyz<R><<<blocks(b.n, 256), 256, 0, s>>>(b, (const R*)geo[0], (const R*)geo[2], (const R*)geo[3],
                                                   (const R*)geo[4], (const R*)mf, (R*)B);
    return cudaGetLastError() == cudaSuccess ? GAM_OK : GAM_ECUDA;
}
template <class R>
int launch_bxyz_adj(const Box& b, const void* const* geo, const void* gB, void* dmf, cudaStream_t s) {
    k_box_bxyz_adj<R><<<blocks(b.n, 256), 256, 0, s>>>(b, (const R*)geo[0], (const R*)geo[2], (const R*)geo[3],
                                                       (const R*)geo[4], (const R*)gB, (R*)dmf);
    return cudaGetLastError() == cudaSuccess ? GAM_OK : GAM_ECUDA;
}
template <class R>
int launch_gather(const Box& b, int comp, int nc, const void* in, void* out, cudaStream_t s) {
    k_bc_gather<R><<<blocks(b.n, 256), 256, 0, s>>>(b, comp, nc, (const R*)in, (R*)out);
    return cudaGetLastError() == cudaSuccess ? GAM_OK : GAM_ECUDA;
}
// the tables of the EnforceBCs adjoint for this configuration on the current
// device and context, built and uploaded on first use (synchronous copies)
// and kept for the life of the process
int bc_adj_device_tables(const Box& b, BcAdjDev* out) {
    struct Entry {
        int dev, Nip, Njp, Nkp, bc[6];
        unsigned long long ctx;  // uploaded again in a new context of the device (after cudaDeviceReset)
        BcAdjDev d;
    };
    static std::mutex mu;
    static std::vector<Entry> cache;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return GAM_ECUDA;
    std::lock_guard<std::mutex> lock(mu);
    const unsigned long long ctx = gam_current_ctx_id();
    for (const Entry& e : cache)
        if (e.dev == dev && e.ctx == ctx && e.Nip == b.Nip && e.Njp == b.Njp && e.Nkp == b.Nkp &&
            std::equal(e.bc, e.bc + 6, b.bc)) {
            *out = e.d;
            return GAM_OK;
        }
    Entry e;
    e.dev = dev; e.ctx = ctx; e.Nip = b.Nip; e.Njp = b.Njp; e.Nkp = b.Nkp;
    std::copy(b.bc, b.bc + 6, e.bc);
    for (int f = 0; f < 4; f++) {
        std::vector<int> code, rowStart, src;
        bc_adj_tables(b, f - 1, code, rowStart, src);
        const std::vector<int>* v[3] = {&code, &rowStart, &src};
        const int** dst[3] = {&e.d.code[f], &e.d.rowStart[f], &e.d.src[f]};
        for (int q = 0; q < 3; q++) {
            int* d = nullptr;
            const size_t bytes = std::max<size_t>(1, v[q]->size()) * sizeof(int);
            if (cudaMalloc((void**)&d, bytes) != cudaSuccess) return GAM_ECUDA;
            if (!v[q]->empty() && cudaMemcpy(d, v[q]->data(), v[q]->size() * sizeof(int), cudaMemcpyHostToDevice) !=
                                      cudaSuccess)
                return GAM_ECUDA;
            *dst[q] = d;
        }
    }
    cache.push_back(e);
    *out = e.d;
    return GAM_OK;
}

#define TRY(x)              \
    do {                    \
        int rc_ = (x);      \
        if (rc_) return rc_; \
    } while (0)

// predictor, the limiter field of the start, electric field and fluxes into
// the forward slots of the work area
int forward_stages(const gam_params* p, int fp32, const Box& b, const Work& w, const void* const* geo,
                   const double* const* bg, const void* const* st, double dt, double odt, cudaStream_t s) {
    if (cudaMemsetAsync(w.p[0], 0, w.fwd_bytes, s) != cudaSuccess) return GAM_ECUDA;
    const void* g5[5] = {geo[0], geo[1], geo[2], geo[3], geo[4]};
    void* out8[8] = {w.p[QW], w.p[Wn], w.p[Dh], w.p[VdV], w.p[QB], w.p[abh], w.p[Bnf], w.p[bn]};
    TRY(gam_predict_stage(p, fp32, st, g5, 0.5 * dt, odt, out8, nullptr, nullptr, nullptr, s));
    TRY(fp32 ? launch_bxyz<float>(b, geo, st[1], w.p[Blim], s) : launch_bxyz<double>(b, geo, st[1], w.p[Blim], s));
    TRY(gam_efield_forward_save(p, fp32, w.p[Dh], w.p[abh], w.p[bn], w.p[VdV], geo[0], geo[1], geo[5], geo[6],
                                geo[7], bg ? bg[2] : nullptr, dt, w.p[AVf], w.p[E], w.p[ESV], s));
    TRY(gam_flux_forward_save(p, fp32, w.p[QW], w.p[Wn], w.p[QB], w.p[Blim], w.p[Bnf], geo[0], geo[1], geo[8],
                              bg ? bg[0] : nullptr, bg ? bg[1] : nullptr, w.p[gF], w.p[mF], w.p[FSV], s));
    return GAM_OK;
}

int args_ok(const gam_params* p, const void* const* geo, const double* const* bg, const void* const* st, int fp32,
            void* work) {
    if (!geo || !st || !work) return GAM_EINVAL;
    for (int q = 0; q < 9; q++)
        if (!geo[q] && q != 4) return GAM_EINVAL;
    if (fp32 && !geo[4]) return GAM_EINVAL;
    for (int q = 0; q < 4; q++)
        if (!st[q]) return GAM_EINVAL;
    if (p->doBackground && (!bg || !bg[0] || !bg[1] || !bg[2] || !bg[3])) return GAM_EINVAL;
    return GAM_OK;
}

}  // namespace gam_stepadj

using namespace gam_stepadj;

extern "C" int gam_step_work_bytes(const gam_params* p, int32_t fp32, int64_t* bytes) {
    TRY(check(p));
    if (!bytes) return GAM_EINVAL;
    *bytes = (int64_t)layout(make_box(p), fp32, nullptr, has_iside(p)).bytes;
    return GAM_OK;
}

namespace gam_stepadj {
// applyUpdate into UG, UM (Bs its scratch), bFlux2Fld of its fluxes into UB,
// then the I-side fills of UG, UM in place
int update_and_fill(const gam_params* p, int fp32, const Box& b, const Work& w, const void* const* geo,
                    const double* const* bg, const void* const* st, double dt, const gam_iside* is, void* Bs,
                    cudaStream_t s) {
    const size_t es = fp32 ? 4 : 8;
    if (cudaMemsetAsync(w.p[UG], 0, 5 * b.n * es, s) != cudaSuccess ||
        cudaMemsetAsync(w.p[UM], 0, 3 * b.n * es, s) != cudaSuccess ||
        cudaMemsetAsync(w.p[UB], 0, 3 * b.n * es, s) != cudaSuccess ||
        cudaMemsetAsync(Bs, 0, 3 * b.n * es, s) != cudaSuccess)
        return GAM_ECUDA;
    const void* in5[5] = {st[0], st[1], w.p[E], w.p[gF], w.p[mF]};
    const void* g4[4] = {geo[0], geo[2], geo[3], geo[4]};
    void* upd[3] = {w.p[UG], w.p[UM], Bs};
    TRY(gam_update_stage(p, fp32, in5, g4, bg ? bg[3] : nullptr, dt, upd, nullptr, nullptr, nullptr, nullptr, s));
    TRY(fp32 ? launch_bxyz<float>(b, geo, w.p[UM], w.p[UB], s) : launch_bxyz<double>(b, geo, w.p[UM], w.p[UB], s));
    const void* g2[2] = {geo[1], geo[8]};
    return gam_iside_fill(p, fp32, g2, is, w.p[UB], w.p[UG], w.p[UM], s);
}

int step_fwd_save(const gam_params* p, int32_t fp32, const void* const* geo, const double* const* bg,
                  const gam_iside* is, const void* const* st, double dt, double odt, void* const* nxt, void* work,
                  void* stream) {
    TRY(check(p));
    TRY(args_ok(p, geo, bg, st, fp32, work));
    if (!nxt || !nxt[0] || !nxt[1] || !nxt[2]) return GAM_EINVAL;
    cudaStream_t s = (cudaStream_t)stream;
    const Box b = make_box(p);
    const bool iside = has_iside(p);
    const Work w = layout(b, fp32, work, iside);
    const size_t es = fp32 ? 4 : 8;
    TRY(forward_stages(p, fp32, b, w, geo, bg, st, dt, odt, s));
    if (iside) {
        // applyUpdate and the I-side fills into UG, UM (kept for the adjoint),
        // then the copying boundaries and the closing bFlux2Fld
        TRY(update_and_fill(p, fp32, b, w, geo, bg, st, dt, is, nxt[2], s));
        if (fp32) {
            TRY(launch_gather<float>(b, -1, 5, w.p[UG], nxt[0], s));
            for (int d = 0; d < 3; d++)
                TRY(launch_gather<float>(b, d, 1, (float*)w.p[UM] + d * b.n, (float*)nxt[1] + d * b.n, s));
        } else {
            TRY(launch_gather<double>(b, -1, 5, w.p[UG], nxt[0], s));
            for (int d = 0; d < 3; d++)
                TRY(launch_gather<double>(b, d, 1, (double*)w.p[UM] + d * b.n, (double*)nxt[1] + d * b.n, s));
        }
        if (cudaMemsetAsync(nxt[2], 0, 3 * b.n * es, s) != cudaSuccess) return GAM_ECUDA;
        return fp32 ? launch_bxyz<float>(b, geo, nxt[1], nxt[2], s) : launch_bxyz<double>(b, geo, nxt[1], nxt[2], s);
    }
    // applyUpdate into the work area (the adjoint's dnG, dnM arrays, free until
    // gam_step_adj), nxtB as its scratch
    void* upd[3] = {w.p[dnG], w.p[dnM], nxt[2]};
    if (cudaMemsetAsync(w.p[dnG], 0, 5 * b.n * es, s) != cudaSuccess ||
        cudaMemsetAsync(w.p[dnM], 0, 3 * b.n * es, s) != cudaSuccess ||
        cudaMemsetAsync(nxt[2], 0, 3 * b.n * es, s) != cudaSuccess)
        return GAM_ECUDA;
    const void* in5[5] = {st[0], st[1], w.p[E], w.p[gF], w.p[mF]};
    const void* g4[4] = {geo[0], geo[2], geo[3], geo[4]};
    TRY(gam_update_stage(p, fp32, in5, g4, bg ? bg[3] : nullptr, dt, upd, nullptr, nullptr, nullptr, nullptr, s));
    // EnforceBCs, then the closing bFlux2Fld
    if (fp32) {
        TRY(launch_gather<float>(b, -1, 5, upd[0], nxt[0], s));
        for (int d = 0; d < 3; d++)
            TRY(launch_gather<float>(b, d, 1, (float*)upd[1] + d * b.n, (float*)nxt[1] + d * b.n, s));
    } else {
        TRY(launch_gather<double>(b, -1, 5, upd[0], nxt[0], s));
        for (int d = 0; d < 3; d++)
            TRY(launch_gather<double>(b, d, 1, (double*)upd[1] + d * b.n, (double*)nxt[1] + d * b.n, s));
    }
    if (cudaMemsetAsync(nxt[2], 0, 3 * b.n * es, s) != cudaSuccess) return GAM_ECUDA;
    return fp32 ? launch_bxyz<float>(b, geo, nxt[1], nxt[2], s) : launch_bxyz<double>(b, geo, nxt[1], nxt[2], s);
}

int step_adj(const gam_params* p, int32_t fp32, const void* const* geo, const double* const* bg, const gam_iside* is,
             const void* const* st, double dt, double odt, int32_t saved, const void* const* dnxt, void* const* dst,
             void* dinflow, void* work, void* stream) {
    TRY(check(p));
    TRY(args_ok(p, geo, bg, st, fp32, work));
    if (!dnxt || !dnxt[0] || !dnxt[1] || !dst || !dst[0] || !dst[1] || !dst[2] || !dst[3]) return GAM_EINVAL;
    cudaStream_t s = (cudaStream_t)stream;
    const Box b = make_box(p);
    const bool iside = has_iside(p);
    const Work w = layout(b, fp32, work, iside);
    const size_t es = fp32 ? 4 : 8;
    if (!saved) TRY(forward_stages(p, fp32, b, w, geo, bg, st, dt, odt, s));
    if (!saved && iside) TRY(update_and_fill(p, fp32, b, w, geo, bg, st, dt, is, w.p[aBm], s));
    // zero what the adjoint stages add into: dBnf (each flux adds its face's
    // part). The gathers store dQW, dWn, dQB, dBlim, dDh and dVdV on every
    // cell and dabh, dbn on every position, which is all the later stages
    // read of them; dAVf is not used with the gathers; the update stage stores
    // dE, dgF and dmF whole, sU, sM and aB are written before they are read,
    // dnG and dnM are written whole
    if (cudaMemsetAsync(w.p[dBnf], 0, 3 * b.n * es, s) != cudaSuccess) return GAM_ECUDA;
    // adjoint of the state's field: B = bFlux2Fld(magFlux), added to a copy
    // of the flux adjoint (read in place when there is no field adjoint)
    const void* gMf = dnxt[1];
    if (dnxt[2]) {
        if (cudaMemcpyAsync(w.p[tM], dnxt[1], 3 * b.n * es, cudaMemcpyDeviceToDevice, s) != cudaSuccess)
            return GAM_ECUDA;
        TRY(fp32 ? launch_bxyz_adj<float>(b, geo, dnxt[2], w.p[tM], s)
                 : launch_bxyz_adj<double>(b, geo, dnxt[2], w.p[tM], s));
        gMf = w.p[tM];
    }
    // adjoint of EnforceBCs: the gas and the three flux directions in one launch
    BcAdjDev tab;
    TRY(bc_adj_device_tables(b, &tab));
    const dim3 tgrid(blocks(b.n, 256), 4);
    if (fp32)
        k_bc_gather_adj_tab<float><<<tgrid, 256, 0, s>>>(b, tab, (const float*)dnxt[0], (float*)w.p[dnG],
                                                        (const float*)gMf, (float*)w.p[dnM]);
    else
        k_bc_gather_adj_tab<double><<<tgrid, 256, 0, s>>>(b, tab, (const double*)dnxt[0], (double*)w.p[dnG],
                                                         (const double*)gMf, (double*)w.p[dnM]);
    if (cudaGetLastError() != cudaSuccess) return GAM_ECUDA;
    const SideStreams* side = side_streams();
    cudaStream_t s1 = side ? side->s[0] : s;
    if (iside) {
        // the I-side fills (in place on dnG, dnM; the field they read gets
        // its adjoint in aBm), then bFlux2Fld of the update's fluxes
        if (cudaMemsetAsync(w.p[aBm], 0, 3 * b.n * es, s) != cudaSuccess) return GAM_ECUDA;
        const void* g2[2] = {geo[1], geo[8]};
        TRY(gam_iside_adjoint(p, fp32, g2, is, w.p[UG], w.p[UB], w.p[dnG], w.p[dnM], w.p[aBm], dinflow, s));
        TRY(fp32 ? launch_bxyz_adj<float>(b, geo, w.p[aBm], w.p[dnM], s)
                 : launch_bxyz_adj<double>(b, geo, w.p[aBm], w.p[dnM], s));
    }
    // applyUpdate, CalcStress, CalcElecField, the limiter field, Predictor
    const void* in5[5] = {st[0], st[1], w.p[E], w.p[gF], w.p[mF]};
    const void* g4[4] = {geo[0], geo[2], geo[3], geo[4]};
    const void* dup[2] = {w.p[dnG], w.p[dnM]};
    void* dsu[5] = {dst[0], dst[1], w.p[dE], w.p[dgF], w.p[dmF]};
    TRY(gam_update_adjoint_store(p, fp32, in5, g4, bg ? bg[3] : nullptr, dt, dup, w.p[sU], w.p[sM], dsu, s));
    // the flux and E-field adjoints gather their stencil adjoints through
    // their own parts of RS in a fixed order (the same bits on every call);
    // they read and write disjoint arrays, so the E-field adjoint runs on the
    // side stream beside the flux adjoint and the bFlux2Fld adjoint after it
    if (side) TRY(fork(side, 1, s));
    const size_t rsE = (size_t)120 * b.n * es;  // the flux adjoint's 120 components come first
    TRY(gam_efield_adjoint_saved(p, fp32, w.p[Dh], w.p[abh], w.p[bn], w.p[VdV], geo[0], geo[1], geo[5], geo[6],
                                 geo[7], bg ? bg[2] : nullptr, dt, w.p[AVf], w.p[dE], w.p[dDh], w.p[dabh], w.p[dbn],
                                 w.p[dVdV], w.p[dAVf], (char*)w.p[RS] + rsE, w.p[ESV], s1));
    TRY(gam_flux_adjoint_gather(p, fp32, w.p[QW], w.p[Wn], w.p[QB], w.p[Blim], w.p[Bnf], geo[0], geo[1], geo[8],
                                bg ? bg[0] : nullptr, bg ? bg[1] : nullptr, w.p[dgF], w.p[dmF], w.p[dQW], w.p[dWn],
                                w.p[dQB], w.p[dBlim], w.p[dBnf], w.p[RS], w.p[FSV], s));
    TRY(fp32 ? launch_bxyz_adj<float>(b, geo, w.p[dBlim], dst[1], s)
             : launch_bxyz_adj<double>(b, geo, w.p[dBlim], dst[1], s));
    if (side) TRY(join(side, 1, s));
    const void* g5[5] = {geo[0], geo[1], geo[2], geo[3], geo[4]};
    const void* din8[8] = {w.p[dQW], w.p[dWn], w.p[dDh], w.p[dVdV], w.p[dQB], w.p[dabh], w.p[dBnf], w.p[dbn]};
    return gam_predict_stage(p, fp32, st, g5, 0.5 * dt, odt, nullptr, din8, w.p[aB], dst, s);
}
}  // namespace gam_stepadj

extern "C" int gam_step_fwd_save(const gam_params* p, int32_t fp32, const void* const* geo, const double* const* bg,
                                 const void* const* st, double dt, double odt, void* const* nxt, void* work,
                                 void* stream) {
    if (p && has_iside(p)) return GAM_EINVAL;  // the I-side boundaries need gam_step_fwd_save_iside
    return step_fwd_save(p, fp32, geo, bg, nullptr, st, dt, odt, nxt, work, stream);
}
extern "C" int gam_step_adj(const gam_params* p, int32_t fp32, const void* const* geo, const double* const* bg,
                            const void* const* st, double dt, double odt, int32_t saved, const void* const* dnxt,
                            void* const* dst, void* work, void* stream) {
    if (p && has_iside(p)) return GAM_EINVAL;
    return step_adj(p, fp32, geo, bg, nullptr, st, dt, odt, saved, dnxt, dst, nullptr, work, stream);
}
extern "C" int gam_step_fwd_save_iside(const gam_params* p, int32_t fp32, const void* const* geo,
                                       const double* const* bg, const gam_iside* is, const void* const* st, double dt,
                                       double odt, void* const* nxt, void* work, void* stream) {
    return step_fwd_save(p, fp32, geo, bg, is, st, dt, odt, nxt, work, stream);
}
extern "C" int gam_step_adj_iside(const gam_params* p, int32_t fp32, const void* const* geo, const double* const* bg,
                                  const gam_iside* is, const void* const* st, double dt, double odt, int32_t saved,
                                  const void* const* dnxt, void* const* dst, void* dinflow, void* work,
                                  void* stream) {
    return step_adj(p, fp32, geo, bg, is, st, dt, odt, saved, dnxt, dst, dinflow, work, stream);
}
