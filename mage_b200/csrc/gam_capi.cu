// C ABI of the GAMERA step (include/gamgpu.h): handle, device memory, layout
// conversion, step sequencing with CUDA graphs, diagnostics.
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>
#include "../../include/gamgpu.h"
#include "gam_layout.cuh"
#include "gam_types.cuh"

// variant launchers (gam_step_strict.cu, gam_step_fast.cu)
void gam_strict_step_f64(const Ctx<double>& C, int cur, cudaStream_t s);
void gam_strict_dt_f64(const Ctx<double>& C, int cur, cudaStream_t s);
void gam_fast_step_f64(const Ctx<double>& C, int cur, cudaStream_t s);
void gam_fast_dt_f64(const Ctx<double>& C, int cur, cudaStream_t s);
void gam_fast_step_f32(const Ctx<float>& C, int cur, cudaStream_t s);
void gam_fast_dt_f32(const Ctx<float>& C, int cur, cudaStream_t s);
void gam_strict_prepare_f64();
void gam_strict_profile_f64(const Ctx<double>& C, int cur, cudaStream_t s, int reps, double* ms);
void gam_fast_profile_f64(const Ctx<double>& C, int cur, cudaStream_t s, int reps, double* ms);
void gam_fast_profile_f32(const Ctx<float>& C, int cur, cudaStream_t s, int reps, double* ms);
void gam_fast_prepare_f64();
void gam_fast_phase_f64(const Ctx<double>& C, int cur, cudaStream_t s, int phase);
void gam_fast_phase_f32(const Ctx<float>& C, int cur, cudaStream_t s, int phase);
void gam_strict_phase_f64(const Ctx<double>& C, int cur, cudaStream_t s, int phase);
void gam_fast_halo_f64(const Ctx<double>& C, int cur, cudaStream_t s, int dside, int unpack, int copyB, void* buf);
void gam_fast_halo_f32(const Ctx<float>& C, int cur, cudaStream_t s, int dside, int unpack, int copyB, void* buf);
void gam_strict_halo_f64(const Ctx<double>& C, int cur, cudaStream_t s, int dside, int unpack, int copyB, void* buf);
void gam_fast_prepare_f32();
// set-up (gam_geom.cu)
void gam_geom_fortran_to_box_d(const GamBox& b, const double* src, double* dst, bool face, int nc, cudaStream_t s);
void gam_geom_fortran_to_box_f(const GamBox& b, const double* src, float* dst, bool face, int nc, cudaStream_t s);
void gam_geom_box_to_fortran_d(const GamBox& b, const double* src, double* dst, bool face, int nc, cudaStream_t s);
void gam_geom_box_to_fortran_f(const GamBox& b, const float* src, double* dst, bool face, int nc, cudaStream_t s);
void gam_geom_fill(double* p, long n, double v, cudaStream_t s);
void gam_geom_d2f(const double* src, float* dst, long n, cudaStream_t s);
void gam_geom_dxf(const GamBox& b, const double* xfc, const double* xyzcc, float* dxf, cudaStream_t s);
void gam_geom_metric(const GamBox& b, const double* xyz, double* face, double* xfc, double* Tf, double* vol,
                     double* xyzcc, double* dijk, double* dl, double* edge, double* Te, double* Teb,
                     const GamRingGeo& ring, cudaStream_t s);
void gam_geom_ic_ot(const GamBox& b, const double* xyzcc, const double* face, double* Gas, double* mf, double gamma,
                    cudaStream_t s);
void gam_geom_ic_case(const GamBox& b, const double* xyz, const double* xyzcc, const double* vol, double* Gas,
                      double* mf, double* lA, double gamma, int which, double a, double bb, cudaStream_t s);
void gam_geom_ic_bw(const GamBox& b, const double* xyz, const double* vol, double* Gas, double* mf, double* lA,
                    double gamma, const double* bw, bool doMHD, cudaStream_t s);
void gam_geom_ic_wind(const GamBox& b, const double* xyz, double* Gas, double* mf, double* lA, double gamma,
                      double dFloor, double pFloor, const double* wind, uint64_t seed, double amp, cudaStream_t s);
void gam_geom_b0_dipole(const GamBox& b, const double* xyz, const double* face, const double* vol, const double* Te,
                        double M0, double* fcB0, double* bFlux0, double* edgB0, double* B0, double* dpB0, double* fS,
                        cudaStream_t s);
// diagnostics (gam_diag.cu)
void gam_diag_divb(const GamBox& b, const double* mf, const double* bFlux0, double* partial, double* out,
                   cudaStream_t s);
void gam_diag_divb_f(const GamBox& b, const float* mf, const double* bFlux0, double* partial, double* out,
                     cudaStream_t s);
void gam_diag_totals(const GamBox& b, const double* Gas, const double* vol, double* partial, double* out,
                     cudaStream_t s);
void gam_diag_totals_f(const GamBox& b, const float* Gas, const float* vol, double* partial, double* out,
                       cudaStream_t s);
void gam_diag_min3(const GamBox& b, const double* dijk, double* dl, cudaStream_t s);
int gam_diag_partials(const GamBox& b);

// FP64 metric, always held (the FP32 form rounds it once)
struct GeoD {
    double *vol, *xyzcc, *dl, *dijk, *face, *xfc, *Tf, *edge, *Te, *Teb, *xyz;
};

// background field (FP64 in both forms), present when doBackground
struct BgD {
    double *fcB0, *bFlux0, *edgB0, *B0, *dpB0;
};

struct gam_handle {
    gam_params p;
    GamBox b;
    BgD bg{};
    double* windTab = nullptr;  // device: wC, wF(3), sF(3) of the solar-wind BC
    double* ionTab = nullptr;   // device: the ionospheric boundary's tables (gam_set_ionosphere)
    GamRingGeo ringGeo{};       // ring averaging about the LFM axis (gam_set_rings)
    bool haveRings = false;
    long ionCap = 0;
    double* ionWind = nullptr;  // device: the wind side of its hooks (WindEFix, NudgeSW weights)
    double ionDtSW0 = 0.0;
    bool haveBg = false, haveWind = false, haveInflow = false, haveIon = false;
    cudaStream_t s = nullptr;
    cudaStream_t own_s = nullptr;  // the handle's own stream (s unless gam_set_stream gave another)
    int nasync = 0;                // device-resident tile steps since the last gam_step_status
    // per side (I lo, I hi, J lo, J hi, K lo, K hi): the side is an edge of
    // the whole grid (gam_set_tile_edges), where CalcDT takes the ghost layer
    int tileEdge[6] = {1, 1, 1, 1, 1, 1};
    bool dtActive = false;         // CalcDT over the active cells only (the magnetosphere's bounds)
    bool f32 = false;
    std::vector<void*> allocs;
    GeoD gd{};
    // bulk views in the compute precision
    Ctx<double> cd{};
    Ctx<float> cf{};
    GamScalars* sc = nullptr;   // device
    double* staging = nullptr;  // device, Fortran-layout transfer buffer
    double* partial = nullptr;  // device, reduction partials
    double* dres = nullptr;     // device, reduction results
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    cudaGraphExec_t pgraph[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};  // [parity][phase] (tile steps)
    int cur = 0;
    bool haveGeo = false, haveState = false, haveXyz = false;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaStream_t aux[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    cudaEvent_t evs[8] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    double lastMs = 0.0;
    std::string err;
};

static int fail(gam_handle* h, int code, const std::string& msg) {
    if (h) h->err = msg;
    return code;
}
static void drop_graphs(gam_handle* h);
static bool is_tile(const gam_handle* h) {
    for (int n = 0; n < 6; n++)
        if (h->p.bc[n] == GAM_BC_HALO) return true;
    return false;
}
static int ion_wind_tables(gam_handle* h);
#define CK(h, call)                                                                            \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                 \
            return fail(h, GAM_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_));    \
    } while (0)

template <class T> static T* dalloc(gam_handle* h, long n, cudaError_t* e) {
    void* p = nullptr;
    *e = cudaMalloc(&p, sizeof(T) * (size_t)n);
    if (*e == cudaSuccess) {
        h->allocs.push_back(p);
#ifdef GAM_BOUNDS_CHECK
        cudaMemsetAsync(p, 0xFF, sizeof(T) * (size_t)n, h->s);  // NaN canaries
#else
        cudaMemsetAsync(p, 0, sizeof(T) * (size_t)n, h->s);
#endif
    }
    return (T*)p;
}

extern "C" int gam_default_params(gam_params* p, int32_t Nip, int32_t Njp, int32_t Nkp) {
    if (!p) return GAM_EINVAL;
    memset(p, 0, sizeof(*p));
    p->Nip = Nip; p->Njp = Njp; p->Nkp = Nkp; p->nG = 4;
    p->gamma = 5.0 / 3.0;
    p->pdmb = 0.75;
    p->CFL = 0.5 / (p->pdmb + 0.5) < 0.3 ? 0.5 / (p->pdmb + 0.5) : 0.3;
    p->Vd0 = 0.5; p->cHogH = 0.25; p->cHogM = 0.25;
    p->dFloor = 1.0e-12; p->pFloor = 1.0e-12;
    p->tFin = 1.0; p->dt0 = 0.0; p->limDT0 = 1.0e-3; p->fixedTimestep = -1.0;
    p->rmeth = GAM_RECON_8CENT; p->doLFMLim = 1; p->doMHD = 1; p->doBackground = 0; p->do25D = (Nkp == 1);
    p->precision = GAM_FP64; p->strict = 0;
    for (int n = 0; n < 6; n++) p->bc[n] = GAM_BC_PERIODIC;
    p->doBoris = 0;
    p->Ca = 1.0e12;  // HUGE (kdefs.F90:20), the reference's Ca without Boris
    p->doAB3 = 0;
    return GAM_OK;
}

template <class R> static void fill_dev_params(DevParams<R>& P, const gam_params& p) {
    P.gamma = (R)p.gamma;
    P.gm1 = (R)(p.gamma - 1);
    P.CFL = (R)p.CFL;
    P.pdmb = (R)p.pdmb;
    P.Vd0 = (R)p.Vd0;
    P.cHogH = (R)p.cHogH;
    P.cHogM = (R)p.cHogM;
    P.doBoris = p.doBoris;
    P.Ca = p.Ca;
    P.doAB3 = p.doAB3;
    P.dFloor = (R)p.dFloor;
    P.pFloor = (R)p.pFloor;
    P.doMHD = p.doMHD; P.doLFMLim = p.doLFMLim; P.do25D = p.do25D; P.doBackground = p.doBackground;
    P.up7 = p.rmeth == GAM_RECON_7UP;
    for (int n = 0; n < 6; n++) P.bc[n] = p.bc[n];
    P.dtKlo = P.dtKhi = 1;
    P.dtIlo = P.dtIhi = P.dtJlo = P.dtJhi = 1;
}

template <class R> static int alloc_bulk(gam_handle* h, Ctx<R>& C) {
    cudaError_t e = cudaSuccess;
    const long fs = h->b.fs;
#define A(ptr, n)                                                   \
    do {                                                            \
        ptr = dalloc<R>(h, (n) * fs, &e);                           \
        if (e != cudaSuccess) return fail(h, GAM_ECUDA, "cudaMalloc failed (out of device memory?)"); \
    } while (0)
    for (int q = 0; q < 2; q++) {
        A(C.st[q].Gas, 5);
        A(C.st[q].mf, 3);
        A(C.st[q].B, 3);
    }
    A(C.w.QW, 5); A(C.w.QB, 3); A(C.w.Dh, 1); A(C.w.Wn, 5); A(C.w.Bl, 3); A(C.w.VdV, 3);
    A(C.w.abh, 3); A(C.w.bn, 3); A(C.w.Bnf, 3); A(C.w.AVf, 9); A(C.w.E, 3);
    A(C.w.gF, 15); A(C.w.mF, 9);
    // CalcElecField starts from E = 0 (fields.F90:88) and E2Flux
    // (fields.F90:37-46) reads edges next to the computed ones, which stay
    // zero; the edge kernels never write them, so E is zeroed once here, also
    // in the bounds-check build whose other arrays start as NaN canaries
    CK(h, cudaMemsetAsync(C.w.E, 0, 3 * fs * sizeof(R), h->s));
    // a 2.5-D grid computes no K fluxes, and Flux2Deltas (stress.F90:150-190)
    // still adds their difference: zero, as the solver's arrays start
    CK(h, cudaMemsetAsync(C.w.gF, 0, 15 * fs * sizeof(R), h->s));
    CK(h, cudaMemsetAsync(C.w.mF, 0, 9 * fs * sizeof(R), h->s));
    C.oomf = nullptr;
    if (h->p.doAB3) A(C.oomf, 3);
    if (sizeof(R) == sizeof(double)) {
        C.g.vol = (const R*)h->gd.vol; C.g.xyzcc = (const R*)h->gd.xyzcc; C.g.dl = (const R*)h->gd.dl;
        C.g.face = (const R*)h->gd.face; C.g.xfc = (const R*)h->gd.xfc; C.g.Tf = (const R*)h->gd.Tf;
        C.g.edge = (const R*)h->gd.edge; C.g.Te = (const R*)h->gd.Te; C.g.Teb = (const R*)h->gd.Teb;
        C.g.dxf = nullptr;
    } else {
        R *vol, *xyzcc, *dl, *face, *xfc, *Tf, *edge, *Te, *Teb, *dxf;
        A(vol, 1); A(xyzcc, 3); A(dl, 1); A(face, 3); A(xfc, 9); A(Tf, 27); A(edge, 3); A(Te, 27); A(Teb, 12);
        A(dxf, 18);
        C.g.vol = vol; C.g.xyzcc = xyzcc; C.g.dl = dl; C.g.face = face; C.g.xfc = xfc; C.g.Tf = Tf;
        C.g.edge = edge; C.g.Te = Te; C.g.Teb = Teb; C.g.dxf = dxf;
    }
#undef A
    C.g.fcB0 = h->bg.fcB0;
    C.g.bFlux0 = h->bg.bFlux0;
    C.g.edgB0 = h->bg.edgB0;
    C.g.B0 = h->bg.B0;
    C.g.dpB0 = h->bg.dpB0;
    C.b = h->b;
    fill_dev_params(C.P, h->p);
    C.sc = h->sc;
    C.gamma = h->p.gamma;
    C.gm1 = h->p.gamma - 1;
    const char* kv = getenv("GAM_KVAR");  // launch-configuration experiments
    C.kvar = kv ? atoi(kv) : 0;
    return GAM_OK;
}

extern "C" int gam_create(const gam_params* p, gam_handle** out) {
    if (!p || !out) return GAM_EINVAL;
    *out = nullptr;
    gam_handle* h = new gam_handle();
    h->p = *p;
    auto bad = [&](int code, const char* m) {
        h->err = m;
        *out = h;
        return code;
    };
    if (p->nG != 4) return bad(GAM_EINVAL, "nG must be 4");
    if (p->Nip < 16 || p->Nip % 8 != 0) return bad(GAM_EBADDIM, "Grid I-size must be >= 16 and divisible by 8");
    if (p->Njp < 1 || p->Nkp < 1) return bad(GAM_EBADDIM, "Njp and Nkp must be >= 1");
    if (p->do25D && p->Nkp != 1) return bad(GAM_EBADDIM, "do25D needs Nkp == 1");
    if (!p->do25D && (p->Njp < 4 || p->Nkp < 4)) return bad(GAM_EBADDIM, "3-D grids need Njp, Nkp >= 4");
    // the ghost fill is one gather whose sources are active cells: a periodic
    // direction needs as many active layers as ghost layers
    if (p->Njp < 4) return bad(GAM_EBADDIM, "Njp must be >= 4 (4 ghost layers are filled from active layers)");
    if (p->precision != GAM_FP64 && p->precision != GAM_FP32) return bad(GAM_EINVAL, "unknown precision");
    if (p->precision == GAM_FP32 && p->strict) return bad(GAM_EINVAL, "strict applies to the FP64 form only");
    {
        // boundary kinds per side: inner I periodic/none/SphIn/inflow/ionosphere, outer I
        // periodic/none/wind/zero-gradient, J periodic/none/zero-gradient,
        // K periodic/none; any side of a tile may be a halo instead
        const int* c = p->bc;
        auto in = [](int v, int a, int b2, int c2) { return v == a || v == b2 || v == c2 || v == GAM_BC_HALO; };
        if (!(in(c[0], GAM_BC_PERIODIC, GAM_BC_NONE, GAM_BC_SPHIN) || c[0] == GAM_BC_INFLOW || c[0] == GAM_BC_ION) ||
            !(in(c[1], GAM_BC_PERIODIC, GAM_BC_NONE, GAM_BC_WIND) || c[1] == GAM_BC_ZEROGRAD) ||
            !(in(c[2], GAM_BC_PERIODIC, GAM_BC_NONE, GAM_BC_ZEROGRAD) || c[2] == GAM_BC_LFM) ||
            !(in(c[3], GAM_BC_PERIODIC, GAM_BC_NONE, GAM_BC_ZEROGRAD) || c[3] == GAM_BC_LFM) ||
            !in(c[4], GAM_BC_PERIODIC, GAM_BC_NONE, GAM_BC_NONE) || !in(c[5], GAM_BC_PERIODIC, GAM_BC_NONE, GAM_BC_NONE))
            return bad(GAM_EINVAL, "unsupported boundary kind for this side");
        for (int d = 0; d < 3; d++)
            if ((c[2 * d] == GAM_BC_PERIODIC) != (c[2 * d + 1] == GAM_BC_PERIODIC))
                return bad(GAM_EINVAL, "a periodic direction needs both sides periodic");
        if (c[0] == GAM_BC_ION && c[4] != GAM_BC_PERIODIC)
            return bad(GAM_EINVAL, "the ionospheric boundary wraps k: the k boundaries must be periodic");
        if (c[0] == GAM_BC_PERIODIC && (c[2] == GAM_BC_ZEROGRAD || c[3] == GAM_BC_ZEROGRAD))
            return bad(GAM_EINVAL, "zero-gradient J with periodic I is not supported");
        if (c[2] == GAM_BC_LFM || c[3] == GAM_BC_LFM) {
            const bool ok2 = c[2] == GAM_BC_LFM || c[2] == GAM_BC_HALO, ok3 = c[3] == GAM_BC_LFM || c[3] == GAM_BC_HALO;
            if (!ok2 || !ok3) return bad(GAM_EINVAL, "an LFM pole's other J side is the other pole or a tile's halo");
            if (c[4] != GAM_BC_PERIODIC || p->do25D)
                return bad(GAM_EINVAL, "the LFM pole wraps k: the k boundaries must be periodic (3-D)");
            if (p->Nkp < 8 || p->Nkp % 2) return bad(GAM_EBADDIM, "the LFM pole needs an even Nkp >= 8");
        }
    }
    if (p->do25D && (p->bc[4] != GAM_BC_PERIODIC || p->bc[5] != GAM_BC_PERIODIC))
        return bad(GAM_EINVAL, "do25D replicates k: the k boundaries must be periodic");
    if (p->doBackground && !p->doMHD) return bad(GAM_EINVAL, "a background field needs doMHD");
    if (p->doBoris && !(p->Ca > 0.0)) return bad(GAM_EINVAL, "doBoris needs Ca > 0");
    h->b = gam_make_box(p->Nip, p->Njp, p->Nkp);
    h->f32 = p->precision == GAM_FP32;
    if (cudaStreamCreateWithFlags(&h->s, cudaStreamNonBlocking) != cudaSuccess) return bad(GAM_ECUDA, "no CUDA device");
    h->own_s = h->s;
    cudaEventCreate(&h->ev0);
    cudaEventCreate(&h->ev1);
    cudaError_t e = cudaSuccess;
    const long fs = h->b.fs;
    GeoD& g = h->gd;
#define AD(ptr, n)                                                     \
    do {                                                               \
        ptr = dalloc<double>(h, (n) * fs, &e);                         \
        if (e != cudaSuccess) return bad(GAM_ECUDA, "cudaMalloc failed (out of device memory?)"); \
    } while (0)
    AD(g.vol, 1); AD(g.xyzcc, 3); AD(g.dl, 1); AD(g.dijk, 3); AD(g.face, 3); AD(g.xfc, 9); AD(g.Tf, 27);
    AD(g.edge, 3); AD(g.Te, 27); AD(g.Teb, 12); AD(g.xyz, 3);
    if (p->doBackground) {
        AD(h->bg.fcB0, 9); AD(h->bg.bFlux0, 3); AD(h->bg.edgB0, 6); AD(h->bg.B0, 3); AD(h->bg.dpB0, 3);
    }
#undef AD
    if (p->bc[1] == GAM_BC_WIND) {
        h->windTab = dalloc<double>(h, 7L * 4 * (h->b.Nj + 1) * (h->b.Nk + 1), &e);
        if (e != cudaSuccess) return bad(GAM_ECUDA, "cudaMalloc failed (wind tables)");
    }
    // staging: the largest Fortran array passed through (Tf/Te: 27 face-sized comps)
    long nface = (long)(h->b.Ni + 1) * (h->b.Nj + 1) * (h->b.Nk + 1);
    h->staging = dalloc<double>(h, 27 * nface, &e);
    if (e != cudaSuccess) return bad(GAM_ECUDA, "cudaMalloc failed (staging)");
    h->partial = dalloc<double>(h, 8 * (long)gam_diag_partials(h->b), &e);
    h->dres = dalloc<double>(h, 16, &e);
    h->sc = dalloc<GamScalars>(h, 1, &e);
    if (e != cudaSuccess) return bad(GAM_ECUDA, "cudaMalloc failed");
    if (h->f32)
        gam_fast_prepare_f32();
    else if (p->strict)
        gam_strict_prepare_f64();
    else
        gam_fast_prepare_f64();
    int rc = h->f32 ? alloc_bulk<float>(h, h->cf) : alloc_bulk<double>(h, h->cd);
    if (rc != GAM_OK) {
        *out = h;
        return rc;
    }
    // side streams and events for the parallel branches of the step graph
    for (int q = 0; q < 5; q++)
        if (cudaStreamCreateWithFlags(&h->aux[q], cudaStreamNonBlocking) != cudaSuccess)
            return bad(GAM_ECUDA, "stream creation failed");
    for (int q = 0; q < 8; q++)
        if (cudaEventCreateWithFlags(&h->evs[q], cudaEventDisableTiming) != cudaSuccess)
            return bad(GAM_ECUDA, "event creation failed");
    for (int q = 0; q < 5; q++) h->cd.aux[q] = h->cf.aux[q] = h->aux[q];
    for (int q = 0; q < 8; q++) h->cd.ev[q] = h->cf.ev[q] = h->evs[q];
    GamScalars s0;
    memset(&s0, 0, sizeof(s0));
    s0.tFin = p->tFin; s0.dt0 = p->dt0; s0.limDT0 = p->limDT0; s0.CFL = p->CFL;
    s0.fixedTimestep = p->fixedTimestep > 0;
    s0.dt = p->fixedTimestep > 0 ? p->fixedTimestep : 0.0;
    double hugedt = 1.0e12;
    memcpy(&s0.dtmin_bits, &hugedt, 8);
#ifdef GAM_BOUNDS_CHECK
    // test hook: a smaller index limit than the box makes the checks fire on
    // in-bounds indices, so the reporting path can be exercised safely
    if (const char* lim = getenv("GAM_BOUNDS_LIMIT")) s0.oobLimit = atoll(lim);
#endif
    if (cudaMemcpyAsync(h->sc, &s0, sizeof(s0), cudaMemcpyHostToDevice, h->s) != cudaSuccess ||
        cudaStreamSynchronize(h->s) != cudaSuccess)
        return bad(GAM_ECUDA, "initialisation copy failed");
    *out = h;
    return GAM_OK;
}

extern "C" int gam_destroy(gam_handle* h) {
    if (!h) return GAM_EINVAL;
    if (h->s) cudaStreamSynchronize(h->s);
    for (int q = 0; q < 2; q++) {
        if (h->graph[q]) cudaGraphExecDestroy(h->graph[q]);
        for (int ph = 0; ph < 2; ph++)
            if (h->pgraph[q][ph]) cudaGraphExecDestroy(h->pgraph[q][ph]);
    }
    for (void* p : h->allocs) cudaFree(p);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    for (int q = 0; q < 8; q++)
        if (h->evs[q]) cudaEventDestroy(h->evs[q]);
    for (int q = 0; q < 5; q++)
        if (h->aux[q]) cudaStreamDestroy(h->aux[q]);
    if (h->own_s) cudaStreamDestroy(h->own_s);  // a stream given by gam_set_stream stays the caller's
    delete h;
    return GAM_OK;
}

extern "C" const char* gam_last_error(gam_handle* h) { return h ? h->err.c_str() : "null handle"; }

static long n_face(const GamBox& b) { return (long)(b.Ni + 1) * (b.Nj + 1) * (b.Nk + 1); }
static long n_cell(const GamBox& b) { return (long)b.Ni * b.Nj * b.Nk; }

// host Fortran array -> FP64 box array
static int up_d(gam_handle* h, const double* src, double* dst, bool face, int nc) {
    long n = (face ? n_face(h->b) : n_cell(h->b)) * nc;
    CK(h, cudaMemcpyAsync(h->staging, src, sizeof(double) * n, cudaMemcpyHostToDevice, h->s));
    gam_geom_fortran_to_box_d(h->b, h->staging, dst, face, nc, h->s);
    return GAM_OK;
}
template <class R> static int up_r(gam_handle* h, const double* src, R* dst, bool face, int nc) {
    long n = (face ? n_face(h->b) : n_cell(h->b)) * nc;
    CK(h, cudaMemcpyAsync(h->staging, src, sizeof(double) * n, cudaMemcpyHostToDevice, h->s));
    if (sizeof(R) == sizeof(double))
        gam_geom_fortran_to_box_d(h->b, h->staging, (double*)dst, face, nc, h->s);
    else
        gam_geom_fortran_to_box_f(h->b, h->staging, (float*)dst, face, nc, h->s);
    return GAM_OK;
}
template <class R> static int down_r(gam_handle* h, const R* src, double* dst, bool face, int nc) {
    long n = (face ? n_face(h->b) : n_cell(h->b)) * nc;
    if (sizeof(R) == sizeof(double))
        gam_geom_box_to_fortran_d(h->b, (const double*)src, h->staging, face, nc, h->s);
    else
        gam_geom_box_to_fortran_f(h->b, (const float*)src, h->staging, face, nc, h->s);
    CK(h, cudaMemcpyAsync(dst, h->staging, sizeof(double) * n, cudaMemcpyDeviceToHost, h->s));
    CK(h, cudaStreamSynchronize(h->s));
    return GAM_OK;
}

// FP32 form: round the FP64 metric once into the FP32 copies
static void sync_geo_f32(gam_handle* h) {
    if (!h->f32) return;
    Geo<float>& g = h->cf.g;
    const long fs = h->b.fs;
    gam_geom_d2f(h->gd.vol, (float*)g.vol, fs, h->s);
    gam_geom_d2f(h->gd.xyzcc, (float*)g.xyzcc, 3 * fs, h->s);
    gam_geom_d2f(h->gd.dl, (float*)g.dl, fs, h->s);
    gam_geom_d2f(h->gd.face, (float*)g.face, 3 * fs, h->s);
    gam_geom_d2f(h->gd.xfc, (float*)g.xfc, 9 * fs, h->s);
    gam_geom_d2f(h->gd.Tf, (float*)g.Tf, 27 * fs, h->s);
    gam_geom_d2f(h->gd.edge, (float*)g.edge, 3 * fs, h->s);
    gam_geom_d2f(h->gd.Te, (float*)g.Te, 27 * fs, h->s);
    gam_geom_d2f(h->gd.Teb, (float*)g.Teb, 12 * fs, h->s);
    gam_geom_dxf(h->b, h->gd.xfc, h->gd.xyzcc, (float*)g.dxf, h->s);
}

static bool has_lfm(const gam_handle* h) { return h->p.bc[2] == GAM_BC_LFM || h->p.bc[3] == GAM_BC_LFM; }

// ------------------------------------------------------------ rings (LFM axis)
// InitRings's defaults for gid "lfm" (ringutils.F90:126-190)
extern "C" int gam_ring_defaults(int32_t Np, int32_t aggressive, int32_t* NumR, int32_t* Nch) {
    if (!NumR || !Nch) return GAM_EINVAL;
    static const int d8[] = {4}, d16[] = {8}, d32[] = {8, 16}, d64[] = {8, 16, 32, 32},
                     d64a[] = {8, 16, 32, 32, 32, 32, 32, 32}, d128[] = {8, 16, 32, 32, 64, 64, 64, 64},
                     d128a[] = {8, 16, 32, 32, 64, 64, 64, 64, 64, 64, 64, 64},
                     d256[] = {8, 16, 32, 32, 64, 64, 64, 64, 128, 128, 128, 128},
                     d256a[] = {8, 16, 32, 32, 64, 64, 64, 64, 128, 128, 128, 128, 128, 128, 128, 128},
                     d512[] = {8, 16, 32, 32, 64, 64, 64, 64, 128, 128, 128, 128, 256, 256, 256, 256},
                     d512a[] = {8, 16, 32, 32, 64, 64, 64, 64, 128, 128, 128, 128, 128, 128, 256, 256, 256, 256,
                                256, 256, 256, 256};
    const int* t = nullptr;
    int n = 0;
#define GAM_RING_CASE(np, a, b2)                                   \
    case np:                                                       \
        if (aggressive) { t = a; n = sizeof(a) / sizeof(int); }     \
        else { t = b2; n = sizeof(b2) / sizeof(int); }               \
        break;
    switch (Np) {
        GAM_RING_CASE(8, d8, d8)
        GAM_RING_CASE(16, d16, d16)
        GAM_RING_CASE(32, d32, d32)
        GAM_RING_CASE(64, d64a, d64)
        GAM_RING_CASE(128, d128a, d128)
        GAM_RING_CASE(256, d256a, d256)
        GAM_RING_CASE(512, d512a, d512)
        default: return GAM_EINVAL;
    }
#undef GAM_RING_CASE
    *NumR = n;
    for (int q = 0; q < 32; q++) Nch[q] = q < n ? t[q] : 0;
    return GAM_OK;
}

extern "C" int gam_set_rings(gam_handle* h, int32_t NumR, const int32_t* Nch, int32_t recon, int32_t NFTmag,
                             int32_t doClean, int32_t doFastClean) {
    if (!h || !Nch) return GAM_EINVAL;
    if (!has_lfm(h)) return fail(h, GAM_ESTATE, "no J side is the LFM pole (GAM_BC_LFM)");
    if (h->haveGeo) return fail(h, GAM_ESTATE, "the rings enter the metric: set them before the geometry");
    const GamBox& b = h->b;
    const int Np = b.Nkp;
    const bool doS = h->p.bc[2] == GAM_BC_LFM, doE = h->p.bc[3] == GAM_BC_LFM;
    if (NumR < 1 || NumR > 32 || NumR >= b.Njp) return fail(h, GAM_EINVAL, "1 <= NumR <= 32 and NumR < Njp");
    if (doS && doE && b.Njp <= 2 * NumR + 2) return fail(h, GAM_EINVAL, "the rings of the two poles meet: Njp > 2 NumR + 2");
    if (recon < 0 || recon > 2) return fail(h, GAM_EINVAL, "ring reconstruction: 0 PPM, 1 PLM, 2 PCM");
    if (NFTmag < -1 || NFTmag > 2) return fail(h, GAM_EINVAL, "NFTmag in -1..2 (NFTMAX = 2)");
    int ncMax = 0;
    for (int q = 0; q < NumR; q++) {
        if (Nch[q] < 1 || Np % Nch[q]) return fail(h, GAM_EINVAL, "every ring's chunk count must divide Nkp");
        ncMax = std::max(ncMax, (int)Nch[q]);
    }
    GamRingGeo& rg = h->ringGeo;
    rg = GamRingGeo{};
    rg.on = 1;
    rg.doS = doS;
    rg.doE = doE;
    rg.NumR = NumR;
    rg.Np = Np;
    for (int q = 0; q < NumR; q++) rg.Nch[q] = Nch[q];
    // cos / sin of m phi_n at the ring cell centres (CleanRing, ringav.F90:
    // 446-453), host libm like the CPU code: phi = dp n - dp/2, dp = 2 pi / Np
    const double PI = 3.141592653589793;
    std::vector<double> ft(6L * Np);
    const double dp = 2.0 * PI / Np;
    for (int m = 0; m <= 2; m++)
        for (int n = 1; n <= Np; n++) {
            const double phi = dp * n - 0.5 * dp;
            ft[(2 * m) * Np + n - 1] = std::cos(1.0 * m * phi);
            ft[(2 * m + 1) * Np + n - 1] = std::sin(1.0 * m * phi);
        }
    cudaError_t e = cudaSuccess;
    double* dft = dalloc<double>(h, 6L * Np, &e);
    if (e != cudaSuccess) return fail(h, GAM_ECUDA, "device allocation failed (ring tables)");
    CK(h, cudaMemcpyAsync(dft, ft.data(), ft.size() * sizeof(double), cudaMemcpyHostToDevice, h->s));
    const long stride = 5L * (ncMax + 4);  // the chunk values of one ring's 5 variables (shared memory)
    void* sE = h->f32 ? (void*)dalloc<float>(h, 3 * b.fs, &e) : (void*)dalloc<double>(h, 3 * b.fs, &e);
    if (e != cudaSuccess) return fail(h, GAM_ECUDA, "device allocation failed (ring work arrays)");
    RingData R{};
    R.on = 1;
    R.doS = doS;
    R.doE = doE;
    R.NumR = NumR;
    R.Np = Np;
    R.recon = recon;
    R.nft = NFTmag;
    R.clean = doClean ? 1 : 0;
    R.tScl = doFastClean ? 1.0 : (double)(1.0f / (float)Np);  // 1.0/Np in default real
    R.aScl = (double)(2.0f / (float)Np);                          // 2.0/Np in default real
    for (int q = 0; q < NumR; q++) R.Nch[q] = Nch[q];
    R.chunkStride = (int)stride;
    R.ftab = dft;
    R.smoothE = sE;
    h->cd.P.ring = R;
    h->cf.P.ring = R;
    CK(h, cudaStreamSynchronize(h->s));
    drop_graphs(h);
    h->haveRings = true;
    return GAM_OK;
}

extern "C" int gam_set_geometry(gam_handle* h, const double* xyz) {
    if (!h || !xyz) return GAM_EINVAL;
    if (has_lfm(h) && !h->haveRings) return fail(h, GAM_ESTATE, "an LFM pole: call gam_set_rings before the geometry");
    int rc = up_d(h, xyz, h->gd.xyz, true, 3);
    if (rc) return rc;
    GeoD& g = h->gd;
    gam_geom_metric(h->b, g.xyz, g.face, g.xfc, g.Tf, g.vol, g.xyzcc, g.dijk, g.dl, g.edge, g.Te, g.Teb, h->ringGeo,
                    h->s);
    sync_geo_f32(h);
    CK(h, cudaGetLastError());
    CK(h, cudaStreamSynchronize(h->s));
    h->haveGeo = true;
    h->haveXyz = true;
    return GAM_OK;
}

extern "C" int gam_set_geometry_arrays(gam_handle* h, const double* face, const double* xfc, const double* Tf,
                                       const double* volume, const double* xyzcc, const double* di, const double* dj,
                                       const double* dk, const double* edge, const double* Te, const double* Teb) {
    if (!h || !face || !xfc || !Tf || !volume || !xyzcc || !di || !dj || !dk || !edge || !Te || !Teb) return GAM_EINVAL;
    if (has_lfm(h) && !h->haveRings) return fail(h, GAM_ESTATE, "an LFM pole: call gam_set_rings before the geometry");
    GeoD& g = h->gd;
    const long fs = h->b.fs;
    int rc;
    if ((rc = up_d(h, face, g.face, true, 3))) return rc;
    if ((rc = up_d(h, xfc, g.xfc, true, 9))) return rc;
    if ((rc = up_d(h, Tf, g.Tf, true, 27))) return rc;
    if ((rc = up_d(h, volume, g.vol, false, 1))) return rc;
    if ((rc = up_d(h, xyzcc, g.xyzcc, false, 3))) return rc;
    if ((rc = up_d(h, di, g.dijk, false, 1))) return rc;
    if ((rc = up_d(h, dj, g.dijk + fs, false, 1))) return rc;
    if ((rc = up_d(h, dk, g.dijk + 2 * fs, false, 1))) return rc;
    if ((rc = up_d(h, edge, g.edge, true, 3))) return rc;
    if ((rc = up_d(h, Te, g.Te, true, 27))) return rc;
    if ((rc = up_d(h, Teb, g.Teb, true, 12))) return rc;
    gam_diag_min3(h->b, g.dijk, g.dl, h->s);
    sync_geo_f32(h);
    CK(h, cudaGetLastError());
    CK(h, cudaStreamSynchronize(h->s));
    h->haveGeo = true;
    return GAM_OK;
}

extern "C" int gam_get_geometry_arrays(gam_handle* h, double* face, double* xfc, double* Tf, double* volume,
                                       double* xyzcc, double* di, double* dj, double* dk, double* edge, double* Te,
                                       double* Teb) {
    if (!h) return GAM_EINVAL;
    if (!h->haveGeo) return fail(h, GAM_ESTATE, "no geometry set");
    GeoD& g = h->gd;
    const long fs = h->b.fs;
    int rc = GAM_OK;
    if (face && (rc = down_r<double>(h, g.face, face, true, 3))) return rc;
    if (xfc && (rc = down_r<double>(h, g.xfc, xfc, true, 9))) return rc;
    if (Tf && (rc = down_r<double>(h, g.Tf, Tf, true, 27))) return rc;
    if (volume && (rc = down_r<double>(h, g.vol, volume, false, 1))) return rc;
    if (xyzcc && (rc = down_r<double>(h, g.xyzcc, xyzcc, false, 3))) return rc;
    if (di && (rc = down_r<double>(h, g.dijk, di, false, 1))) return rc;
    if (dj && (rc = down_r<double>(h, g.dijk + fs, dj, false, 1))) return rc;
    if (dk && (rc = down_r<double>(h, g.dijk + 2 * fs, dk, false, 1))) return rc;
    if (edge && (rc = down_r<double>(h, g.edge, edge, true, 3))) return rc;
    if (Te && (rc = down_r<double>(h, g.Te, Te, true, 27))) return rc;
    if (Teb && (rc = down_r<double>(h, g.Teb, Teb, true, 12))) return rc;
    return GAM_OK;
}

void gam_fast_bfield_f64(const Ctx<double>& C, int cur, cudaStream_t s);
void gam_fast_bfield_f32(const Ctx<float>& C, int cur, cudaStream_t s);
void gam_strict_bfield_f64(const Ctx<double>& C, int cur, cudaStream_t s);
// State%Bxyz from State%magFlux on the device (a NULL Bxyz upload): the
// bFlux2Fld every step and the initialisation end with (gamapp.F90:88,
// init.F90:205), with this handle's kernels
static int state_bfield(gam_handle* h) {
    if (h->f32)
        gam_fast_bfield_f32(h->cf, h->cur, h->s);
    else if (h->p.strict)
        gam_strict_bfield_f64(h->cd, h->cur, h->s);
    else
        gam_fast_bfield_f64(h->cd, h->cur, h->s);
    CK(h, cudaGetLastError());
    return GAM_OK;
}

template <class R>
static int upload_state_t(gam_handle* h, Ctx<R>& C, const double* Gas, const double* magFlux, const double* Bxyz,
                          const double* oGas, const double* omagFlux) {
    int rc;
    h->cur = 0;
    if ((rc = up_r<R>(h, Gas, C.st[0].Gas, false, 5))) return rc;
    if ((rc = up_r<R>(h, magFlux, C.st[0].mf, true, 3))) return rc;
    if (Bxyz && (rc = up_r<R>(h, Bxyz, C.st[0].B, false, 3))) return rc;
    if (!Bxyz && (rc = state_bfield(h))) return rc;
    if ((rc = up_r<R>(h, oGas, C.st[1].Gas, false, 5))) return rc;
    if ((rc = up_r<R>(h, omagFlux, C.st[1].mf, true, 3))) return rc;
    if (C.oomf) CK(h, cudaMemcpyAsync(C.oomf, C.st[1].mf, 3 * h->b.fs * sizeof(R), cudaMemcpyDeviceToDevice, h->s));
    return GAM_OK;
}

// ooState time: otime - dt (init.F90:238-241 and the restart fallback,
// gioH5.F90:800) unless keepOO (oState and ooState stay on the device)
static int set_scalars(gam_handle* h, double time, double otime, double dt, int32_t ts, bool keepOO = false) {
    GamScalars s;
    CK(h, cudaMemcpyAsync(&s, h->sc, sizeof(s), cudaMemcpyDeviceToHost, h->s));
    CK(h, cudaStreamSynchronize(h->s));
    s.time = time; s.otime = otime; s.t = time; s.dt = dt; s.ts = ts;
    if (!keepOO) s.ootime = otime - dt;
    s.status = 0; s.halted = 0; s.nbad = 0;
    double hugedt = 1.0e12;
    memcpy(&s.dtmin_bits, &hugedt, 8);
    CK(h, cudaMemcpyAsync(h->sc, &s, sizeof(s), cudaMemcpyHostToDevice, h->s));
    CK(h, cudaStreamSynchronize(h->s));
    return GAM_OK;
}

// oState kept on the device (oGas = omagFlux = NULL): only State is replaced;
// after a step the other buffer holds the State before that step, which is
// the driver's oState (CopyState, mhdgroup.F90:202-256)
template <class R>
static int upload_new_state_t(gam_handle* h, Ctx<R>& C, const double* Gas, const double* magFlux, const double* Bxyz) {
    int rc;
    if ((rc = up_r<R>(h, Gas, C.st[h->cur].Gas, false, 5))) return rc;
    if ((rc = up_r<R>(h, magFlux, C.st[h->cur].mf, true, 3))) return rc;
    if (Bxyz && (rc = up_r<R>(h, Bxyz, C.st[h->cur].B, false, 3))) return rc;
    if (!Bxyz && (rc = state_bfield(h))) return rc;
    return GAM_OK;
}

extern "C" int gam_upload_state(gam_handle* h, const double* Gas, const double* magFlux, const double* Bxyz,
                                const double* oGas, const double* omagFlux, double time, double otime, double dt,
                                int32_t ts) {
    if (!h || !Gas || !magFlux || (!oGas) != (!omagFlux)) return GAM_EINVAL;
    if (!Bxyz && !h->haveGeo) return fail(h, GAM_ESTATE, "Bxyz = NULL is computed from the fluxes: set the geometry first");
    int rc;
    if (!oGas) {
        if (!h->haveState) return fail(h, GAM_ESTATE, "oState can stay on the device only after a first full upload");
        rc = h->f32 ? upload_new_state_t<float>(h, h->cf, Gas, magFlux, Bxyz)
                    : upload_new_state_t<double>(h, h->cd, Gas, magFlux, Bxyz);
    } else {
        rc = h->f32 ? upload_state_t<float>(h, h->cf, Gas, magFlux, Bxyz, oGas, omagFlux)
                    : upload_state_t<double>(h, h->cd, Gas, magFlux, Bxyz, oGas, omagFlux);
    }
    if (rc) return rc;
    if ((rc = set_scalars(h, time, otime, dt, ts, !oGas))) return rc;
    CK(h, cudaStreamSynchronize(h->s));
    h->haveState = true;
    return GAM_OK;
}

template <class R> static int set_oo_t(gam_handle* h, Ctx<R>& C, const double* oomagFlux) {
    return up_r<R>(h, oomagFlux, C.oomf, true, 3);
}
extern "C" int gam_set_oostate(gam_handle* h, const double* oomagFlux, double ootime) {
    if (!h || !oomagFlux) return GAM_EINVAL;
    if (!h->p.doAB3) return fail(h, GAM_ESTATE, "ooState is kept only with doAB3");
    if (!h->haveState) return fail(h, GAM_ESTATE, "upload State and oState first");
    int rc = h->f32 ? set_oo_t<float>(h, h->cf, oomagFlux) : set_oo_t<double>(h, h->cd, oomagFlux);
    if (rc) return rc;
    CK(h, cudaMemcpyAsync(&h->sc->ootime, &ootime, sizeof(double), cudaMemcpyHostToDevice, h->s));
    CK(h, cudaStreamSynchronize(h->s));
    return GAM_OK;
}
extern "C" int gam_get_oostate(gam_handle* h, double* oomagFlux, double* ootime) {
    if (!h) return GAM_EINVAL;
    if (!h->p.doAB3) return fail(h, GAM_ESTATE, "ooState is kept only with doAB3");
    if (!h->haveState) return fail(h, GAM_ESTATE, "no state");
    int rc = GAM_OK;
    if (oomagFlux) rc = h->f32 ? down_r<float>(h, h->cf.oomf, oomagFlux, true, 3)
                               : down_r<double>(h, h->cd.oomf, oomagFlux, true, 3);
    if (rc) return rc;
    if (ootime) {
        CK(h, cudaMemcpyAsync(ootime, &h->sc->ootime, sizeof(double), cudaMemcpyDeviceToHost, h->s));
        CK(h, cudaStreamSynchronize(h->s));
    }
    return GAM_OK;
}

template <class R>
static int download_state_t(gam_handle* h, Ctx<R>& C, double* Gas, double* magFlux, double* Bxyz, double* oGas,
                            double* omagFlux) {
    int rc;
    const StateBuf<R>& S = C.st[h->cur];
    const StateBuf<R>& O = C.st[1 - h->cur];
    if (Gas && (rc = down_r<R>(h, S.Gas, Gas, false, 5))) return rc;
    if (magFlux && (rc = down_r<R>(h, S.mf, magFlux, true, 3))) return rc;
    if (Bxyz && (rc = down_r<R>(h, S.B, Bxyz, false, 3))) return rc;
    if (oGas && (rc = down_r<R>(h, O.Gas, oGas, false, 5))) return rc;
    if (omagFlux && (rc = down_r<R>(h, O.mf, omagFlux, true, 3))) return rc;
    return GAM_OK;
}

extern "C" int gam_download_state(gam_handle* h, double* Gas, double* magFlux, double* Bxyz, double* oGas,
                                  double* omagFlux, double* time, double* otime, double* dt, int32_t* ts) {
    if (!h) return GAM_EINVAL;
    if (!h->haveState) return fail(h, GAM_ESTATE, "no state uploaded");
    int rc = h->f32 ? download_state_t<float>(h, h->cf, Gas, magFlux, Bxyz, oGas, omagFlux)
                    : download_state_t<double>(h, h->cd, Gas, magFlux, Bxyz, oGas, omagFlux);
    if (rc) return rc;
    GamScalars s;
    CK(h, cudaMemcpy(&s, h->sc, sizeof(s), cudaMemcpyDeviceToHost));
    if (time) *time = s.time;
    if (otime) *otime = s.otime;
    if (dt) *dt = s.dt;
    if (ts) *ts = s.ts;
    return GAM_OK;
}

static void launch_one(gam_handle* h, int cur) {
    if (h->f32)
        gam_fast_step_f32(h->cf, cur, h->s);
    else if (h->p.strict)
        gam_strict_step_f64(h->cd, cur, h->s);
    else
        gam_fast_step_f64(h->cd, cur, h->s);
}

static int ensure_graph(gam_handle* h, int cur) {
    if (h->graph[cur]) return GAM_OK;
    cudaGraph_t g;
    CK(h, cudaStreamBeginCapture(h->s, cudaStreamCaptureModeThreadLocal));
    launch_one(h, cur);
    CK(h, cudaStreamEndCapture(h->s, &g));
    CK(h, cudaGraphInstantiate(&h->graph[cur], g, 0));
    cudaGraphDestroy(g);
    return GAM_OK;
}

// After a synchronised call: GAM_EBOUNDS if a kernel's index check failed
// (bounds-check build; the record stays until the handle is destroyed)
static int check_bounds(gam_handle* h, const GamScalars& s) {
#ifdef GAM_BOUNDS_CHECK
    if (s.oob) {
        char msg[160];
        snprintf(msg, sizeof(msg), "bounds check failed in kernel %d at box index %lld", s.oobKernel, s.oobIndex);
        return fail(h, GAM_EBOUNDS, msg);
    }
#else
    (void)h;
    (void)s;
#endif
    return GAM_OK;
}

extern "C" int gam_bounds_status(gam_handle* h, int32_t* fired, int32_t* kernel, int64_t* index) {
    if (!h || !fired) return GAM_EINVAL;
#ifdef GAM_BOUNDS_CHECK
    GamScalars s;
    CK(h, cudaMemcpyAsync(&s, h->sc, sizeof(s), cudaMemcpyDeviceToHost, h->s));
    CK(h, cudaStreamSynchronize(h->s));
    *fired = s.oob ? 1 : 0;
    if (kernel) *kernel = s.oob ? s.oobKernel : 0;
    if (index) *index = s.oob ? s.oobIndex : 0;
#else
    *fired = -1;
    if (kernel) *kernel = 0;
    if (index) *index = 0;
#endif
    return GAM_OK;
}

// what a step needs besides the kernels
static int step_ready(gam_handle* h) {
    if (!h->haveGeo) return fail(h, GAM_ESTATE, "gam_step before gam_set_geometry");
    if (!h->haveState) return fail(h, GAM_ESTATE, "gam_step before gam_upload_state");
    if (h->p.doBackground && !h->haveBg) return fail(h, GAM_ESTATE, "doBackground: set the background field first");
    if (h->p.bc[1] == GAM_BC_WIND && !h->haveWind) return fail(h, GAM_ESTATE, "wind boundary: call gam_set_wind first");
    if (h->p.bc[0] == GAM_BC_INFLOW && !h->haveInflow)
        return fail(h, GAM_ESTATE, "inflow boundary: call gam_set_inflow first");
    if ((h->p.bc[0] == GAM_BC_ION && !h->haveIon) || (h->haveIon && h->p.bc[1] == GAM_BC_WIND && !h->cd.P.ion.wind))
        return fail(h, GAM_ESTATE, "ionospheric boundary: call gam_set_ionosphere (and gam_set_wind) first");
    return GAM_OK;
}

extern "C" int gam_step(gam_handle* h, int32_t nsteps, double* dt, double* t) {
    if (!h || nsteps < 0) return GAM_EINVAL;
    if (int rc0 = step_ready(h)) return rc0;
    if (is_tile(h))
        return fail(h, GAM_ESTATE, "a tile steps with gam_step_begin / gam_step_end and a halo exchange");
    int rc;
    if ((rc = ensure_graph(h, 0))) return rc;
    if ((rc = ensure_graph(h, 1))) return rc;
    GamScalars s;
    CK(h, cudaMemcpyAsync(&s, h->sc, sizeof(s), cudaMemcpyDeviceToHost, h->s));
    CK(h, cudaStreamSynchronize(h->s));
    if (s.halted)
        return fail(h, s.status == 5 ? GAM_EDT_DISASTER : GAM_EDT_BAD, "a previous step failed CalcDT; upload a state");
    const int ts0 = s.ts, cur0 = h->cur;
    // host-side range with the reference's priority clock label (gamapp.F90:96-99)
    nvtxRangePushA("Gamera");
    CK(h, cudaEventRecord(h->ev0, h->s));
    for (int n = 0; n < nsteps; n++) CK(h, cudaGraphLaunch(h->graph[(cur0 + n) & 1], h->s));
    CK(h, cudaEventRecord(h->ev1, h->s));
    nvtxRangePop();
    CK(h, cudaMemcpyAsync(&s, h->sc, sizeof(s), cudaMemcpyDeviceToHost, h->s));
    CK(h, cudaStreamSynchronize(h->s));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, h->ev0, h->ev1);
    h->lastMs = ms;
    // every executed step (the failing one included) swapped the buffers once;
    // steps after a failure returned at once
    h->cur = (cur0 + (s.ts - ts0)) & 1;
    if (dt) *dt = s.dt;
    if (t) *t = s.t;
    if (int rcb = check_bounds(h, s)) return rcb;
    if (s.halted)
        return fail(h, s.status == 5 ? GAM_EDT_DISASTER : GAM_EDT_BAD,
                    s.status == 5 ? "CalcDT: timestep too small or not finite" : "CalcDT: timestep dropped 10x or below limDT0");
    return GAM_OK;
}

extern "C" int gam_advance_model(gam_handle* h, double dt, double* t_out) {
    if (!h) return GAM_EINVAL;
    GamScalars s;
    CK(h, cudaMemcpy(&s, h->sc, sizeof(s), cudaMemcpyDeviceToHost));
    const double target = s.t + dt;
    double ddt, t;
    int rc = gam_step(h, 1, &ddt, &t);
    while (rc == GAM_OK && t < target) rc = gam_step(h, 1, &ddt, &t);
    if (t_out) *t_out = t;
    return rc;
}

// The update and boundary kernels write the other state buffer, which holds
// oState: it is copied aside and put back, like the scalars, so the state is
// left as it was. The AB2 spacing the step kernels read is set the way
// k_step_begin sets it (mhdgroup.F90:25-31), also before the first step.
template <class R> static int profile_t(gam_handle* h, Ctx<R>& C, int32_t reps, double* ms, GamScalars s) {
    const long fs = h->b.fs;
    const StateBuf<R>& O = C.st[1 - h->cur];
    R* save = nullptr;
    CK(h, cudaMalloc(&save, 14 * fs * sizeof(R)));
    auto cp = [&](R* d, const R* src, long n) { return cudaMemcpyAsync(d, src, n * sizeof(R), cudaMemcpyDeviceToDevice, h->s); };
    cudaError_t e = cp(save, O.Gas, 5 * fs);
    if (e == cudaSuccess) e = cp(save + 5 * fs, O.mf, 3 * fs);
    if (e == cudaSuccess) e = cp(save + 8 * fs, O.B, 3 * fs);
    if (e == cudaSuccess && C.oomf) e = cp(save + 11 * fs, C.oomf, 3 * fs);
    GamScalars t = s;
    if (fabs(t.otime - t.time) < 1.0e-12) t.otime = t.time - t.dt;
    t.odt = t.time - t.otime;
    t.oodt = t.otime - t.ootime;
    t.pdt = 0.5 * t.dt;
    if (e == cudaSuccess) e = cudaMemcpyAsync(h->sc, &t, sizeof(t), cudaMemcpyHostToDevice, h->s);
    if (e == cudaSuccess) {
        if (h->f32)
            gam_fast_profile_f32(h->cf, h->cur, h->s, reps, ms);
        else if (h->p.strict)
            gam_strict_profile_f64(h->cd, h->cur, h->s, reps, ms);
        else
            gam_fast_profile_f64(h->cd, h->cur, h->s, reps, ms);
        e = cudaGetLastError();
    }
    cudaError_t e2 = cp(O.Gas, save, 5 * fs);
    if (e2 == cudaSuccess) e2 = cp(O.mf, save + 5 * fs, 3 * fs);
    if (e2 == cudaSuccess) e2 = cp(O.B, save + 8 * fs, 3 * fs);
    if (e2 == cudaSuccess && C.oomf) e2 = cp(C.oomf, save + 11 * fs, 3 * fs);
    // restore the scalars the repeated kernels touched (dt reduction, AB2 spacing)
    if (e2 == cudaSuccess) e2 = cudaMemcpyAsync(h->sc, &s, sizeof(s), cudaMemcpyHostToDevice, h->s);
    if (e2 == cudaSuccess) e2 = cudaStreamSynchronize(h->s);
    cudaFree(save);
    CK(h, e);
    CK(h, e2);
    return GAM_OK;
}

extern "C" int gam_profile_step(gam_handle* h, int32_t reps, double* ms, int32_t n) {
    if (!h || !ms || n < 15 || reps < 1) return GAM_EINVAL;
    if (!h->haveGeo || !h->haveState) return fail(h, GAM_ESTATE, "gam_profile_step needs geometry and state");
    if (h->p.doBackground && !h->haveBg) return fail(h, GAM_ESTATE, "doBackground: set the background field first");
    if (h->p.bc[1] == GAM_BC_WIND && !h->haveWind) return fail(h, GAM_ESTATE, "wind boundary: call gam_set_wind first");
    GamScalars s;
    CK(h, cudaMemcpyAsync(&s, h->sc, sizeof(s), cudaMemcpyDeviceToHost, h->s));
    CK(h, cudaStreamSynchronize(h->s));
    return h->f32 ? profile_t<float>(h, h->cf, reps, ms, s) : profile_t<double>(h, h->cd, reps, ms, s);
}

extern "C" int gam_last_step_ms(gam_handle* h, double* ms) {
    if (!h || !ms) return GAM_EINVAL;
    *ms = h->lastMs;
    return GAM_OK;
}

extern "C" int gam_calc_dt(gam_handle* h, double* dt) {
    if (!h || !dt) return GAM_EINVAL;
    if (!h->haveGeo || !h->haveState) return fail(h, GAM_ESTATE, "gam_calc_dt needs geometry and state");
    GamScalars s;
    CK(h, cudaMemcpyAsync(&s, h->sc, sizeof(s), cudaMemcpyDeviceToHost, h->s));
    CK(h, cudaStreamSynchronize(h->s));
    if (s.fixedTimestep) {
        *dt = s.dt;
        return GAM_OK;
    }
    double hugedt = 1.0e12;
    unsigned long long hb;
    memcpy(&hb, &hugedt, 8);
    CK(h, cudaMemcpyAsync(&h->sc->dtmin_bits, &hb, 8, cudaMemcpyHostToDevice, h->s));
    if (h->f32)
        gam_fast_dt_f32(h->cf, h->cur, h->s);
    else if (h->p.strict)
        gam_strict_dt_f64(h->cd, h->cur, h->s);
    else
        gam_fast_dt_f64(h->cd, h->cur, h->s);
    unsigned long long bits;
    CK(h, cudaMemcpyAsync(&bits, &h->sc->dtmin_bits, 8, cudaMemcpyDeviceToHost, h->s));
    CK(h, cudaMemcpyAsync(&h->sc->dtmin_bits, &hb, 8, cudaMemcpyHostToDevice, h->s));
    CK(h, cudaStreamSynchronize(h->s));
    double dtMin;
    memcpy(&dtMin, &bits, 8);
    CK(h, cudaMemcpyAsync(&s, h->sc, sizeof(s), cudaMemcpyDeviceToHost, h->s));
    CK(h, cudaStreamSynchronize(h->s));
    if (int rcb = check_bounds(h, s)) return rcb;
    // step.F90:158-166 clamps (the ts > 0 failure checks belong to a step)
    double d = dtMin;
    if (s.t + d > s.tFin) d = (s.tFin - s.t) > 1.0e-12 ? (s.tFin - s.t) : 1.0e-12;
    if (s.dt0 > 1.0e-12 && d > 10.0 * s.dt0) d = 10.0 * s.dt0;
    *dt = d;
    if (dtMin == hugedt) return fail(h, GAM_EDT_DISASTER, "no timestep was smaller than HUGE");
    return GAM_OK;
}

extern "C" int gam_divb(gam_handle* h, double* total) {
    if (!h || !total) return GAM_EINVAL;
    if (!h->haveState) return fail(h, GAM_ESTATE, "no state");
    // DivB's total includes the background fluxes (doTot, gridutils.F90:749-753)
    const double* b0 = (h->p.doBackground && h->haveBg) ? h->bg.bFlux0 : nullptr;
    if (h->f32)
        gam_diag_divb_f(h->b, h->cf.st[h->cur].mf, b0, h->partial, h->dres, h->s);
    else
        gam_diag_divb(h->b, h->cd.st[h->cur].mf, b0, h->partial, h->dres, h->s);
    CK(h, cudaMemcpyAsync(total, h->dres, 8, cudaMemcpyDeviceToHost, h->s));
    CK(h, cudaStreamSynchronize(h->s));
    return GAM_OK;
}

extern "C" int gam_totals(gam_handle* h, double out[5]) {
    if (!h || !out) return GAM_EINVAL;
    if (!h->haveState || !h->haveGeo) return fail(h, GAM_ESTATE, "no state");
    if (h->f32)
        gam_diag_totals_f(h->b, h->cf.st[h->cur].Gas, h->cf.g.vol, h->partial, h->dres, h->s);
    else
        gam_diag_totals(h->b, h->cd.st[h->cur].Gas, h->gd.vol, h->partial, h->dres, h->s);
    CK(h, cudaMemcpyAsync(out, h->dres, 5 * 8, cudaMemcpyDeviceToHost, h->s));
    CK(h, cudaStreamSynchronize(h->s));
    return GAM_OK;
}

// ------------------------------------------------------------ problem set-up
// Initial conditions computed on the GPU from the metric already set
// (prob.F90 initOT2D / initBW), followed by the reference's initialisation
// order (init.F90:190-244): Bxyz from fluxes, oState = State, boundary
// conditions, first CalcDT, oState%time = t - dt.
template <class R> static int finish_init(gam_handle* h, Ctx<R>& C, double* Gas64, double* mf64, double t0) {
    // Gas64/mf64: FP64 box arrays holding the IC
    const long fs = h->b.fs;
    for (int q = 0; q < 2; q++) {
        if (sizeof(R) == sizeof(double)) {
            cudaMemcpyAsync(C.st[q].Gas, Gas64, 5 * fs * sizeof(double), cudaMemcpyDeviceToDevice, h->s);
            cudaMemcpyAsync(C.st[q].mf, mf64, 3 * fs * sizeof(double), cudaMemcpyDeviceToDevice, h->s);
        } else {
            gam_geom_d2f(Gas64, (float*)C.st[q].Gas, 5 * fs, h->s);
            gam_geom_d2f(mf64, (float*)C.st[q].mf, 3 * fs, h->s);
        }
    }
    CK(h, cudaGetLastError());
    h->cur = 0;
    h->haveState = true;
    int rc = set_scalars(h, t0, t0, 0.0, 0);
    if (rc) return rc;
    return GAM_OK;
}

void gam_strict_init_f64(const Ctx<double>& C, int cur, cudaStream_t s);
void gam_fast_init_f64(const Ctx<double>& C, int cur, cudaStream_t s);
void gam_fast_init_f32(const Ctx<float>& C, int cur, cudaStream_t s);

static int init_common(gam_handle* h, double* Gas64, double* mf64) {
    if (h->p.bc[0] == GAM_BC_INFLOW && !h->haveInflow)
        return fail(h, GAM_ESTATE, "inflow boundary: call gam_set_inflow before the initial condition");
    if (h->p.bc[0] == GAM_BC_ION && !h->haveIon)
        return fail(h, GAM_ESTATE, "ionospheric boundary: call gam_set_ionosphere before the initial condition");
    int rc = h->f32 ? finish_init<float>(h, h->cf, Gas64, mf64, 0.0) : finish_init<double>(h, h->cd, Gas64, mf64, 0.0);
    if (rc) return rc;
    // Bxyz of State, first BCs, copy to oState (init.F90:217-238)
    if (h->f32)
        gam_fast_init_f32(h->cf, 0, h->s);
    else if (h->p.strict)
        gam_strict_init_f64(h->cd, 0, h->s);
    else
        gam_fast_init_f64(h->cd, 0, h->s);
    CK(h, cudaGetLastError());
    // a tile's ghosts arrive with the first halo exchange; the caller
    // finishes with gam_init_finish_halo and gam_set_start
    if (is_tile(h)) return GAM_OK;
    double dt;
    rc = gam_calc_dt(h, &dt);
    if (rc) return rc;
    // Model%dt = CalcDT; oState%time = State%time - Model%dt (init.F90:241-246)
    return set_scalars(h, 0.0, -dt, dt, 0);
}

extern "C" int gam_init_orszag_tang(gam_handle* h) {
    if (!h) return GAM_EINVAL;
    if (!h->haveGeo) return fail(h, GAM_ESTATE, "set the geometry first");
    double* Gas64 = h->staging;
    double* mf64 = h->staging + 5 * h->b.fs;
    if (8 * h->b.fs > 27 * n_face(h->b)) return fail(h, GAM_EINVAL, "staging too small");
    gam_geom_fill(Gas64, 8 * h->b.fs, 0.0, h->s);
    gam_geom_ic_ot(h->b, h->gd.xyzcc, h->gd.face, Gas64, mf64, h->p.gamma, h->s);
    return init_common(h, Gas64, mf64);
}

extern "C" int gam_init_test_problem(gam_handle* h, int32_t which, double a, double b) {
    if (!h || which < GAM_IC_ADV1D || which > GAM_IC_ALFVEN) return GAM_EINVAL;
    if (!h->haveXyz) return fail(h, GAM_ESTATE, "the problem set-ups integrate over cells and edges: call gam_set_geometry first");
    if (11 * h->b.fs > 27 * n_face(h->b)) return fail(h, GAM_EINVAL, "staging too small");
    double* Gas64 = h->staging;
    double* mf64 = h->staging + 5 * h->b.fs;
    double* lA = h->staging + 8 * h->b.fs;
    gam_geom_fill(Gas64, 8 * h->b.fs, 0.0, h->s);
    gam_geom_ic_case(h->b, h->gd.xyz, h->gd.xyzcc, h->gd.vol, Gas64, mf64, lA, h->p.gamma, which - GAM_IC_ADV1D, a, b,
                     h->s);
    return init_common(h, Gas64, mf64);
}

extern "C" int gam_init_blast_wave(gam_handle* h, const double* bw9) {
    if (!h || !bw9) return GAM_EINVAL;
    if (!h->haveXyz) return fail(h, GAM_ESTATE, "the blast-wave IC integrates over cells: call gam_set_geometry first");
    if (11 * h->b.fs > 27 * n_face(h->b)) return fail(h, GAM_EINVAL, "staging too small");
    double* Gas64 = h->staging;
    double* mf64 = h->staging + 5 * h->b.fs;
    double* lA = h->staging + 8 * h->b.fs;
    gam_geom_fill(Gas64, 8 * h->b.fs, 0.0, h->s);
    gam_geom_ic_bw(h->b, h->gd.xyz, h->gd.vol, Gas64, mf64, lA, h->p.gamma, bw9, h->p.doMHD != 0, h->s);
    return init_common(h, Gas64, mf64);
}

// ------------------------------------------------------------ background field and solar wind
static void drop_graphs(gam_handle* h) {
    for (int q = 0; q < 2; q++) {
        if (h->graph[q]) {
            cudaGraphExecDestroy(h->graph[q]);
            h->graph[q] = nullptr;
        }
        for (int ph = 0; ph < 2; ph++)
            if (h->pgraph[q][ph]) {
                cudaGraphExecDestroy(h->pgraph[q][ph]);
                h->pgraph[q][ph] = nullptr;
            }
    }
}
// CalcDT's range per side: the ghost layer where the side is an edge of the
// whole grid (SetDomain, init.F90:511-530; a tile's inner sides stop at its
// active cells, as hasLowerBC / hasUpperBC are false there), the active cells
// only under the magnetosphere's bounds (earthcmi.F90:136-142)
static void set_dt_range(gam_handle* h) {
    int v[6];
    for (int n = 0; n < 6; n++) v[n] = (h->tileEdge[n] && !h->dtActive) ? 1 : 0;
    h->cd.P.dtIlo = h->cf.P.dtIlo = v[0];
    h->cd.P.dtIhi = h->cf.P.dtIhi = v[1];
    h->cd.P.dtJlo = h->cf.P.dtJlo = v[2];
    h->cd.P.dtJhi = h->cf.P.dtJhi = v[3];
    h->cd.P.dtKlo = h->cf.P.dtKlo = v[4];
    h->cd.P.dtKhi = h->cf.P.dtKhi = v[5];
    drop_graphs(h);
}

extern "C" int gam_set_background(gam_handle* h, const double* fcB0, const double* bFlux0, const double* edgB0,
                                  const double* B0, const double* dpB0) {
    if (!h || !fcB0 || !bFlux0 || !edgB0 || !B0 || !dpB0) return GAM_EINVAL;
    if (!h->p.doBackground) return fail(h, GAM_ESTATE, "the handle was created without doBackground");
    int rc;
    if ((rc = up_d(h, fcB0, h->bg.fcB0, false, 9))) return rc;
    if ((rc = up_d(h, bFlux0, h->bg.bFlux0, false, 3))) return rc;
    if ((rc = up_d(h, edgB0, h->bg.edgB0, false, 6))) return rc;
    if ((rc = up_d(h, B0, h->bg.B0, false, 3))) return rc;
    if ((rc = up_d(h, dpB0, h->bg.dpB0, false, 3))) return rc;
    CK(h, cudaGetLastError());
    CK(h, cudaStreamSynchronize(h->s));
    h->haveBg = true;
    return GAM_OK;
}

extern "C" int gam_get_background(gam_handle* h, double* fcB0, double* bFlux0, double* edgB0, double* B0,
                                  double* dpB0) {
    if (!h) return GAM_EINVAL;
    if (!h->haveBg) return fail(h, GAM_ESTATE, "no background field set");
    int rc = GAM_OK;
    if (fcB0 && (rc = down_r<double>(h, h->bg.fcB0, fcB0, false, 9))) return rc;
    if (bFlux0 && (rc = down_r<double>(h, h->bg.bFlux0, bFlux0, false, 3))) return rc;
    if (edgB0 && (rc = down_r<double>(h, h->bg.edgB0, edgB0, false, 6))) return rc;
    if (B0 && (rc = down_r<double>(h, h->bg.B0, B0, false, 3))) return rc;
    if (dpB0 && (rc = down_r<double>(h, h->bg.dpB0, dpB0, false, 3))) return rc;
    return GAM_OK;
}

extern "C" int gam_set_background_dipole(gam_handle* h, double M0) {
    if (!h) return GAM_EINVAL;
    if (!h->p.doBackground) return fail(h, GAM_ESTATE, "the handle was created without doBackground");
    if (!h->haveXyz) return fail(h, GAM_ESTATE, "the dipole background integrates over cells: call gam_set_geometry first");
    if (9 * h->b.fs > 27 * n_face(h->b)) return fail(h, GAM_EINVAL, "staging too small");
    const GeoD& g = h->gd;
    gam_geom_b0_dipole(h->b, g.xyz, g.face, g.vol, g.Te, M0, h->bg.fcB0, h->bg.bFlux0, h->bg.edgB0, h->bg.B0,
                       h->bg.dpB0, h->staging, h->s);
    CK(h, cudaGetLastError());
    CK(h, cudaStreamSynchronize(h->s));
    h->haveBg = true;
    return GAM_OK;
}

// math.F90:332-343 normVec
static void norm_vec(const double* a, double* out) {
    double nA = sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
    for (int x = 0; x < 3; x++) out[x] = nA <= 1.0e-12 ? 0.0 : a[x] / nA;
}
// math.F90:97-111 RampDown
static double ramp_down(double r, double rC, double lC) {
    if (r <= rC) return 1.0;
    if (r >= rC + lC) return 0.0;
    double rScl = (r - rC) / lC;
    double eArg = -1.0 / (1.0 - rScl * rScl);
    return exp(eArg + 1.0);
}
// apps/wind.F90:180-203 wgtWind for a constant wind velocity V: 1 where the
// point faces the wind, ramping to 0 over 90 degrees behind it
static double wgt_wind(const double* V, const double* xyz) {
    double nHat[3], vHat[3], mv[3];
    norm_vec(xyz, nHat);
    norm_vec(V, vHat);
    for (int x = 0; x < 3; x++) mv[x] = -vHat[x];
    double dTh = acos(mv[0] * nHat[0] + mv[1] * nHat[1] + mv[2] * nHat[2]) * 180.0 / 3.141592653589793;
    return ramp_down(dTh, 90.0, 90.0);
}

// The wind blend weights and wind face fluxes of the 4 outer-I ghost layers,
// from the FP64 metric (host libm acos/exp, like the CPU code).
extern "C" int gam_set_wind(gam_handle* h, const double wind[8]) {
    if (!h || !wind) return GAM_EINVAL;
    if (h->p.bc[1] != GAM_BC_WIND) return fail(h, GAM_ESTATE, "the outer I boundary is not the solar wind");
    if (!h->haveGeo) return fail(h, GAM_ESTATE, "set the geometry first");
    const GamBox& b = h->b;
    const int G = 4, i0 = G + b.Nip;  // slab i0 .. i0+4 (ghost cells i0..i0+3, faces up to i0+4)
    const long nrow = (long)(b.Nj + 1) * (b.Nk + 1);
    const long nw = 4 * nrow;
    // components: xyzcc 3, xfc 9, Tf normals 9, face 3
    std::vector<double> sl(24 * 5 * nrow);
    auto slab = [&](const double* comp, int q) -> cudaError_t {
        return cudaMemcpy2DAsync(sl.data() + (size_t)q * 5 * nrow, 5 * sizeof(double), comp + i0,
                                 (size_t)b.sx * sizeof(double), 5 * sizeof(double), (size_t)nrow,
                                 cudaMemcpyDeviceToHost, h->s);
    };
    const GeoD& g = h->gd;
    const long fs = b.fs;
    int q = 0;
    for (int x = 0; x < 3; x++) CK(h, slab(g.xyzcc + x * fs, q++));
    for (int x = 0; x < 9; x++) CK(h, slab(g.xfc + x * fs, q++));
    for (int d = 0; d < 3; d++)
        for (int x = 0; x < 3; x++) CK(h, slab(g.Tf + (x + 9 * d) * fs, q++));
    for (int d = 0; d < 3; d++) CK(h, slab(g.face + d * fs, q++));
    CK(h, cudaStreamSynchronize(h->s));
    auto at = [&](int comp, long row, int o) { return sl[(size_t)comp * 5 * nrow + (size_t)row * 5 + o]; };
    const double V[3] = {wind[2], wind[3], wind[4]}, Bsw[3] = {wind[5], wind[6], wind[7]};
    std::vector<double> tab(7 * nw, 0.0);
    double* wC = tab.data();
    double* wF = tab.data() + nw;
    double* sF = tab.data() + 4 * nw;
    for (int kk = 0; kk <= b.Nk; kk++)
        for (int jj = 0; jj <= b.Nj; jj++) {
            const long row = jj + (long)(b.Nj + 1) * kk;
            for (int n = 1; n <= 4; n++) {
                const long wi = (n - 1) + 4 * row;
                const int o = n - 1;  // ghost cell ig = i0 + n - 1
                if (jj < b.Nj && kk < b.Nk) {
                    double xc[3] = {at(0, row, o), at(1, row, o), at(2, row, o)};
                    wC[wi] = wgt_wind(V, xc);
                }
                for (int d = 0; d < 3; d++) {
                    const int oo = d == 0 ? o + 1 : o;  // I face ig+1; J, K faces of cell ig
                    double xf[3] = {at(3 + 3 * d, row, oo), at(4 + 3 * d, row, oo), at(5 + 3 * d, row, oo)};
                    double nH[3] = {at(12 + 3 * d, row, oo), at(13 + 3 * d, row, oo), at(14 + 3 * d, row, oo)};
                    wF[d * nw + wi] = wgt_wind(V, xf);
                    sF[d * nw + wi] = at(21 + d, row, oo) * (nH[0] * Bsw[0] + nH[1] * Bsw[1] + nH[2] * Bsw[2]);
                }
            }
        }
    CK(h, cudaMemcpyAsync(h->windTab, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice, h->s));
    CK(h, cudaStreamSynchronize(h->s));
    WindData W{};  // n = 0: the constant wind (a series set before is dropped)
    for (int v = 0; v < 8; v++) W.state[v] = wind[v];
    W.wC = h->windTab;
    W.wF = h->windTab + nw;
    W.sF = h->windTab + 4 * nw;
    W.nw = nw;
    h->cd.P.wind = W;
    h->cf.P.wind = W;
    drop_graphs(h);
    h->haveWind = true;
    if (h->haveIon) return ion_wind_tables(h);  // the hooks' wind side
    return GAM_OK;
}

extern "C" int gam_set_wind_series(gam_handle* h, int32_t n, const double* t, const double* rho, const double* P,
                                   const double* V, const double* B, const double* xyzBS, double Bx0, double ByC,
                                   double BzC) {
    if (!h || !t || !rho || !P || !V || !B) return GAM_EINVAL;
    if (h->p.bc[1] != GAM_BC_WIND) return fail(h, GAM_ESTATE, "the outer I boundary is not the solar wind");
    if (n < 2) return fail(h, GAM_EINVAL, "a wind series needs at least two rows");
    double dtMin = t[1] - t[0], dtMax = dtMin, vMax = 0.0;
    for (int r = 1; r + 1 < n; r++) {
        dtMin = std::min(dtMin, t[r + 1] - t[r]);
        dtMax = std::max(dtMax, t[r + 1] - t[r]);
    }
    if (!(dtMin > 0.0) || fabs(dtMin - dtMax) > 1.0e-6 * sqrt(dtMin * dtMin + dtMax * dtMax))
        return fail(h, GAM_EINVAL, "the wind series needs increasing, uniformly spaced times");
    std::vector<double> tab(12 * (size_t)n);
    for (int r = 0; r < n; r++) {
        double* q = tab.data() + 12 * (size_t)r;
        q[0] = t[r];
        q[1] = rho[r];
        for (int x = 0; x < 3; x++) q[2 + x] = V[3 * r + x];
        q[5] = P[r];
        for (int x = 0; x < 3; x++) q[6 + x] = B[3 * r + x];
        q[6] = Bx0 + ByC * q[7] + BzC * q[8];  // readWind (apps/wind.F90:723-727)
        for (int x = 0; x < 3; x++) q[9 + x] = xyzBS ? xyzBS[3 * r + x] : 0.0;
        vMax = std::max(vMax, sqrt(q[2] * q[2] + q[3] * q[3] + q[4] * q[4]));
    }
    if (h->p.doBoris && vMax >= h->p.Ca) return fail(h, GAM_EINVAL, "the solar wind is faster than the Boris speed Ca");
    cudaError_t e = cudaSuccess;
    double* d = dalloc<double>(h, 12L * n, &e);
    if (e != cudaSuccess) return fail(h, GAM_ECUDA, "cudaMalloc failed (wind series)");
    CK(h, cudaMemcpyAsync(d, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice, h->s));
    CK(h, cudaStreamSynchronize(h->s));
    for (WindData* W : {&h->cd.P.wind, &h->cf.P.wind}) {
        W->n = n;
        W->tMin = *std::min_element(t, t + n);
        W->tMax = *std::max_element(t, t + n);
        W->dtW = dtMin;
        W->Bx0 = Bx0; W->ByC = ByC; W->BzC = BzC;
        W->ts = d;
    }
    drop_graphs(h);
    h->haveWind = true;
    if (h->p.bc[0] == GAM_BC_ION) {  // the hooks' wind side takes the constant wind only
        h->cd.P.ion.wind = h->cf.P.ion.wind = 0;
        h->haveIon = false;
    }
    return GAM_OK;
}

extern "C" int gam_set_inflow(gam_handle* h, const double state[8]) {
    if (!h || !state) return GAM_EINVAL;
    if (h->p.bc[0] != GAM_BC_INFLOW) return fail(h, GAM_ESTATE, "the inner I boundary is not an inflow");
    if (!(state[0] > 0.0)) return fail(h, GAM_EINVAL, "inflow density must be positive");
    for (int v = 0; v < 8; v++) {
        h->cd.P.inflow[v] = state[v];
        h->cf.P.inflow[v] = state[v];
    }
    drop_graphs(h);
    h->haveInflow = true;
    return GAM_OK;
}


// ---- the ionospheric inner boundary (bc[0] = GAM_BC_ION)
namespace {
// NORM2 as gfortran evaluates it (scaled sum of squares)
double ion_norm2(const double* a) {
    double scale = 1.0, res = 0.0;
    for (int q = 0; q < 3; q++)
        if (a[q] != 0.0) {
            const double ax = std::fabs(a[q]);
            if (scale < ax) {
                const double val = scale / ax;
                res = 1.0 + res * val * val;
                scale = ax;
            } else {
                const double val = ax / scale;
                res += val * val;
            }
        }
    return scale * std::sqrt(res);
}
// VecDipole (msphutils.F90:534-559), m = (0, 0, M0)
void ion_dipole(double M0, const double* r, double* B) {
    const double rad = ion_norm2(r);
    const double m[3] = {0.0, 0.0, M0};
    const double d = m[0] * r[0] + m[1] * r[1] + m[2] * r[2];
    const double p5 = std::pow(rad, 5.0), p3 = std::pow(rad, 3.0);
    for (int x = 0; x < 3; x++) B[x] = 3 * d * r[x] / p5 - m[x] / p3;
}
// E x B / |B|^2 (cross, math.F90:265-274) with its radial part removed
// (Vec2Perp, math.F90:371-376); vr: the radial part
void ion_exb_perp(const double* E, const double* B, const double* rh, double* v, double* vr) {
    const double c[3] = {E[1] * B[2] - E[2] * B[1], E[2] * B[0] - E[0] * B[2], E[0] * B[1] - E[1] * B[0]};
    const double bb = B[0] * B[0] + B[1] * B[1] + B[2] * B[2];
    double veb[3];
    for (int x = 0; x < 3; x++) veb[x] = c[x] / bb;
    const double d = veb[0] * rh[0] + veb[1] * rh[1] + veb[2] * rh[2];
    for (int x = 0; x < 3; x++) v[x] = veb[x] - d * rh[x];
    *vr = d;
}
}  // namespace

static int ion_wind_tables(gam_handle* h) {
    const GamBox& b = h->b;
    const int G = 4, Nj = b.Nj, Nk = b.Nk;
    const long nrow = (long)(Nj + 1) * (Nk + 1), fs = b.fs;
    const GeoD& g = h->gd;
    const long nWe = 7L * 4 * (b.Njp + 1) * (b.Nkp + 1), nWn = (long)b.Njp * b.Nkp;
    std::vector<double> tab(nWe + nWn, 0.0);
    double* We = tab.data();
    double* Wn = We + nWe;
    double vSW = 0.0;
    {
        // WindEFix (apps/wind.F90:489-566) for the constant wind: the front
        // velocity (-|V|, 0, 0) of RefreshWind with ByC = BzC = 0, the wind
        // EMF -V x B along each edge of shells ie-2 .. ie+1, the weights at
        // the edge centres (host libm, as the constant wind's BC weights)
        const double* ws = h->cd.P.wind.state;
        const double V[3] = {ws[2], ws[3], ws[4]}, Bw[3] = {ws[5], ws[6], ws[7]};
        const double vFr[3] = {-ion_norm2(V), 0.0, 0.0};
        const double Ca = h->p.doBoris ? h->p.Ca : 1.0e12;
        vSW = std::min(ion_norm2(vFr), Ca);
        const double c[3] = {V[1] * Bw[2] - V[2] * Bw[1], V[2] * Bw[0] - V[0] * Bw[2], V[0] * Bw[1] - V[1] * Bw[0]};
        const double swE[3] = {-c[0], -c[1], -c[2]};
        const int c0 = G + b.Nip - 3, nc = 5;  // corner columns ie-2 .. ie+2
        std::vector<double> xv(3 * nc * nrow), xcn(3 * nrow);
        for (int x = 0; x < 3; x++) {
            CK(h, cudaMemcpy2DAsync(xv.data() + (size_t)x * nc * nrow, nc * sizeof(double), g.xyz + x * fs + c0,
                                    (size_t)b.sx * sizeof(double), nc * sizeof(double), (size_t)nrow,
                                    cudaMemcpyDeviceToHost, h->s));
            CK(h, cudaMemcpy2DAsync(xcn.data() + (size_t)x * nrow, sizeof(double), g.xyzcc + x * fs + G + b.Nip - 1,
                                    (size_t)b.sx * sizeof(double), sizeof(double), (size_t)nrow,
                                    cudaMemcpyDeviceToHost, h->s));
        }
        CK(h, cudaStreamSynchronize(h->s));
        auto corner = [&](int col, int jj, int kk, double* r) {
            for (int x = 0; x < 3; x++)
                r[x] = xv[(size_t)x * nc * nrow + ((size_t)jj + (size_t)(Nj + 1) * kk) * nc + col];
        };
        const int ie = b.Nip;  // Fortran indices: is = 1, ie = Nip, box column ii = i + 3
        for (int kk = G; kk <= G + b.Nkp; kk++)
            for (int jj = G; jj <= G + b.Njp; jj++)
                for (int sh = 0; sh < 4; sh++) {
                    const int col = sh, i = ie - 2 + sh;
                    double* t = We + 7 * (sh + 4 * ((long)(jj - G) + (long)(b.Njp + 1) * (kk - G)));
                    double wSW = 0.0;
                    for (int n = 0; n < 3; n++) {
                        double e1[3], e2[3], ecc[3], de[3];
                        corner(col, jj, kk, e1);
                        corner(col + (n == 0), jj + (n == 1), kk + (n == 2), e2);
                        for (int x = 0; x < 3; x++) {
                            ecc[x] = 0.5 * (e1[x] + e2[x]);
                            de[x] = e2[x] - e1[x];
                        }
                        wSW = wgt_wind(V, ecc);
                        t[n] = -1.0;  // unchanged
                        t[3 + n] = 0.0;
                        if (wSW > 1.0e-12) {
                            if (i <= ie) wSW = wSW / (1.0 + ie + 1 - i);
                            t[n] = wSW;
                            t[3 + n] = swE[0] * de[0] + swE[1] * de[1] + swE[2] * de[2];
                        }
                    }
                    t[6] = wSW;  // DiffuseOuter's weight: the K edge's
                }
        // NudgeSW's weights of the last active cells
        for (int kk = G; kk < G + b.Nkp; kk++)
            for (int jj = G; jj < G + b.Njp; jj++) {
                const long row = jj + (long)(Nj + 1) * kk;
                const double r[3] = {xcn[row], xcn[nrow + row], xcn[2 * nrow + row]};
                Wn[(jj - G) + (long)b.Njp * (kk - G)] = wgt_wind(V, r);
            }
    }
    if (!h->ionWind) {
        cudaError_t e = cudaSuccess;
        h->ionWind = dalloc<double>(h, nWe + nWn, &e);
        if (e != cudaSuccess) return fail(h, GAM_ECUDA, "device allocation failed");
    }
    CK(h, cudaMemcpyAsync(h->ionWind, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice, h->s));
    CK(h, cudaStreamSynchronize(h->s));
    for (IonData* I : {&h->cd.P.ion, &h->cf.P.ion}) {
        I->wind = 1;
        I->vSW = vSW;
        I->dtSW0 = h->ionDtSW0;
        I->We = h->ionWind;
        I->Wn = h->ionWind + nWe;
    }
    drop_graphs(h);
    return GAM_OK;
}

extern "C" int gam_set_ionosphere(gam_handle* h, const double* inExyz, const double* inEijk, double M0, double dtCpl,
                                  int32_t doIonPush, int32_t nIonP, double dtSW0) {
    if (!h) return GAM_EINVAL;
    // a tile of the magnetosphere away from the inner boundary takes the
    // hooks of its other sides (WindEFix, NudgeSW, FixEFieldLFM) and the DT
    // bounds; the inner tile also the boundary itself (hasLowerBC(IDIR))
    const bool inner = h->p.bc[0] == GAM_BC_ION;
    if (!inner && h->p.bc[0] != GAM_BC_HALO)
        return fail(h, GAM_ESTATE, "the inner I boundary is not the ionosphere (nor a tile's halo)");
    if (h->p.bc[4] != GAM_BC_PERIODIC)
        return fail(h, GAM_EINVAL, "the magnetosphere's hooks need the whole periodic k range on every tile");
    if (inner && (!inExyz || !inEijk)) return GAM_EINVAL;
    if (!h->haveGeo) return fail(h, GAM_ESTATE, "set the geometry first");
    const GamBox& b = h->b;
    if (!doIonPush || !inner) nIonP = 0;
    if (!inner) doIonPush = 0;
    if (doIonPush && (!(dtCpl > 0.0) || nIonP < 1 || nIonP > b.Nip))
        return fail(h, GAM_EINVAL, "PushIon needs dtCpl > 0 and 1 <= nIonP <= Nip");
    const bool windHooks = h->p.bc[1] == GAM_BC_WIND;
    if (windHooks) {
        if (!h->haveXyz) return fail(h, GAM_ESTATE, "WindEFix needs the grid corners: set the geometry with gam_set_geometry");
        if (h->haveWind && h->cd.P.wind.n != 0)
            return fail(h, GAM_ESTATE, "the wind side of the hooks takes the constant wind (gam_set_wind)");
        if (!(dtSW0 > 0.0)) return fail(h, GAM_EINVAL, "NudgeSW needs dtSW0 > 0");
        if (nIonP >= b.Nip) return fail(h, GAM_EINVAL, "PushIon and NudgeSW would act on the same shell");
    }
    if (!inner) {
        IonData I{};
        I.on = 1;
        h->cd.P.ion = I;
        h->cf.P.ion = I;
        h->ionDtSW0 = dtSW0;
        h->dtActive = true;
        set_dt_range(h);
        h->haveIon = true;
        if (windHooks && h->haveWind) return ion_wind_tables(h);
        return GAM_OK;
    }
    const int G = 4, Nj = b.Nj, Nk = b.Nk, ncol = G + nIonP;
    const long nrow = (long)(Nj + 1) * (Nk + 1);
    // box columns 0 .. G+nIonP-1 of xyzcc (3) and column G of the J, K edge lengths
    std::vector<double> xc(3 * ncol * nrow), el(2 * nrow);
    const GeoD& g = h->gd;
    const long fs = b.fs;
    for (int x = 0; x < 3; x++)
        CK(h, cudaMemcpy2DAsync(xc.data() + (size_t)x * ncol * nrow, ncol * sizeof(double), g.xyzcc + x * fs,
                                (size_t)b.sx * sizeof(double), ncol * sizeof(double), (size_t)nrow,
                                cudaMemcpyDeviceToHost, h->s));
    for (int d = 1; d < 3; d++)
        CK(h, cudaMemcpy2DAsync(el.data() + (size_t)(d - 1) * nrow, sizeof(double), g.edge + d * fs + G,
                                (size_t)b.sx * sizeof(double), sizeof(double), (size_t)nrow, cudaMemcpyDeviceToHost,
                                h->s));
    CK(h, cudaStreamSynchronize(h->s));
    auto X = [&](int ii, int jj, int kk, double* r) {
        for (int x = 0; x < 3; x++) r[x] = xc[(size_t)x * ncol * nrow + ((size_t)jj + (size_t)(Nj + 1) * kk) * ncol + ii];
    };
    // inExyz(s, j, k, x): (1:5, jsg:jeg, ksg:keg, 1:3); inEijk (1:6, jsg:jeg+1, ksg:keg+1, 1:3)
    auto Exyz = [&](int sh, int jj, int kk, int x) { return inExyz[sh + 5 * (jj + (long)Nj * (kk + (long)Nk * x))]; };
    auto Eijk = [&](int sh, int jj, int kk, int x) {
        return inEijk[sh + 6 * (jj + (long)(Nj + 1) * (kk + (long)(Nk + 1) * x))];
    };
    const long nVg = 3L * 4 * Nj * Nk, nVp = 3L * nIonP * b.Njp * b.Nkp, nEe = 2L * Nj * Nk;
    std::vector<double> tab(nVg + nVp + nEe, 0.0);
    double* Vg = tab.data();
    double* Vp = Vg + nVg;
    double* Ee = Vp + nVp;
    // ghost cells (IonInner, earthcmi.F90:466-528 with CellPlasmaBC): the
    // E x B velocity of shell 5-n at the ghost cell's centre (k wrapped),
    // perpendicular to the radius plus its inward radial part
    for (int kk = 0; kk < Nk; kk++)
        for (int jj = 0; jj < Nj; jj++) {
            int kp = kk, jp = jj;
            if (kk < G) kp = kk + b.Nkp;
            else if (kk >= G + b.Nkp) kp = kk - b.Nkp;
            // across the LFM pole: the conjugate (mirrored j, k + Nkp/2)
            const GamRingGeo& rg = h->ringGeo;
            if (rg.on && ((rg.doS && jj < G) || (rg.doE && jj > G + b.Njp - 1 && jj <= G + b.Njp + 3))) {
                jp = jj < G ? 2 * G - 1 - jj : 2 * G + 2 * b.Njp - 1 - jj;
                kp = kk + b.Nkp / 2;
                if (kp > G + b.Nkp - 1) kp -= b.Nkp;
            }
            for (int n = 1; n <= 4; n++) {
                double r[3], B[3], rh[3], E[3], v[3], vr;
                X(G - n, jp, kp, r);
                ion_dipole(M0, r, B);
                for (int x = 0; x < 3; x++) E[x] = Exyz(4 - n, jp, kp, x);
                norm_vec(r, rh);
                ion_exb_perp(E, B, rh, v, &vr);
                const double vin = std::min(vr, 0.0);
                double* o = Vg + 3 * ((n - 1) + 4 * ((long)jj + (long)Nj * kk));
                for (int x = 0; x < 3; x++) o[x] = v[x] + vin * rh[x];
            }
        }
    // PushIon's target velocity (earthcmi.F90:618-630): shell 5's E x B in
    // the dipole at the cell centre, perpendicular to the radius
    for (int kk = G; kk < G + b.Nkp; kk++)
        for (int jj = G; jj < G + b.Njp; jj++)
            for (int ii = G; ii < G + nIonP; ii++) {
                double r[3], B[3], rh[3], E[3], vr;
                X(ii, jj, kk, r);
                ion_dipole(M0, r, B);
                for (int x = 0; x < 3; x++) E[x] = Exyz(4, jj, kk, x);
                norm_vec(r, rh);
                ion_exb_perp(E, B, rh, Vp + 3 * ((ii - G) + (long)nIonP * ((jj - G) + (long)b.Njp * (kk - G))), &vr);
            }
    // IonEFix (msphutils.F90:225-238): edge x inEijk(5) on the first shell
    for (int kk = 0; kk < Nk; kk++)
        for (int jj = 0; jj < Nj; jj++) {
            const long row = jj + (long)(Nj + 1) * kk, q = jj + (long)Nj * kk;
            Ee[2 * q] = el[row] * Eijk(4, jj, kk, 1);
            Ee[2 * q + 1] = el[nrow + row] * Eijk(4, jj, kk, 2);
        }
    if ((long)tab.size() > h->ionCap) {
        cudaError_t e = cudaSuccess;
        h->ionTab = dalloc<double>(h, (long)tab.size(), &e);
        if (e != cudaSuccess) return fail(h, GAM_ECUDA, "device allocation failed");
        h->ionCap = (long)tab.size();
    }
    CK(h, cudaMemcpyAsync(h->ionTab, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice, h->s));
    CK(h, cudaStreamSynchronize(h->s));
    IonData I{};
    I.on = 1;
    I.push = doIonPush ? 1 : 0;
    I.nIonP = nIonP;
    I.dtCpl = dtCpl;
    I.Vg = h->ionTab;
    I.Vp = h->ionTab + nVg;
    I.Ee = h->ionTab + nVg + nVp;
    h->cd.P.ion = I;
    h->cf.P.ion = I;
    h->ionDtSW0 = dtSW0;
    h->dtActive = true;
    set_dt_range(h);
    h->haveIon = true;
    // the wind side of the hooks, now or when the constant wind is set
    if (windHooks && h->haveWind) return ion_wind_tables(h);
    return GAM_OK;
}

extern "C" int gam_init_dipole_wind(gam_handle* h, const double wind[8], uint64_t seed, double amp) {
    if (!h || !wind) return GAM_EINVAL;
    if (!h->haveXyz) return fail(h, GAM_ESTATE, "the vector potential is integrated along edges: call gam_set_geometry first");
    if (h->p.doBackground && !h->haveBg) return fail(h, GAM_ESTATE, "set the background field first");
    if (11 * h->b.fs > 27 * n_face(h->b)) return fail(h, GAM_EINVAL, "staging too small");
    int rc;
    if (h->p.bc[1] == GAM_BC_WIND && (rc = gam_set_wind(h, wind))) return rc;
    double* Gas64 = h->staging;
    double* mf64 = h->staging + 5 * h->b.fs;
    double* lA = h->staging + 8 * h->b.fs;
    gam_geom_fill(Gas64, 8 * h->b.fs, 0.0, h->s);
    gam_geom_ic_wind(h->b, h->gd.xyz, Gas64, mf64, lA, h->p.gamma, h->p.dFloor, h->p.pFloor, wind, seed, amp, h->s);
    return init_common(h, Gas64, mf64);
}

// ------------------------------------------------------------ restart files
// A binary stand-in for the restart dump of writeH5Res / readH5Restart
// (src/gamera/gioH5.F90:636-858): State and oState with their ghosts, the
// times, ts, dt and dt0. Layout: a 72-byte header (magic "GAMRST01", Nip, Njp,
// Nkp as int32, one int32 zero, t, State%time, oState%time, dt, dt0 as
// float64, ts as int32, one int32 zero), then Gas, magFlux, Bxyz, oGas,
// omagFlux as float64 Fortran-ordered arrays with ghosts, little endian.
struct GamRestartHeader {
    char magic[8];
    int32_t Nip, Njp, Nkp, zero0;
    double t, time, otime, dt, dt0;
    int32_t ts, zero1;
};
static_assert(sizeof(GamRestartHeader) == 72, "restart header layout");

extern "C" int gam_write_restart(gam_handle* h, const char* path) {
    if (!h || !path) return GAM_EINVAL;
    if (!h->haveState) return fail(h, GAM_ESTATE, "no state to write");
    const long nc = n_cell(h->b), nf = n_face(h->b);
    std::vector<double> Gas(5 * nc), mf(3 * nf), B(3 * nc), oGas(5 * nc), omf(3 * nf);
    GamRestartHeader hd;
    memset(&hd, 0, sizeof(hd));
    memcpy(hd.magic, "GAMRST01", 8);
    hd.Nip = h->p.Nip; hd.Njp = h->p.Njp; hd.Nkp = h->p.Nkp;
    int rc = gam_download_state(h, Gas.data(), mf.data(), B.data(), oGas.data(), omf.data(), &hd.time, &hd.otime,
                                &hd.dt, &hd.ts);
    if (rc) return rc;
    GamScalars s;
    CK(h, cudaMemcpy(&s, h->sc, sizeof(s), cudaMemcpyDeviceToHost));
    hd.t = s.t;
    hd.dt0 = s.dt0;
    FILE* f = fopen(path, "wb");
    if (!f) return fail(h, GAM_EINVAL, std::string("cannot open ") + path + " for writing");
    bool ok = fwrite(&hd, sizeof(hd), 1, f) == 1;
    for (auto* v : {&Gas, &mf, &B, &oGas, &omf}) ok = ok && fwrite(v->data(), sizeof(double), v->size(), f) == v->size();
    ok = (fclose(f) == 0) && ok;
    if (!ok) return fail(h, GAM_EINVAL, std::string("write to ") + path + " failed");
    return GAM_OK;
}

extern "C" int gam_read_restart(gam_handle* h, const char* path) {
    if (!h || !path) return GAM_EINVAL;
    FILE* f = fopen(path, "rb");
    if (!f) return fail(h, GAM_EINVAL, std::string("cannot open ") + path);
    GamRestartHeader hd;
    if (fread(&hd, sizeof(hd), 1, f) != 1 || memcmp(hd.magic, "GAMRST01", 8) != 0) {
        fclose(f);
        return fail(h, GAM_EINVAL, std::string(path) + " is not a restart file of this library");
    }
    if (hd.Nip != h->p.Nip || hd.Njp != h->p.Njp || hd.Nkp != h->p.Nkp) {
        fclose(f);
        return fail(h, GAM_EBADDIM, "restart grid size differs from the handle's");
    }
    const long nc = n_cell(h->b), nf = n_face(h->b);
    std::vector<double> Gas(5 * nc), mf(3 * nf), B(3 * nc), oGas(5 * nc), omf(3 * nf);
    bool ok = true;
    for (auto* v : {&Gas, &mf, &B, &oGas, &omf}) ok = ok && fread(v->data(), sizeof(double), v->size(), f) == v->size();
    fclose(f);
    if (!ok) return fail(h, GAM_EINVAL, std::string(path) + " is truncated");
    int rc = gam_upload_state(h, Gas.data(), mf.data(), B.data(), oGas.data(), omf.data(), hd.time, hd.otime, hd.dt,
                              hd.ts);
    if (rc) return rc;
    GamScalars s;
    CK(h, cudaMemcpy(&s, h->sc, sizeof(s), cudaMemcpyDeviceToHost));
    s.t = hd.t;
    s.dt0 = hd.dt0;
    CK(h, cudaMemcpy(h->sc, &s, sizeof(s), cudaMemcpyHostToDevice));
    return GAM_OK;
}

// ------------------------------------------------------------ tiles (k-slabs and I/J/K tiles)
static void launch_phase(gam_handle* h, int cur, int phase) {
    if (h->f32)
        gam_fast_phase_f32(h->cf, cur, h->s, phase);
    else if (h->p.strict)
        gam_strict_phase_f64(h->cd, cur, h->s, phase);
    else
        gam_fast_phase_f64(h->cd, cur, h->s, phase);
}
static int ensure_phase_graph(gam_handle* h, int cur, int phase) {
    if (h->pgraph[cur][phase]) return GAM_OK;
    cudaGraph_t g;
    CK(h, cudaStreamBeginCapture(h->s, cudaStreamCaptureModeThreadLocal));
    launch_phase(h, cur, phase);
    CK(h, cudaStreamEndCapture(h->s, &g));
    CK(h, cudaGraphInstantiate(&h->pgraph[cur][phase], g, 0));
    cudaGraphDestroy(g);
    return GAM_OK;
}
static int require_slab(gam_handle* h) {
    if (!is_tile(h)) return fail(h, GAM_ESTATE, "the handle is not a tile (no side is GAM_BC_HALO)");
    if (!h->haveGeo || !h->haveState) return fail(h, GAM_ESTATE, "set the geometry and the state first");
    return GAM_OK;
}

extern "C" int gam_tile_halo_bytes(gam_handle* h, int32_t dir, int64_t* bytes) {
    if (!h || !bytes || dir < 0 || dir > 2) return GAM_EINVAL;
    const GamBox& b = h->b;
    // 11 components x 4 layers x the face-box extents across dir
    const long nu = dir == 0 ? b.Nj + 1 : b.Ni + 1, nv = dir == 2 ? b.Nj + 1 : b.Nk + 1;
    *bytes = 11L * 4 * nu * nv * (h->f32 ? 4 : 8);
    return GAM_OK;
}
extern "C" int gam_halo_bytes(gam_handle* h, int64_t* bytes) { return gam_tile_halo_bytes(h, 2, bytes); }

static int halo_call(gam_handle* h, int dir, int side, int unpack, int copyB, void* buf) {
    if (!h || !buf || (side != 0 && side != 1) || dir < 0 || dir > 2) return GAM_EINVAL;
    int rc = require_slab(h);
    if (rc) return rc;
    if (h->p.bc[2 * dir + side] != GAM_BC_HALO) return fail(h, GAM_ESTATE, "this side of the tile is not a halo");
    const int dside = side + 2 * dir;
    if (h->f32)
        gam_fast_halo_f32(h->cf, h->cur, h->s, dside, unpack, copyB, buf);
    else if (h->p.strict)
        gam_strict_halo_f64(h->cd, h->cur, h->s, dside, unpack, copyB, buf);
    else
        gam_fast_halo_f64(h->cd, h->cur, h->s, dside, unpack, copyB, buf);
    CK(h, cudaGetLastError());
    if (h->s == h->own_s) CK(h, cudaStreamSynchronize(h->s));
    return GAM_OK;
}
extern "C" int gam_tile_halo_pack(gam_handle* h, int32_t dir, int32_t side, void* dev_buf) {
    return halo_call(h, dir, side, 0, 0, dev_buf);
}
extern "C" int gam_tile_halo_unpack(gam_handle* h, int32_t dir, int32_t side, const void* dev_buf, int32_t copyB) {
    return halo_call(h, dir, side, 1, copyB ? 1 : 0, const_cast<void*>(dev_buf));
}
extern "C" int gam_halo_pack(gam_handle* h, int32_t side, void* dev_buf) { return halo_call(h, 2, side, 0, 0, dev_buf); }
extern "C" int gam_halo_unpack(gam_handle* h, int32_t side, const void* dev_buf, int32_t copyB) {
    return halo_call(h, 2, side, 1, copyB ? 1 : 0, const_cast<void*>(dev_buf));
}

extern "C" int gam_init_finish_halo(gam_handle* h, double* dt_local) {
    if (!h || !dt_local) return GAM_EINVAL;
    int rc = require_slab(h);
    if (rc) return rc;
    const long fs = h->b.fs;
    const size_t w = h->f32 ? 4 : 8;
    void* S[3] = {h->f32 ? (void*)h->cf.st[h->cur].Gas : (void*)h->cd.st[h->cur].Gas,
                  h->f32 ? (void*)h->cf.st[h->cur].mf : (void*)h->cd.st[h->cur].mf,
                  h->f32 ? (void*)h->cf.st[h->cur].B : (void*)h->cd.st[h->cur].B};
    void* O[3] = {h->f32 ? (void*)h->cf.st[1 - h->cur].Gas : (void*)h->cd.st[1 - h->cur].Gas,
                  h->f32 ? (void*)h->cf.st[1 - h->cur].mf : (void*)h->cd.st[1 - h->cur].mf,
                  h->f32 ? (void*)h->cf.st[1 - h->cur].B : (void*)h->cd.st[1 - h->cur].B};
    const long nc[3] = {5, 3, 3};
    for (int q = 0; q < 3; q++) CK(h, cudaMemcpyAsync(O[q], S[q], nc[q] * fs * w, cudaMemcpyDeviceToDevice, h->s));
    void* oo = h->f32 ? (void*)h->cf.oomf : (void*)h->cd.oomf;
    if (oo) CK(h, cudaMemcpyAsync(oo, S[1], 3 * fs * w, cudaMemcpyDeviceToDevice, h->s));  // ooState = State
    return gam_calc_dt(h, dt_local);
}

extern "C" int gam_set_start(gam_handle* h, double dt) {
    if (!h) return GAM_EINVAL;
    return set_scalars(h, 0.0, -dt, dt, 0);
}

extern "C" int gam_step_begin(gam_handle* h) {
    if (!h) return GAM_EINVAL;
    int rc = require_slab(h);
    if (rc || (rc = step_ready(h))) return rc;
    GamScalars s;
    CK(h, cudaMemcpyAsync(&s, h->sc, sizeof(s), cudaMemcpyDeviceToHost, h->s));
    CK(h, cudaStreamSynchronize(h->s));
    if (s.halted) return fail(h, s.status == 5 ? GAM_EDT_DISASTER : GAM_EDT_BAD, "a previous step failed CalcDT");
    if ((rc = ensure_phase_graph(h, h->cur, 0))) return rc;
    if ((rc = ensure_phase_graph(h, h->cur, 1))) return rc;
    CK(h, cudaEventRecord(h->ev0, h->s));
    CK(h, cudaGraphLaunch(h->pgraph[h->cur][0], h->s));
    return GAM_OK;
}

extern "C" int gam_dt_partial(gam_handle* h, uint64_t* dtmin_bits, int32_t* nbad) {
    if (!h || !dtmin_bits || !nbad) return GAM_EINVAL;
    GamScalars s;
    CK(h, cudaMemcpyAsync(&s, h->sc, sizeof(s), cudaMemcpyDeviceToHost, h->s));
    CK(h, cudaStreamSynchronize(h->s));
    *dtmin_bits = s.dtmin_bits;
    *nbad = s.nbad;
    return GAM_OK;
}

extern "C" int gam_step_end(gam_handle* h, uint64_t dtmin_bits, int32_t nbad, double* dt, double* t) {
    if (!h) return GAM_EINVAL;
    int rc = require_slab(h);
    if (rc) return rc;
    unsigned long long bits = dtmin_bits;
    int nb = nbad;
    CK(h, cudaMemcpyAsync(&h->sc->dtmin_bits, &bits, sizeof(bits), cudaMemcpyHostToDevice, h->s));
    CK(h, cudaMemcpyAsync(&h->sc->nbad, &nb, sizeof(nb), cudaMemcpyHostToDevice, h->s));
    CK(h, cudaGraphLaunch(h->pgraph[h->cur][1], h->s));
    CK(h, cudaEventRecord(h->ev1, h->s));
    GamScalars s;
    CK(h, cudaMemcpyAsync(&s, h->sc, sizeof(s), cudaMemcpyDeviceToHost, h->s));
    CK(h, cudaStreamSynchronize(h->s));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, h->ev0, h->ev1);
    h->lastMs = ms;
    h->cur ^= 1;
    if (dt) *dt = s.dt;
    if (t) *t = s.t;
    if (int rcb = check_bounds(h, s)) return rcb;
    if (s.halted)
        return fail(h, s.status == 5 ? GAM_EDT_DISASTER : GAM_EDT_BAD,
                    s.status == 5 ? "CalcDT: timestep too small or not finite" : "CalcDT: timestep dropped 10x or below limDT0");
    return GAM_OK;
}

// device-resident k-slab steps: the dt candidate leaves and the reduced
// value returns through device memory
__global__ void k_partial_out(const GamScalars* sc, int64_t* bits, int64_t* nbad) {
    *bits = (int64_t)sc->dtmin_bits;
    *nbad = (int64_t)sc->nbad;
}
__global__ void k_partial_in(GamScalars* sc, const int64_t* bits, const int64_t* nbad) {
    sc->dtmin_bits = (unsigned long long)*bits;
    sc->nbad = (int)*nbad;
}

extern "C" int gam_set_stream(gam_handle* h, void* stream) {
    if (!h) return GAM_EINVAL;
    cudaStream_t ns = stream ? (cudaStream_t)stream : h->own_s;
    if (ns != h->s) CK(h, cudaStreamSynchronize(h->s));  // work already enqueued finishes first
    h->s = ns;
    return GAM_OK;
}

extern "C" int gam_step_begin_dev(gam_handle* h) {
    if (!h) return GAM_EINVAL;
    int rc = require_slab(h);
    if (rc || (rc = step_ready(h))) return rc;
    if ((rc = ensure_phase_graph(h, h->cur, 0))) return rc;
    if ((rc = ensure_phase_graph(h, h->cur, 1))) return rc;
    if (h->nasync == 0) CK(h, cudaEventRecord(h->ev0, h->s));
    CK(h, cudaGraphLaunch(h->pgraph[h->cur][0], h->s));
    return GAM_OK;
}

extern "C" int gam_dt_partial_dev(gam_handle* h, int64_t* dtmin_bits, int64_t* nbad) {
    if (!h || !dtmin_bits || !nbad) return GAM_EINVAL;
    k_partial_out<<<1, 1, 0, h->s>>>(h->sc, dtmin_bits, nbad);
    CK(h, cudaGetLastError());
    return GAM_OK;
}

extern "C" int gam_step_end_dev(gam_handle* h, const int64_t* dtmin_bits, const int64_t* nbad) {
    if (!h || !dtmin_bits || !nbad) return GAM_EINVAL;
    int rc = require_slab(h);
    if (rc) return rc;
    k_partial_in<<<1, 1, 0, h->s>>>(h->sc, dtmin_bits, nbad);
    CK(h, cudaGetLastError());
    CK(h, cudaGraphLaunch(h->pgraph[h->cur][1], h->s));
    CK(h, cudaEventRecord(h->ev1, h->s));
    h->cur ^= 1;
    h->nasync++;
    return GAM_OK;
}

extern "C" int gam_step_status(gam_handle* h, double* dt, double* t) {
    if (!h) return GAM_EINVAL;
    GamScalars s;
    CK(h, cudaMemcpyAsync(&s, h->sc, sizeof(s), cudaMemcpyDeviceToHost, h->s));
    CK(h, cudaStreamSynchronize(h->s));
    if (h->nasync > 0) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, h->ev0, h->ev1);
        h->lastMs = ms;
    }
    h->nasync = 0;
    if (dt) *dt = s.dt;
    if (t) *t = s.t;
    if (int rcb = check_bounds(h, s)) return rcb;
    if (s.halted)
        return fail(h, s.status == 5 ? GAM_EDT_DISASTER : GAM_EDT_BAD,
                    s.status == 5 ? "CalcDT: timestep too small or not finite" : "CalcDT: timestep dropped 10x or below limDT0");
    return GAM_OK;
}

extern "C" int gam_set_tile_edges(gam_handle* h, int32_t dir, int32_t lowest, int32_t highest) {
    if (!h || dir < 0 || dir > 2) return GAM_EINVAL;
    if (!is_tile(h)) return fail(h, GAM_ESTATE, "the handle is not a tile");
    h->tileEdge[2 * dir] = lowest ? 1 : 0;
    h->tileEdge[2 * dir + 1] = highest ? 1 : 0;
    set_dt_range(h);
    return GAM_OK;
}
extern "C" int gam_set_slab_edges(gam_handle* h, int32_t lowest, int32_t highest) {
    return gam_set_tile_edges(h, 2, lowest, highest);
}
