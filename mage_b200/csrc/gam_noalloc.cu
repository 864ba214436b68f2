// Conserved totals over caller-owned device arrays, without allocating.
//
// Some callers cannot allocate device memory while they run: a host code
// whose device memory is handed out by another framework's pool (a PyTorch
// caching allocator, a coupler that reserves everything at start-up), or a
// driver that must not call cudaMalloc between set-up and shutdown because
// allocation synchronises the device and may fail once memory is fragmented.
// gam_totals_noalloc serves them: it reads the caller's Fortran-layout State%Gas
// and Grid%volume on the device, writes the five totals to the caller's device
// buffer, and keeps its block partial sums in the fixed file-scope array below
// instead of calling cudaMalloc.
#include <cuda.h>
#include <cuda_runtime.h>
#include <mutex>
#include <stdio.h>
#include <string.h>
#include "../../include/gamgpu.h"

namespace {

constexpr int NA_NT = 256;       // threads per block
constexpr long NA_CHUNK = 8192;  // active cells summed by one block
constexpr int NA_MAXB = 8192;    // partial-sum slots per variable
// At most NA_MAXB * NA_CHUNK = 67,108,864 active cells per call. The array
// (5 x 8192 doubles = 320 KiB) exists on every device that loads the library
// and stays there until the process exits.
constexpr long NA_MAX_CELLS = (long)NA_MAXB * NA_CHUNK;
static __device__ __align__(256) double g_totals_scratch[5 * NA_MAXB];

constexpr int NA_MAX_DEVICES = 64;
std::mutex g_mu;
// Per device: the array's address and the id of the context it belongs to.
// cudaDeviceReset destroys the context (and the module that holds the array);
// the next call then runs in a new context with a new id and looks the
// address up again instead of passing a stale one.
double* g_scratch_addr[NA_MAX_DEVICES] = {nullptr};
unsigned long long g_scratch_ctx[NA_MAX_DEVICES] = {0};

// Id of the calling thread's current context (0 if none), through the
// driver's entry points as the runtime exposes them (no link to libcuda).
unsigned long long current_ctx_id() {
    typedef CUresult (*CtxGetCurrent)(CUcontext*);
    typedef CUresult (*CtxGetId)(CUcontext, unsigned long long*);
    static CtxGetCurrent get_cur = nullptr;
    static CtxGetId get_id = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_cur = (CtxGetCurrent)f;
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = (CtxGetId)f;
    }
    if (!get_cur || !get_id) return 0;
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (get_cur(&ctx) != CUDA_SUCCESS || !ctx) return 0;
    if (get_id(ctx, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// Block b sums the active cells [b*CHUNK, (b+1)*CHUNK) of Gas*volume in a
// fixed pattern and tree, so the result does not depend on timing.
__global__ void k_na_partials(const double* __restrict__ Gas, const double* __restrict__ vol, int Nip, int Njp,
                              int Nkp, long ncells, double* scratch) {
    __shared__ double sh[5][NA_NT];
    const long Ni = Nip + 8, Nj = Njp + 8, Nk = Nkp + 8, ncomp = Ni * Nj * Nk;
    const long c0 = blockIdx.x * NA_CHUNK;
    const long c1 = c0 + NA_CHUNK < ncells ? c0 + NA_CHUNK : ncells;
    double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    for (long q = c0 + threadIdx.x; q < c1; q += NA_NT) {
        const long i = 4 + q % Nip, r = q / Nip, j = 4 + r % Njp, k = 4 + r / Njp;
        const long c = i + Ni * (j + Nj * k);
        const double dV = vol[c];
        for (int v = 0; v < 5; v++) acc[v] += Gas[v * ncomp + c] * dV;
    }
    for (int v = 0; v < 5; v++) sh[v][threadIdx.x] = acc[v];
    __syncthreads();
    for (int w = NA_NT / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            for (int v = 0; v < 5; v++) sh[v][threadIdx.x] += sh[v][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int v = 0; v < 5; v++) scratch[v * NA_MAXB + blockIdx.x] = sh[v][0];
}

// One block adds the nb partials of each variable in a fixed order.
__global__ void k_na_final(const double* __restrict__ scratch, int nb, double* out) {
    __shared__ double sh[5][NA_NT];
    for (int v = 0; v < 5; v++) {
        double a = 0.0;
        for (int q = threadIdx.x; q < nb; q += NA_NT) a += scratch[v * NA_MAXB + q];
        sh[v][threadIdx.x] = a;
    }
    __syncthreads();
    for (int w = NA_NT / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            for (int v = 0; v < 5; v++) sh[v][threadIdx.x] += sh[v][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int v = 0; v < 5; v++) out[v] = sh[v][0];
}

void put_err(char* err, int errlen, const char* msg) {
    if (err && errlen > 0) {
        strncpy(err, msg, (size_t)errlen - 1);
        err[errlen - 1] = '\0';
    }
}

}  // namespace

extern "C" int gam_totals_noalloc(const double* Gas, const double* volume, int32_t Nip, int32_t Njp, int32_t Nkp,
                                  double* out, void* stream, char* err, int32_t errlen) {
    if (!Gas || !volume || !out) {
        put_err(err, errlen, "gam_totals_noalloc: null array pointer");
        return GAM_EINVAL;
    }
    if (Nip < 1 || Njp < 1 || Nkp < 1) {
        put_err(err, errlen, "gam_totals_noalloc: grid sizes must be >= 1");
        return GAM_EBADDIM;
    }
    const long ncells = (long)Nip * Njp * Nkp;
    if (ncells > NA_MAX_CELLS) {
        char m[200];
        snprintf(m, sizeof(m), "gam_totals_noalloc: %ld active cells exceed the fixed scratch limit of %ld", ncells,
                 NA_MAX_CELLS);
        put_err(err, errlen, m);
        return GAM_EINVAL;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= NA_MAX_DEVICES) {
        put_err(err, errlen, "gam_totals_noalloc: no current CUDA device");
        return GAM_ECUDA;
    }
    double* scratch;
    {
        // set-up, once per device and context: the device address of the
        // array, looked up with this device current (the first call on a
        // device does this, so make it outside any stream capture); looked up
        // again after cudaDeviceReset, which gives the device a new context
        std::lock_guard<std::mutex> lock(g_mu);
        const unsigned long long id = current_ctx_id();
        if (!g_scratch_addr[dev] || id == 0 || id != g_scratch_ctx[dev]) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_totals_scratch);
            if (e != cudaSuccess) {
                put_err(err, errlen, cudaGetErrorString(e));
                return GAM_ECUDA;
            }
            g_scratch_addr[dev] = (double*)p;
            g_scratch_ctx[dev] = current_ctx_id();  // the lookup made the context current if it was not
        }
        scratch = g_scratch_addr[dev];
    }
    const int nb = (int)((ncells + NA_CHUNK - 1) / NA_CHUNK);
    cudaStream_t s = (cudaStream_t)stream;
    // an error left pending by an earlier, unrelated launch on this thread is
    // reported here as this call's GAM_ECUDA
    k_na_partials<<<nb, NA_NT, 0, s>>>(Gas, volume, Nip, Njp, Nkp, ncells, scratch);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        put_err(err, errlen, cudaGetErrorString(e));
        return GAM_ECUDA;
    }
    k_na_final<<<1, NA_NT, 0, s>>>(scratch, nb, out);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        put_err(err, errlen, cudaGetErrorString(e));
        return GAM_ECUDA;
    }
    return GAM_OK;
}
