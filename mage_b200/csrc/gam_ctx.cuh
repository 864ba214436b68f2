// Id of the calling thread's current CUDA context (0 if none or if the driver
// does not report it), through the driver's entry points as the runtime
// exposes them (no link to libcuda). Host-side caches of device objects
// (streams, events, device tables) key on it next to the device number, so
// that after cudaDeviceReset, which gives the device a new context, they are
// made again instead of used stale.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

inline unsigned long long gam_current_ctx_id() {
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
