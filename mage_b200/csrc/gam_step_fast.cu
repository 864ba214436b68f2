// Step kernels of the product path (FMA contraction on): FP64 drop-in form
// and FP32 precision form.
#define GAM_NS gam_fast
#define GAM_CUDA_MATH 1
#define GAM_FAST_RECIP 1  // shared divisors as one reciprocal (Quot)
#include "gam_step_impl.cuh"

void gam_fast_step_f64(const Ctx<double>& C, int cur, cudaStream_t s) { gam_fast::launch_step<double>(C, cur, s); }
void gam_fast_dt_f64(const Ctx<double>& C, int cur, cudaStream_t s) { gam_fast::launch_dt_only<double>(C, cur, s); }
void gam_fast_step_f32(const Ctx<float>& C, int cur, cudaStream_t s) { gam_fast::launch_step<float>(C, cur, s); }
void gam_fast_dt_f32(const Ctx<float>& C, int cur, cudaStream_t s) { gam_fast::launch_dt_only<float>(C, cur, s); }
void gam_fast_init_f64(const Ctx<double>& C, int cur, cudaStream_t s) { gam_fast::launch_init<double>(C, cur, s); }
void gam_fast_bfield_f64(const Ctx<double>& C, int cur, cudaStream_t s) { gam_fast::launch_bfield<double>(C, cur, s); }
void gam_fast_bfield_f32(const Ctx<float>& C, int cur, cudaStream_t s) { gam_fast::launch_bfield<float>(C, cur, s); }
void gam_fast_init_f32(const Ctx<float>& C, int cur, cudaStream_t s) { gam_fast::launch_init<float>(C, cur, s); }
void gam_fast_prepare_f64() { gam_fast::prepare<double>(); }
void gam_fast_prepare_f32() { gam_fast::prepare<float>(); }
void gam_fast_profile_f64(const Ctx<double>& C, int cur, cudaStream_t s, int reps, double* ms) { gam_fast::profile_step<double>(C, cur, s, reps, ms); }
void gam_fast_profile_f32(const Ctx<float>& C, int cur, cudaStream_t s, int reps, double* ms) { gam_fast::profile_step<float>(C, cur, s, reps, ms); }
void gam_fast_phase_f64(const Ctx<double>& C, int cur, cudaStream_t s, int phase) { gam_fast::launch_step_phase<double>(C, cur, s, phase); }
void gam_fast_halo_f64(const Ctx<double>& C, int cur, cudaStream_t s, int dside, int unpack, int copyB, void* buf) { gam_fast::launch_halo<double>(C, cur, s, dside, unpack, copyB, buf); }
void gam_fast_phase_f32(const Ctx<float>& C, int cur, cudaStream_t s, int phase) { gam_fast::launch_step_phase<float>(C, cur, s, phase); }
void gam_fast_halo_f32(const Ctx<float>& C, int cur, cudaStream_t s, int dside, int unpack, int copyB, void* buf) { gam_fast::launch_halo<float>(C, cur, s, dside, unpack, copyB, buf); }
