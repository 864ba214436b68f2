// FP64 step kernels without FMA contraction (built with -fmad=false): every
// operation is one IEEE-rounded +, -, *, / or sqrt in the reference's order,
// so the result equals an IEEE-strict CPU evaluation of the same step.
#define GAM_NS gam_strict
#define GAM_STRICT_KERNELS 1
#include "gam_step_impl.cuh"

void gam_strict_step_f64(const Ctx<double>& C, int cur, cudaStream_t s) { gam_strict::launch_step<double>(C, cur, s); }
void gam_strict_dt_f64(const Ctx<double>& C, int cur, cudaStream_t s) { gam_strict::launch_dt_only<double>(C, cur, s); }
void gam_strict_init_f64(const Ctx<double>& C, int cur, cudaStream_t s) { gam_strict::launch_init<double>(C, cur, s); }
void gam_strict_bfield_f64(const Ctx<double>& C, int cur, cudaStream_t s) { gam_strict::launch_bfield<double>(C, cur, s); }
void gam_strict_prepare_f64() { gam_strict::prepare<double>(); }
void gam_strict_profile_f64(const Ctx<double>& C, int cur, cudaStream_t s, int reps, double* ms) { gam_strict::profile_step<double>(C, cur, s, reps, ms); }
void gam_strict_phase_f64(const Ctx<double>& C, int cur, cudaStream_t s, int phase) { gam_strict::launch_step_phase<double>(C, cur, s, phase); }
void gam_strict_halo_f64(const Ctx<double>& C, int cur, cudaStream_t s, int dside, int unpack, int copyB, void* buf) { gam_strict::launch_halo<double>(C, cur, s, dside, unpack, copyB, buf); }
