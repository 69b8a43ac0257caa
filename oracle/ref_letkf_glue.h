// ref_letkf_glue.h -- ORACLE TOOLING (test infrastructure only): the interface between
// the two halves of the reference-side LETKF checker (ref_letkf_glue.cu, which sees the
// reference's headers, and ref_letkf_solver.cu, which sees cuBLAS and cuSOLVER).
// All launches go to the default stream; callers synchronise.
#pragma once
#include <cstddef>

namespace glue {
int n_obs_total();    // n_obs = 3 n_obs_x^2 (letkf.cu:45-56)
int n_obs_side();     // n_obs_x
float inflation();    // beta = LETKF_COVINF as the reference's `real` (letkf.cu:32)
int xyprune();        // DA_XYPRUNE (config.h:185)
float obs_error_u();  // OBS_ERROR_U, OBS_ERROR_RHO as the reference's `real` (config.h:191-198)
float obs_error_rho();
void pack_xk(const float* f, float* xk, int nxy);
void pack_yk(const float* f, float* yk, int nx, int ny);
void set_yo(float* yo, size_t stride, const float* uo, const float* vo, const float* ro, int nx, int ny, int M,
            int j_off);
void set_rR(float* rR, int n_rows, size_t stride, int nx, int i_batch0, int n_batch);
}  // namespace glue
