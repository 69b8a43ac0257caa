// ref_letkf_solver.h -- ORACLE TOOLING (test infrastructure only): the reference's
// LETKF analysis (ref_letkf_solver.cu) behind plain device pointers, so that drivers
// that see the reference's headers (which pull in the legacy cublas.h) need not see
// cuBLAS v2 or cuSOLVER.
#pragma once
#include <vector>

namespace refletkf {
// The analysis of the M members' populations f_in[k] (device, [9][ny][nx], the
// reference's layout) with the observation fields ro, uo, vo (device, [ny][nx], NaN
// off the observation lattice) into f_out[k] (device; may be f_in[k]): the points of
// the reference ranks that meet rows [j0, j1) are written, the others left alone.
// lam (device, [ny*nx][M], or null) receives the eigenvalues.  Returns 0 when
// syevjBatched ran, 1 for the per-matrix syevj stand-in (M > 32).  Synchronous.
int analyse(const std::vector<const float*>& f_in, const std::vector<float*>& f_out, const float* ro,
            const float* uo, const float* vo, int nx, int ny, int j0, int j1, float* lam);
}  // namespace refletkf
