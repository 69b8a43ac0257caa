// ref_letkf_glue.cu -- ORACLE TOOLING (test infrastructure only).
//
// The glue half of the reference-side LETKF checker (ref_letkf_solver.cu holds the
// solver half and describes the whole).  This translation unit includes the
// reference's src/config.h and src/lbm.h unmodified, compiled where they lie with the
// reference's nvcc flags and -D knobs (oracle/Makefile), and restates letkf.cu's glue
// kernels in the same types and expressions, with the grid size taken at run time:
// set_rR (letkf.cu:75-114), pack_xk (:133-143), pack_yk (:148-187, the moments rf, uf,
// vf of lbm.h:72-109), set_yo (:230-269).  It is a separate unit because the reference's
// headers include the legacy <cublas.h>, which CUDA 12 refuses beside the <cublas_v2.h>
// that <cusolverDn.h> includes.
#include <cstdlib>

#include "config.h"
#include "lbm.h"
#include "ref_letkf_glue.h"

#ifndef DA_LETKF
#error build with -DDA_LETKF (oracle/Makefile)
#endif

// ---- window geometry and parameters (letkf.cu:29-56) -------------------------
static constexpr auto xyprune = config::da_xyprune;
static constexpr real beta = LETKF_COVINF;
#ifndef LETKF_RLOC_LEN
static constexpr real d_local = xyprune - 1;
static constexpr int n_obs_local = xyprune == 1 ? 0 : 2;
static constexpr int obs_offset = xyprune == 1 ? 0 : 1;
static constexpr int n_obs_x = xyprune == 1 ? 1 : 4;
#else
static constexpr real d_local = LETKF_RLOC_LEN * xyprune;
static constexpr int obs_offset = 0;
static constexpr int n_obs_local = LETKF_RLOC_LEN * 2;
static constexpr int n_obs_x = n_obs_local * 2 + 1;
#endif
static constexpr int n_obs = n_obs_x * n_obs_x * 3;

// ---- letkf.cu's glue, restated with the grid size at run time ------------------------
__global__ void k_pack_xk(const real* f, real* xk, int nxy) {  // letkf.cu:133-143
    const int i = threadIdx.x + blockDim.x * blockIdx.x;
    const int q = blockIdx.y;
    if (i >= nxy) return;
    xk[q + config::Q * i] = f[i + nxy * q];
}

__global__ void k_pack_yk(const real* f, real* yk, int nx, int ny) {  // letkf.cu:148-187
    const int ir = threadIdx.x, jr = threadIdx.y;
    const int r = ir + jr * n_obs_x;
    const int it = blockIdx.x, jt = blockIdx.y;
    const int bt = it + nx * jt;
    const int ig = it, jg = jt;
    const int io = (int(ig / xyprune) + ir - (n_obs_local - obs_offset)) * xyprune;
    const int jo = (int(jg / xyprune) + jr - (n_obs_local - obs_offset)) * xyprune;
    const int di = abs(ig - io);
    const int dj = abs(jg - jo);
    const int iop = (io + nx) % nx;
    const int jop = (jo + ny) % ny;
    real fc[config::Q];
    for (int q = 0; q < config::Q; q++) fc[q] = f[iop + nx * jop + nx * ny * q];
    auto rc = rf(fc);
    auto uc = uf(fc, rc);
    auto vc = vf(fc, rc);
    if (di > n_obs_local * xyprune || dj > n_obs_local * xyprune) { uc = 0; vc = 0; rc = 0; }
    const auto k = r + n_obs * bt;
    yk[k] = uc;
    yk[k + n_obs_x * n_obs_x] = vc;
    yk[k + 2 * n_obs_x * n_obs_x] = rc;
}

__global__ void k_set_yo(real* yo, size_t stride, const real* uo, const real* vo, const real* ro, int nx, int ny,
                         int j_off) {  // letkf.cu:230-269
    const int ir = threadIdx.x, jr = threadIdx.y;
    const int r = ir + jr * n_obs_x;
    const int it = blockIdx.x, jt = blockIdx.y;
    const int bt = it + nx * jt;
    const int ig = it, jg = jt + j_off;
    const int io = (int(ig / xyprune) + ir - (n_obs_local - obs_offset)) * xyprune;
    const int jo = (int(jg / xyprune) + jr - (n_obs_local - obs_offset)) * xyprune;
    const int di = abs(ig - io);
    const int dj = abs(jg - jo);
    const int iop = (io + nx) % nx;
    const int jop = (jo + ny) % ny;
    const int i = iop + nx * jop;
    const int k = r + n_obs * bt;
    auto uc = uo[i];
    auto vc = vo[i];
    auto rc = ro[i];
    if (di > n_obs_local * xyprune || dj > n_obs_local * xyprune) { uc = 0; vc = 0; rc = 0; }
    (void)stride;
    yo[k] = uc;
    yo[k + n_obs_x * n_obs_x] = vc;
    yo[k + 2 * n_obs_x * n_obs_x] = rc;
}

__global__ void k_set_rR(real* e, int n_rows, size_t stride, int nx, int i_batch0) {  // letkf.cu:75-114
    const int i_obs = threadIdx.x, j_obs = threadIdx.y;
    const int ij_obs = i_obs + n_obs_x * j_obs;
    const int i_batch = blockIdx.z;
    const int i0_stt = 0;
    const int j0_stt = i_batch0 / nx;
    const int i_stt = i0_stt + i_batch % nx;
    const int j_stt = j0_stt + i_batch / nx;
    const int k = ij_obs + ij_obs * n_rows + i_batch * stride;
    const int kofs = n_obs_x * n_obs_x + (n_obs_x * n_obs_x) * n_rows;
    e[k] = powf(config::obs_error_u, real(-2));
    e[k + kofs] = powf(config::obs_error_u, real(-2));
    e[k + 2 * kofs] = powf(config::obs_error_rho, real(-2));
    if (xyprune > 1) {
        constexpr real cutoff = d_local + 1e-6;
        const int io_stt = (int(i_stt / xyprune) + i_obs - (n_obs_local - obs_offset)) * xyprune;
        const int jo_stt = (int(j_stt / xyprune) + j_obs - (n_obs_local - obs_offset)) * xyprune;
        const real di = i_stt - io_stt;
        const real dj = j_stt - jo_stt;
        const real d = sqrtf(di * di + dj * dj) / cutoff;
        const real gaspari_cohn =
            (d <= 0) ? 1 :
            (d <= 1) ? -d * d * d * d * d / 4. + d * d * d * d / 2. + d * d * d * 5. / 8. - d * d * 5. / 3. + 1 :
            (d <= 2) ? d * d * d * d * d / 12. - d * d * d * d / 2. + d * d * d * 5. / 8. + d * d * 5. / 3. - d * 5 + 4 -
                           2. / 3. / d :
                       0;
        e[k] *= gaspari_cohn;
        e[k + kofs] *= gaspari_cohn;
        e[k + 2 * kofs] *= gaspari_cohn;
    }
}

namespace glue {
int n_obs_total() { return n_obs; }
int n_obs_side() { return n_obs_x; }
float inflation() { return beta; }
int xyprune() { return ::xyprune; }
float obs_error_u() { return config::obs_error_u; }
float obs_error_rho() { return config::obs_error_rho; }
void pack_xk(const float* f, float* xk, int nxy) {
    k_pack_xk<<<dim3((unsigned(nxy) + 255) / 256, config::Q), 256>>>(f, xk, nxy);
}
void pack_yk(const float* f, float* yk, int nx, int ny) {
    k_pack_yk<<<dim3(nx, ny), dim3(n_obs_x, n_obs_x)>>>(f, yk, nx, ny);
}
void set_yo(float* yo, size_t stride, const float* uo, const float* vo, const float* ro, int nx, int ny, int M,
            int j_off) {
    k_set_yo<<<dim3(nx, ny / M), dim3(n_obs_x, n_obs_x)>>>(yo, stride, uo, vo, ro, nx, ny, j_off);
}
void set_rR(float* rR, int n_rows, size_t stride, int nx, int i_batch0, int n_batch) {
    k_set_rR<<<dim3(1, 1, n_batch), dim3(n_obs_x, n_obs_x)>>>(rR, n_rows, stride, nx, i_batch0);
}
}  // namespace glue
