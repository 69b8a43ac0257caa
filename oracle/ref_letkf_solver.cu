// ref_letkf_solver.cu -- ORACLE TOOLING (test infrastructure only).
//
// The reference's LETKF analysis as its own code computes it, where that code cannot
// be built here.  The reference's solver class (src/util/letkf_solver.h) and its
// driver (src/letkf.cu) include <mpi.h> and <hdf5.h> (through util/cu_matrix.hpp and
// util/mpi_wrapper.hpp); neither library is installed, so those two files cannot be
// compiled.  All of the analysis arithmetic sits in NVIDIA libraries the reference
// calls, plus a few elementwise kernels.  This half of our checker therefore:
//
//   * takes the glue of letkf.cu from ref_letkf_glue.cu, which includes the
//     reference's src/config.h and src/lbm.h unmodified (compiled where they lie, with
//     the reference's nvcc flags and -D knobs, by oracle/Makefile) and restates
//     set_rR (letkf.cu:75-114), pack_xk (:133-143), pack_yk (:148-187) and set_yo
//     (:230-269) in the same types and expressions, with the grid size taken at run
//     time (the reference fixes nx = 256 at compile time); update_xk (:315-328) is
//     k_scatter here;
//   * restates letkf_solver<float>::solve_evd / solve_xa (letkf_solver.h:235-349)
//     call for call: cublasSgemmStridedBatched with the reference wrapper's
//     m, n, k, leading dimensions and strides (cu_matrix_cublas_wrapper.hpp:163-223),
//     cublasScopy / cublasSaxpy over whole buffers (:95-139), the elementwise
//     kernels of cu_matrix.hpp (set_identity :189-205, set_diag :207-230,
//     columnwise_add :233-251, export_column_mean :271-298), and
//     cusolverDnSsyevjBatched with tolerance 1e-6, at most 100 sweeps, unsorted,
//     lower triangle (cu_matrix_eigensolver_wrapper.hpp:186-238);
//   * runs the M "ranks" of the reference one after another: rank r analyses the
//     grid points [r*nxy/M, (r+1)*nxy/M) of every member (letkf.cu:35-37), which
//     is what the reference's alltoall transposes deliver to it.
//
// syevjBatched takes n <= 32.  For M > 32 the reference calls EigenG-Batched,
// which is not available; there each matrix goes to cusolverDnSsyevj with the same
// Jacobi parameters instead (an EVD stand-in, reported to the caller).
// The info buffer holds one int per matrix (the reference allocates one int for
// the whole batch, cu_matrix_eigensolver_wrapper.hpp:219, and cuSOLVER writes
// batchSize of them).
//
// Used by ref_letkf_harness.cu (one analysis of given inputs) and ref_osse_harness.cu
// (the reference's whole forecast-and-assimilate cycle).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <cusolverDn.h>

#include "ref_letkf_glue.h"
#include "ref_letkf_solver.h"

using real = float;  // the reference's `real` without DOUBLE_PRECISION (config.h:113-119)
static constexpr int n_stt = 9;  // config::Q

#define CK(x)                                                                                  \
    do {                                                                                       \
        cudaError_t e_ = (x);                                                                  \
        if (e_ != cudaSuccess) {                                                               \
            std::fprintf(stderr, "%s:%d: %s\n", __FILE__, __LINE__, cudaGetErrorString(e_));    \
            std::exit(2);                                                                      \
        }                                                                                      \
    } while (0)
#define CKB(x)                                                                                 \
    do {                                                                                       \
        cublasStatus_t s_ = (x);                                                               \
        if (s_ != CUBLAS_STATUS_SUCCESS) {                                                     \
            std::fprintf(stderr, "%s:%d: cublas status %d\n", __FILE__, __LINE__, int(s_));    \
            std::exit(2);                                                                      \
        }                                                                                      \
    } while (0)
#define CKS(x)                                                                                 \
    do {                                                                                       \
        cusolverStatus_t s_ = (x);                                                             \
        if (s_ != CUSOLVER_STATUS_SUCCESS) {                                                   \
            std::fprintf(stderr, "%s:%d: cusolver status %d\n", __FILE__, __LINE__, int(s_));  \
            std::exit(2);                                                                      \
        }                                                                                      \
    } while (0)

// ---- batched column-major matrices (cu_matrix.hpp array3dx, align_stride 1) ----
struct Mat {
    real* p = nullptr;
    int rows = 0, cols = 0, batch = 0;
    size_t stride() const { return size_t(rows) * cols; }
    size_t size() const { return stride() * batch; }
    void init(int r, int c, int b) {
        rows = r; cols = c; batch = b;
        CK(cudaMalloc(&p, sizeof(real) * size()));
        CK(cudaMemset(p, 0, sizeof(real) * size()));
    }
    void free() { cudaFree(p); p = nullptr; }
    void zero() { CK(cudaMemset(p, 0, sizeof(real) * size())); }
};

// ---- elementwise kernels of cu_matrix.hpp, same expressions ---------------------
__global__ void k_set_identity(real* ptr, int n, size_t stride, real scale) {  // :189-205
    const auto i = threadIdx.x, j = blockIdx.x, b = blockIdx.y;
    const auto idx = i + n * j + stride * b;
    const real s = (i == j ? scale : 0);
    ptr[idx] = s;
}
__global__ void k_set_diag(real* ptr, int n, size_t stride, const real* vp, size_t v_stride, real scale,
                           real power) {  // :207-230
    const auto i = threadIdx.x, j = blockIdx.x, b = blockIdx.y;
    const auto idx = i + n * j + stride * b;
    if (i == j) {
        const auto v_idx = i + v_stride * b;
        ptr[idx] = scale * pow(vp[v_idx], power);
    } else {
        ptr[idx] = 0;
    }
}
__global__ void k_columnwise_add(real* ptr, int n_rows, size_t stride, const real* vp, size_t v_stride,
                                 real scale) {  // :233-251
    const auto i = threadIdx.x, j = blockIdx.x, b = blockIdx.y;
    const auto idx = i + n_rows * j + stride * b;
    const auto v_idx = i + v_stride * b;
    ptr[idx] += scale * vp[v_idx];
}
__global__ void k_zero_vec(real* vp, size_t v_stride) {  // :281-284
    vp[threadIdx.x + v_stride * blockIdx.x] = 0;
}
__global__ void k_mean_add_column(const real* ptr, int n_rows, size_t n_cols, size_t stride, real* vp,
                                  size_t v_stride, int j) {  // :286-295
    const auto i = threadIdx.x, b = blockIdx.x;
    const auto idx = i + n_rows * j + stride * b;
    const auto v_idx = i + v_stride * b;
    vp[v_idx] += ptr[idx] / n_cols;
}

void set_identity(Mat& m, real scale) {
    k_set_identity<<<dim3(m.rows, m.batch), m.rows>>>(m.p, m.rows, m.stride(), scale);
    CK(cudaDeviceSynchronize());
}
void set_diag(Mat& m, const Mat& v, real scale, real power) {
    k_set_diag<<<dim3(m.rows, m.batch), m.rows>>>(m.p, m.rows, m.stride(), v.p, v.stride(), scale, power);
    CK(cudaDeviceSynchronize());
}
void columnwise_add(Mat& m, const Mat& v, real scale) {
    k_columnwise_add<<<dim3(m.cols, m.batch), m.rows>>>(m.p, m.rows, m.stride(), v.p, v.stride(), scale);
    CK(cudaDeviceSynchronize());
}
void export_column_mean(const Mat& m, Mat& v) {
    k_zero_vec<<<m.batch, m.rows>>>(v.p, v.stride());
    CK(cudaDeviceSynchronize());
    const size_t n_cols = m.cols;
    for (int j = 0; j < m.cols; j++) {
        k_mean_add_column<<<m.batch, m.rows>>>(m.p, m.rows, n_cols, m.stride(), v.p, v.stride(), j);
        CK(cudaDeviceSynchronize());
    }
}

// ---- cuBLAS calls as the reference's wrapper makes them ----------------------------
struct Blas {
    cublasHandle_t h;
    Blas() { CKB(cublasCreate(&h)); }
    ~Blas() { cublasDestroy(h); }
    void copy(const Mat& x, Mat& y) {  // :95-125
        CKB(cublasScopy(h, int(x.size()), x.p, 1, y.p, 1));
    }
    void axpy(real alpha, const Mat& x, Mat& y) {  // :127-139
        CKB(cublasSaxpy(h, int(x.size()), &alpha, x.p, 1, y.p, 1));
    }
    // C = alpha op(A) op(B) + beta C (:163-195)
    void gemm(Mat& C, const Mat& A, const Mat& B, cublasOperation_t ta = CUBLAS_OP_N,
              cublasOperation_t tb = CUBLAS_OP_N, real alpha = 1, real beta_ = 0) {
        const int k = ta == CUBLAS_OP_N ? A.cols : A.rows;
        CKB(cublasSgemmStridedBatched(h, ta, tb, C.rows, C.cols, k, &alpha, A.p, A.rows, (long long)A.stride(), B.p,
                                      B.rows, (long long)B.stride(), &beta_, C.p, C.rows, (long long)C.stride(),
                                      C.batch));
    }
    // y = alpha op(A) x + beta y as a gemm with n = 1 (:197-223)
    void gemv(Mat& y, const Mat& A, const Mat& x, cublasOperation_t ta = CUBLAS_OP_N, real alpha = 1,
              real beta_ = 0) {
        const int k = ta == CUBLAS_OP_N ? A.cols : A.rows;
        CKB(cublasSgemmStridedBatched(h, ta, CUBLAS_OP_N, y.rows, 1, k, &alpha, A.p, A.rows, (long long)A.stride(),
                                      x.p, x.rows, (long long)x.stride(), &beta_, y.p, y.rows,
                                      (long long)y.stride(), y.batch));
    }
};

// ---- the eigensolver (cu_matrix_eigensolver_wrapper.hpp:168-238) --------------------
struct Eigen {
    cusolverDnHandle_t h;
    syevjInfo_t params;
    Eigen() {
        CKS(cusolverDnCreate(&h));
        CKS(cusolverDnCreateSyevjInfo(&params));
        CKS(cusolverDnXsyevjSetTolerance(params, 1e-6));
        CKS(cusolverDnXsyevjSetMaxSweeps(params, 100));
        CKS(cusolverDnXsyevjSetSortEig(params, 0));
    }
    ~Eigen() {
        cudaFree(work);
        cudaFree(info);
        cusolverDnDestroySyevjInfo(params);
        cusolverDnDestroy(h);
    }
    // work space and info buffer, grown on demand and kept, as the reference's
    // workspace_.reallocate / info_.reallocate keep theirs
    real* work = nullptr;
    int* info = nullptr;
    size_t work_cap = 0, info_cap = 0;
    void reserve(size_t lwork, size_t ninfo) {
        if (lwork > work_cap) {
            cudaFree(work);
            CK(cudaMalloc(&work, sizeof(real) * lwork));
            work_cap = lwork;
        }
        if (ninfo > info_cap) {
            cudaFree(info);
            CK(cudaMalloc(&info, sizeof(int) * ninfo));
            info_cap = ninfo;
        }
    }
    // V holds Q on entry; returns 0 (batched) or 1 (per-matrix stand-in for n > 32)
    int solve(Mat& V, Mat& d) {
        const int n = V.rows, nb = V.batch;
        int lwork = 0;
        int evd = 0;
        if (n <= 32) {
            CKS(cusolverDnSsyevjBatched_bufferSize(h, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n, V.p, n, d.p,
                                                   &lwork, params, nb));
            reserve(size_t(lwork), size_t(nb));
            CKS(cusolverDnSsyevjBatched(h, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n, V.p, n, d.p, work,
                                        lwork, info, params, nb));
        } else {
            evd = 1;
            CKS(cusolverDnSsyevj_bufferSize(h, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n, V.p, n, d.p,
                                            &lwork, params));
            reserve(size_t(lwork), size_t(nb));
            for (int b = 0; b < nb; b++)
                CKS(cusolverDnSsyevj(h, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n, V.p + V.stride() * b, n,
                                     d.p + d.stride() * b, work, lwork, info + b, params));
        }
        CK(cudaDeviceSynchronize());
        std::vector<int> h_info(nb);
        CK(cudaMemcpy(h_info.data(), info, sizeof(int) * nb, cudaMemcpyDeviceToHost));
        for (int b = 0; b < nb; b++)
            if (h_info[b] != 0) std::fprintf(stderr, "warning: syevj info[%d] = %d\n", b, h_info[b]);
        return evd;
    }
};

// the alltoall transposes (letkf_solver.h:135-215): rank r receives, from every
// member k, that member's packed values of the rank's batch
__global__ void k_gather(const real* src_k, real* dst, int rows, int n_ens, int k, int i_batch0, int n_batch) {
    const int i = threadIdx.x;
    const int b = blockIdx.x;
    if (b >= n_batch || i >= rows) return;
    dst[i + size_t(rows) * k + size_t(rows) * n_ens * b] = src_k[i + size_t(rows) * (i_batch0 + b)];
}

// update_xk (letkf.cu:315-328): member k's analysis populations of the rank's batch
__global__ void k_scatter(const real* Xsol, real* f_k, int n_ens, int k, int i_batch0, int n_batch, int nxy) {
    const int q = threadIdx.x;
    const int b = blockIdx.x;
    if (b >= n_batch || q >= n_stt) return;
    f_k[(i_batch0 + b) + size_t(nxy) * q] = Xsol[q + size_t(n_stt) * k + size_t(n_stt) * n_ens * b];
}
__global__ void k_lambda(const real* d, real* lam, int n_ens, int i_batch0, int n_batch) {
    const int k = threadIdx.x;
    const int b = blockIdx.x;
    if (b >= n_batch || k >= n_ens) return;
    lam[size_t(i_batch0 + b) * n_ens + k] = d[k + size_t(n_ens) * b];
}


namespace {
// The solver's matrices, allocated once for a (grid, members) shape and kept, as the
// reference's init_geo (letkf_solver.h:78-109) allocates them once per rank; every rank
// below starts from zeroed matrices, as a fresh init_geo would give it.
struct Workspace {
    int nx = 0, ny = 0, M = 0;
    std::vector<real*> xk, yk;
    Mat X, Y, yo, xbar, ybar, dX, dY, dyo, rR, Q, V, d, D, tmp_ee, tmp_oe, tmp_o, tmp_e, P, w, W, Xsol;
    Blas* blas = nullptr;
    Eigen* eigen = nullptr;
    std::vector<Mat*> mats() {
        return {&X, &Y, &yo, &xbar, &ybar, &dX, &dY, &dyo, &rR, &Q, &V, &d, &D, &tmp_ee, &tmp_oe, &tmp_o, &tmp_e, &P,
                &w, &W, &Xsol};
    }
    void ensure(int nx_, int ny_, int M_) {
        if (nx_ == nx && ny_ == ny && M_ == M) return;
        for (real* p : xk) cudaFree(p);
        for (real* p : yk) cudaFree(p);
        for (Mat* m : mats())
            if (m->p) m->free();
        nx = nx_; ny = ny_; M = M_;
        const size_t nxy = size_t(nx) * ny;
        const int n_obs = glue::n_obs_total();
        const int n_batch = int(nxy / M);
        xk.assign(M, nullptr);
        yk.assign(M, nullptr);
        for (int k = 0; k < M; k++) {
            CK(cudaMalloc(&xk[k], sizeof(real) * n_stt * nxy));
            CK(cudaMalloc(&yk[k], sizeof(real) * n_obs * nxy));
        }
        X.init(n_stt, M, n_batch); Y.init(n_obs, M, n_batch); yo.init(n_obs, 1, n_batch);
        xbar.init(n_stt, 1, n_batch); ybar.init(n_obs, 1, n_batch); dyo.init(n_obs, 1, n_batch);
        dX.init(n_stt, M, n_batch); dY.init(n_obs, M, n_batch);
        rR.init(n_obs, n_obs, n_batch);
        Q.init(M, M, n_batch); V.init(M, M, n_batch); d.init(M, 1, n_batch); D.init(M, M, n_batch);
        tmp_ee.init(M, M, n_batch); tmp_oe.init(n_obs, M, n_batch); tmp_o.init(n_obs, 1, n_batch);
        tmp_e.init(M, 1, n_batch); P.init(M, M, n_batch); w.init(M, 1, n_batch); W.init(M, M, n_batch);
        Xsol.init(n_stt, M, n_batch);
        if (!blas) blas = new Blas();
        if (!eigen) eigen = new Eigen();
    }
};
Workspace ws;  // the drivers are single-threaded
}  // namespace

namespace refletkf {

int analyse(const std::vector<const float*>& f_in, const std::vector<float*>& f_out, const float* ro_d,
            const float* uo_d, const float* vo_d, int nx, int ny, int j0, int j1, float* lam) {
    const int M = int(f_in.size());
    const int n_obs = glue::n_obs_total();
    const real beta = glue::inflation();
    const size_t nxy = size_t(nx) * ny;
    if (M < 2 || int(f_out.size()) != M || ny % M || j0 < 0 || j1 > ny || j0 >= j1) {
        std::fprintf(stderr, "refletkf::analyse: bad arguments\n");
        std::exit(1);
    }
    // members' packed state and observation ensemble (the reference's xk, yk per rank)
    ws.ensure(nx, ny, M);
    std::vector<real*>& xk = ws.xk;
    std::vector<real*>& yk = ws.yk;
    const real *ro = ro_d, *uo = uo_d, *vo = vo_d;
    // every member packs its xk and yk over the whole grid (letkf.cu:133-187)
    for (int k = 0; k < M; k++) {
        glue::pack_xk(f_in[k], xk[k], int(nxy));
        glue::pack_yk(f_in[k], yk[k], nx, ny);
        CK(cudaDeviceSynchronize());
    }

    Blas& blas = *ws.blas;
    Eigen& eigen = *ws.eigen;
    int evd = 0;
    const int n_batch = int(nxy / M);
    for (int rank = 0; rank < M; rank++) {
        const int i_batch0 = n_batch * rank;
        const int r_j0 = i_batch0 / nx, r_j1 = (i_batch0 + n_batch) / nx;
        if (r_j1 <= j0 || r_j0 >= j1) continue;
        // init_geo (letkf_solver.h:80-109): the kept matrices, zeroed
        for (Mat* m : ws.mats()) m->zero();
        Mat &X = ws.X, &Y = ws.Y, &yo = ws.yo, &xbar = ws.xbar, &ybar = ws.ybar, &dX = ws.dX, &dY = ws.dY,
            &dyo = ws.dyo, &rR = ws.rR, &Q = ws.Q, &V = ws.V, &d = ws.d, &D = ws.D, &tmp_ee = ws.tmp_ee,
            &tmp_oe = ws.tmp_oe, &tmp_o = ws.tmp_o, &tmp_e = ws.tmp_e, &P = ws.P, &w = ws.w, &W = ws.W,
            &Xsol = ws.Xsol;
        set_identity(rR, 1);
        // set_rR (init_letkf) and the inputs of this rank
        glue::set_rR(rR.p, rR.rows, rR.stride(), nx, i_batch0, n_batch);
        CK(cudaDeviceSynchronize());
        for (int k = 0; k < M; k++) {
            k_gather<<<n_batch, n_obs>>>(yk[k], Y.p, n_obs, M, k, i_batch0, n_batch);
            k_gather<<<n_batch, n_stt>>>(xk[k], X.p, n_stt, M, k, i_batch0, n_batch);
        }
        glue::set_yo(yo.p, yo.stride(), uo, vo, ro, nx, ny, M, i_batch0 / nx);
        CK(cudaDeviceSynchronize());

        // solve_evd (letkf_solver.h:235-272)
        export_column_mean(Y, ybar);
        blas.copy(Y, dY);
        columnwise_add(dY, ybar, -1);
        blas.copy(yo, dyo);
        blas.axpy(-1, ybar, dyo);
        set_identity(Q, (size_t(M) - 1) / beta);
        blas.gemm(tmp_oe, rR, dY);
        blas.gemm(Q, dY, tmp_oe, CUBLAS_OP_T, CUBLAS_OP_N, 1, 1);
        blas.copy(Q, V);
        evd = eigen.solve(V, d);

        // solve_xa (letkf_solver.h:274-349)
        export_column_mean(X, xbar);
        blas.copy(X, dX);
        columnwise_add(dX, xbar, -1);
        set_diag(D, d, 1, -1);
        blas.gemm(tmp_ee, D, V, CUBLAS_OP_N, CUBLAS_OP_T);
        blas.gemm(P, V, tmp_ee);
        blas.gemv(tmp_o, rR, dyo);
        blas.gemv(tmp_e, dY, tmp_o, CUBLAS_OP_T);
        blas.gemv(w, P, tmp_e);
        set_diag(D, d, 1, -0.5);
        blas.gemm(tmp_ee, D, V, CUBLAS_OP_N, CUBLAS_OP_T);
        blas.gemm(W, V, tmp_ee, CUBLAS_OP_N, CUBLAS_OP_N, sqrt(size_t(M) - 1));
        columnwise_add(W, w, 1);
        blas.gemm(Xsol, dX, W);
        columnwise_add(Xsol, xbar, 1);
        CK(cudaDeviceSynchronize());

        // update_xk of every member, and the eigenvalues
        for (int k = 0; k < M; k++) k_scatter<<<n_batch, 32>>>(Xsol.p, f_out[k], M, k, i_batch0, n_batch, int(nxy));
        if (lam) k_lambda<<<n_batch, (M + 31) / 32 * 32>>>(d.p, lam, M, i_batch0, n_batch);
        CK(cudaDeviceSynchronize());
    }
    return evd;
}

}  // namespace refletkf
