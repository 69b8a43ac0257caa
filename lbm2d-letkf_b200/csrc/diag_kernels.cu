// diag_kernels.cu -- FP64 domain reductions over the macroscopic fields:
// kinetic energy, enstrophy and mass of one member or of the ensemble mean
// (the quantities stdata::inspect prints, data.cu:458-542), and the RMSE of the
// ensemble-mean velocity against a truth field (ensemble_stat/main.cpp:108-177).
#include "lbl_internal.h"

namespace lbl {
namespace {

// mean over the selected members of field `var` (0 rho, 1 u, 2 v) at cell ij
__device__ __forceinline__ double field(const float* mac, int nxy, int m0, int m1, int var, int ij) {
    double s = 0;
    for (int m = m0; m < m1; m++) s += mac[(size_t(m) * 3 + var) * nxy + ij];
    return s / double(m1 - m0);
}

__device__ __forceinline__ void block_add(double v, double* out) {
    __shared__ double red[32];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) red[w] = v;
    __syncthreads();
    if (w == 0) {
        v = (l < (blockDim.x >> 5)) ? red[l] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (l == 0) atomicAdd(out, v);
    }
    __syncthreads();
}

__global__ void diag_kernel(const float* __restrict__ mac, int nx, int ny, int m0, int m1, double dx,
                            double* __restrict__ red) {
    const int nxy = nx * ny;
    const int ij = blockIdx.x * blockDim.x + threadIdx.x;
    double e = 0, z = 0, r = 0;
    if (ij < nxy) {
        const int i = ij % nx, j = ij / nx;
        const int ie = j * nx + (i + 1) % nx, iw = j * nx + (i - 1 + nx) % nx;
        const int jn = ((j + 1) % ny) * nx + i, js = ((j - 1 + ny) % ny) * nx + i;
        const double u = field(mac, nxy, m0, m1, 1, ij), v = field(mac, nxy, m0, m1, 2, ij);
        const double vx = (field(mac, nxy, m0, m1, 2, ie) - field(mac, nxy, m0, m1, 2, iw)) / (2 * dx);
        const double uy = (field(mac, nxy, m0, m1, 1, jn) - field(mac, nxy, m0, m1, 1, js)) / (2 * dx);
        e = 0.5 * (u * u + v * v);
        z = 0.5 * (vx - uy) * (vx - uy);
        r = field(mac, nxy, m0, m1, 0, ij);
    }
    block_add(e, red + 0);
    block_add(z, red + 1);
    block_add(r, red + 2);
}

// over the cells [ij0, ij0 + n) of each plane (the whole grid, or a y-slab's own rows)
__global__ void rmse_kernel(const float* __restrict__ mac, int nxy, int M, const float* __restrict__ ut,
                            const float* __restrict__ vt, double* __restrict__ red, int ij0, int n) {
    const int ij = ij0 + blockIdx.x * blockDim.x + threadIdx.x;
    double s = 0;
    if (ij < ij0 + n) {
        const double du = field(mac, nxy, 0, M, 1, ij) - double(ut[ij]);
        const double dv = field(mac, nxy, 0, M, 2, ij) - double(vt[ij]);
        s = du * du + dv * dv;
    }
    block_add(s, red);
}

// Output fields of every member and the ensemble statistics, in the reference's
// FP32 operation order so that the files match its host loops bit for bit
// (io.cu:61-139): vor = (ve - vw) / (2 dx) - (un - us) / (2 dx) per member; over the
// members in order, mean_u += u, mean_v += v, mean_w += vor, w2 += (1/M)(vor vor);
// then means *= 1/M and std = sqrt(w2 - mean_w^2) (all zero for M = 1).  Every
// operation is an explicitly rounded intrinsic, so nothing is contracted into an FMA.
// A NaN vorticity sets *nan (io.cu:79-83).
__global__ void output_fields_kernel(const float* __restrict__ mac, int nx, int ny, int M, float two_dx,
                                     float* __restrict__ vor, float* __restrict__ stats, int* __restrict__ nan) {
    const int nxy = nx * ny;
    const int ij = blockIdx.x * blockDim.x + threadIdx.x;
    if (ij >= nxy) return;
    const int i = ij % nx, j = ij / nx;
    const int ie = j * nx + (i + 1) % nx, iw = j * nx + (i - 1 + nx) % nx;
    const int jn = ((j + 1) % ny) * nx + i, js = ((j - 1 + ny) % ny) * nx + i;
    const float iv = __fdiv_rn(1.f, float(M));
    float um = 0.f, vm = 0.f, wm = 0.f, w2 = 0.f;
    bool bad = false;
    for (int m = 0; m < M; m++) {
        const float* u = mac + (size_t(m) * 3 + 1) * nxy;
        const float* v = mac + (size_t(m) * 3 + 2) * nxy;
        const float uy = __fdiv_rn(__fsub_rn(u[jn], u[js]), two_dx);
        const float vx = __fdiv_rn(__fsub_rn(v[ie], v[iw]), two_dx);
        const float w = __fsub_rn(vx, uy);
        vor[size_t(m) * nxy + ij] = w;
        bad |= (w != w);
        um = __fadd_rn(um, u[ij]);
        vm = __fadd_rn(vm, v[ij]);
        wm = __fadd_rn(wm, w);
        w2 = __fadd_rn(w2, __fmul_rn(iv, __fmul_rn(w, w)));
    }
    if (M > 1) {
        um = __fmul_rn(um, iv);
        vm = __fmul_rn(vm, iv);
        wm = __fmul_rn(wm, iv);
        w2 = __fsqrt_rn(__fsub_rn(w2, __fmul_rn(wm, wm)));
    } else {
        um = vm = wm = w2 = 0.f;
    }
    stats[ij] = um;
    stats[nxy + ij] = vm;
    stats[2 * nxy + ij] = wm;
    stats[3 * nxy + ij] = w2;
    if (bad) atomicOr(nan, 1);
}

}  // namespace

void launch_output_fields(const lbl_ctx* c, const float* mac, float* vor, float* stats, int* nan, cudaStream_t s) {
    output_fields_kernel<<<(c->P.nxy + 255) / 256, 256, 0, s>>>(mac, c->P.nx, c->P.ny, c->P.M, c->P.two_dx, vor,
                                                                 stats, nan);
}

void launch_diag(const lbl_ctx* c, const float* mac, int member, double* red, cudaStream_t s) {
    const int m0 = member < 0 ? 0 : member, m1 = member < 0 ? c->P.M : member + 1;
    cudaMemsetAsync(red, 0, 3 * sizeof(double), s);
    diag_kernel<<<(c->P.nxy + 255) / 256, 256, 0, s>>>(mac, c->P.nx, c->P.ny, m0, m1, double(c->P.dx), red);
}

// the cells the RMSE covers: the whole grid, or a y-slab's own rows (not its halos)
void rmse_cells(const lbl_ctx* c, int* ij0, int* n) {
    *ij0 = c->slab_ny ? c->slab_halo * c->P.nx : 0;
    *n = c->slab_ny ? (c->P.ny - 2 * c->slab_halo) * c->P.nx : c->P.nxy;
}

void launch_rmse(const lbl_ctx* c, const float* mac, const float* ut, const float* vt, double* red, cudaStream_t s) {
    int ij0, n;
    rmse_cells(c, &ij0, &n);
    cudaMemsetAsync(red, 0, sizeof(double), s);
    rmse_kernel<<<(n + 255) / 256, 256, 0, s>>>(mac, c->P.nxy, c->P.M, ut, vt, red, ij0, n);
}

// red[1] = sqrt(red[0] / n), the RMSE the host would form (IEEE division and square root)
__global__ void rmse_finish_kernel(double* red, int n) { red[1] = sqrt(red[0] / double(n)); }
void launch_rmse_finish(const lbl_ctx* c, double* red, cudaStream_t s) {
    int ij0, n;
    rmse_cells(c, &ij0, &n);
    rmse_finish_kernel<<<1, 1, 0, s>>>(red, n);
}

}  // namespace lbl
