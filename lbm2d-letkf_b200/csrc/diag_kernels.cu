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

__global__ void rmse_kernel(const float* __restrict__ mac, int nxy, int M, const float* __restrict__ ut,
                            const float* __restrict__ vt, double* __restrict__ red) {
    const int ij = blockIdx.x * blockDim.x + threadIdx.x;
    double s = 0;
    if (ij < nxy) {
        const double du = field(mac, nxy, 0, M, 1, ij) - double(ut[ij]);
        const double dv = field(mac, nxy, 0, M, 2, ij) - double(vt[ij]);
        s = du * du + dv * dv;
    }
    block_add(s, red);
}

}  // namespace

void launch_diag(const lbl_ctx* c, const float* mac, int member, double* red, cudaStream_t s) {
    const int m0 = member < 0 ? 0 : member, m1 = member < 0 ? c->P.M : member + 1;
    cudaMemsetAsync(red, 0, 3 * sizeof(double), s);
    diag_kernel<<<(c->P.nxy + 255) / 256, 256, 0, s>>>(mac, c->P.nx, c->P.ny, m0, m1, double(c->P.dx), red);
}

void launch_rmse(const lbl_ctx* c, const float* mac, const float* ut, const float* vt, double* red, cudaStream_t s) {
    cudaMemsetAsync(red, 0, sizeof(double), s);
    rmse_kernel<<<(c->P.nxy + 255) / 256, 256, 0, s>>>(mac, c->P.nxy, c->P.M, ut, vt, red);
}

}  // namespace lbl
