// closure.cu -- data and training for the learned eddy-viscosity closure (closure.h).
//
//   lbl_closure_generate  runs the engine on a fine grid, box-filters every snapshot
//                         onto a grid `filter` times coarser and turns it into
//                         (features, target) samples: the target is the Smagorinsky
//                         multiplier that matches the filtered subgrid stress,
//                         m* = -(tau_d : S) / (2 S:S) / ((Cs dx)^2 |S|), in [0, 8]
//   lbl_closure_grad      loss and gradient over a sample set (fused forward/backward)
//   lbl_closure_train     Adam on random minibatches with the same fused kernel
//
// The network keeps FP32 master parameters and computes with their BF16 copies under
// the operand contract of closure.h (FP16 matrix operands, FP32 sums).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "closure.h"
#include "lbl_internal.h"

#define CLOSURE_CK(call)                              \
    do {                                              \
        if ((call) != cudaSuccess) return LBL_ERR_CUDA; \
    } while (0)

namespace lbl {
namespace {

void set_err(char* err, size_t cap, const std::string& msg) {
    if (err && cap > 0) {
        const size_t n = std::min(cap - 1, msg.size());
        std::memcpy(err, msg.data(), n);
        err[n] = '\0';
    }
}

// ---------------------------------------------------------------------------
// data: F x F box filter of (u, v, uu, uv, vv) of one member's fine macros
// ---------------------------------------------------------------------------
__global__ void box_filter_kernel(const float* __restrict__ mac, int nxf, int nyf, int F, float* __restrict__ out,
                                  int nxc, int nyc) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nxc * nyc) return;
    const int I = c % nxc, J = c / nxc;
    const size_t nf = size_t(nxf) * nyf;
    const float* u = mac + nf;
    const float* v = mac + 2 * nf;
    double su = 0, sv = 0, suu = 0, suv = 0, svv = 0;
    for (int b = 0; b < F; b++)
        for (int a = 0; a < F; a++) {
            const size_t ij = size_t(I * F + a) + size_t(nxf) * (J * F + b);
            const double uu = u[ij], vv = v[ij];
            su += uu; sv += vv; suu += uu * uu; suv += uu * vv; svv += vv * vv;
        }
    const double inv = 1.0 / (double(F) * F);
    const size_t nc = size_t(nxc) * nyc;
    out[c] = float(su * inv);
    out[nc + c] = float(sv * inv);
    out[2 * nc + c] = float(suu * inv);
    out[3 * nc + c] = float(suv * inv);
    out[4 * nc + c] = float(svv * inv);
}

// features and Smagorinsky-multiplier target on the coarse grid (spacing h)
__global__ void closure_sample_kernel(const float* __restrict__ filt, int nxc, int nyc, float h, float cs,
                                      ClosureScales sc, float* __restrict__ feat, float* __restrict__ target) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nxc * nyc) return;
    const int I = c % nxc, J = c / nxc;
    const size_t nc = size_t(nxc) * nyc;
    const float* ub = filt;
    const float* vb = filt + nc;
    auto at = [&](const float* a, int i, int j) { return a[((i + nxc) % nxc) + size_t(nxc) * ((j + nyc) % nyc)]; };
    const float inv2h = 1.f / (2.f * h);
    const float ux = (at(ub, I + 1, J) - at(ub, I - 1, J)) * inv2h;
    const float uy = (at(ub, I, J + 1) - at(ub, I, J - 1)) * inv2h;
    const float vx = (at(vb, I + 1, J) - at(vb, I - 1, J)) * inv2h;
    const float vy = (at(vb, I, J + 1) - at(vb, I, J - 1)) * inv2h;
    float x[kMlpIn];
    const float smag = closure_features(ux, uy, vx, vy, sc, x);
#pragma unroll
    for (int k = 0; k < kMlpIn; k++) feat[size_t(c) * kMlpIn + k] = x[k];
    // subgrid stress of the filter and its deviatoric part
    const float u = ub[c], v = vb[c];
    const float t11 = filt[2 * nc + c] - u * u, t12 = filt[3 * nc + c] - u * v, t22 = filt[4 * nc + c] - v * v;
    const float tr = 0.5f * (t11 + t22);
    const float s11 = ux, s22 = vy, s12 = 0.5f * (uy + vx);
    const float ss = s11 * s11 + 2.f * s12 * s12 + s22 * s22;
    const float tds = (t11 - tr) * s11 + 2.f * t12 * s12 + (t22 - tr) * s22;
    const float base = cs * cs * sc.dx * sc.dx * smag;
    float m = 1.f;  // no strain: keep Smagorinsky
    if (ss > 1e-12f && base > 0.f) m = -tds / (2.f * ss) / base;
    target[c] = fminf(fmaxf(m, 0.f), 8.f);
}

// ---------------------------------------------------------------------------
// training: fused forward + backward.  A warp takes 32 samples (one per lane),
// stages their activations and deltas in shared memory, and lane l then sums the
// gradient of hidden unit l over the 32 samples (row l of dW1, dW2, and db1, db2,
// dW3); per-warp sums go to the global gradient with one atomic per parameter.
// ---------------------------------------------------------------------------
constexpr int kTrainWarps = 4;
struct Stage {  // per warp: 32 samples
    float x[32][kMlpIn];
    float a1[32][kMlpHid + 1];
    float d1[32][kMlpHid + 1];
    float a2[32][kMlpHid + 1];
    float d2[32][kMlpHid + 1];
    float dz[32];
};

__device__ __forceinline__ float gelu_grad(float x) {
    const float k = 0.7978845608f, x2 = x * x;
    const float t = tanhf(k * (x + 0.044715f * x * x2));
    return 0.5f * (1.f + t) + 0.5f * x * (1.f - t * t) * k * (1.f + 3.f * 0.044715f * x2);
}

__device__ __forceinline__ uint32_t hash32(uint64_t a) {
    a ^= a >> 33; a *= 0xff51afd7ed558ccdull; a ^= a >> 33; a *= 0xc4ceb9fe1a85ec53ull; a ^= a >> 33;
    return uint32_t(a);
}

// samples: idx == nullptr -> all n in order; else idx_seed != 0 draws batch random indices
__global__ void __launch_bounds__(32 * kTrainWarps) mlp_grad_kernel(const __nv_bfloat16* __restrict__ pw,
                                                                   const float* __restrict__ feat,
                                                                   const float* __restrict__ tgt, size_t n,
                                                                   int batch, uint64_t idx_seed,
                                                                   float* __restrict__ grad, float* __restrict__ loss) {
    extern __shared__ float smem[];
    float* p = smem;                                             // parameters as float
    Stage* st = reinterpret_cast<Stage*>(smem + ((kMlpParams + 3) & ~3));
    for (int k = threadIdx.x; k < kMlpParams; k += blockDim.x) p[k] = param_value(pw, k);
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    Stage& S = st[warp];
    float gW1[kMlpIn] = {0}, gW2[kMlpHid] = {0};
    float gb1 = 0, gb2 = 0, gW3 = 0, gb3 = 0, lsum = 0;
    const int per_pass = gridDim.x * kTrainWarps * 32;
    for (int base = (blockIdx.x * kTrainWarps + warp) * 32; base < batch; base += per_pass) {
        const int s = base + lane;
        const bool valid = s < batch;
        size_t sample = 0;
        if (valid) sample = idx_seed ? size_t(hash32(idx_seed * 0x9E3779B97F4A7C15ull + uint64_t(s)) % n) : size_t(s);
        float x[kMlpIn], h1[kMlpHid], a1[kMlpHid], h2[kMlpHid];
#pragma unroll
        for (int k = 0; k < kMlpIn; k++) x[k] = valid ? f16_round(feat[sample * kMlpIn + k]) : 0.f;
#pragma unroll
        for (int i = 0; i < kMlpHid; i++) {
            float h = p[kMlpB1 + i];
#pragma unroll
            for (int k = 0; k < kMlpIn; k++) h = fmaf(p[kMlpW1 + i * kMlpIn + k], x[k], h);
            h1[i] = h;
            a1[i] = f16_round(mlp_gelu(h));  // the layer-2 operand (gradient passes straight through)
        }
        float z = p[kMlpB3];
#pragma unroll 4
        for (int i = 0; i < kMlpHid; i++) {
            float h = p[kMlpB2 + i];
#pragma unroll
            for (int j = 0; j < kMlpHid; j++) h = fmaf(p[kMlpW2 + i * kMlpHid + j], a1[j], h);
            h2[i] = h;
            z = fmaf(p[kMlpW3 + i], f16_round(mlp_gelu(h)), z);  // the layer-3 operand
        }
        const float y = mlp_softplus(z);
        const float t = valid ? tgt[sample] : 0.f;
        const float err = valid ? (y - t) : 0.f;
        lsum += err * err;
        // d(mean squared error)/dz
        const float dz = valid ? 2.f * err / float(batch) * (1.f / (1.f + expf(-z))) : 0.f;
        float d2[kMlpHid];
#pragma unroll
        for (int i = 0; i < kMlpHid; i++) d2[i] = dz * p[kMlpW3 + i] * gelu_grad(h2[i]);
        // stage: x, a1, d1 (from d2), a2, d2, dz
#pragma unroll
        for (int k = 0; k < kMlpIn; k++) S.x[lane][k] = x[k];
#pragma unroll
        for (int j = 0; j < kMlpHid; j++) {
            float da = 0.f;
#pragma unroll
            for (int i = 0; i < kMlpHid; i++) da = fmaf(p[kMlpW2 + i * kMlpHid + j], d2[i], da);
            S.a1[lane][j] = a1[j];
            S.d1[lane][j] = da * gelu_grad(h1[j]);
        }
#pragma unroll
        for (int i = 0; i < kMlpHid; i++) {
            S.a2[lane][i] = f16_round(mlp_gelu(h2[i]));
            S.d2[lane][i] = d2[i];
        }
        S.dz[lane] = dz;
        __syncwarp();
        // lane l: hidden unit l over the warp's 32 samples
        for (int q = 0; q < 32; q++) {
            const float d1l = S.d1[q][lane], d2l = S.d2[q][lane];
#pragma unroll
            for (int k = 0; k < kMlpIn; k++) gW1[k] = fmaf(d1l, S.x[q][k], gW1[k]);
            gb1 += d1l;
#pragma unroll
            for (int j = 0; j < kMlpHid; j++) gW2[j] = fmaf(d2l, S.a1[q][j], gW2[j]);
            gb2 += d2l;
            gW3 = fmaf(S.dz[q], S.a2[q][lane], gW3);
            gb3 += S.dz[q];
        }
        __syncwarp();
    }
#pragma unroll
    for (int k = 0; k < kMlpIn; k++) atomicAdd(grad + kMlpW1 + lane * kMlpIn + k, gW1[k]);
    atomicAdd(grad + kMlpB1 + lane, gb1);
#pragma unroll
    for (int j = 0; j < kMlpHid; j++) atomicAdd(grad + kMlpW2 + lane * kMlpHid + j, gW2[j]);
    atomicAdd(grad + kMlpB2 + lane, gb2);
    atomicAdd(grad + kMlpW3 + lane, gW3);
    if (lane == 0) atomicAdd(grad + kMlpB3, gb3);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
    if (lane == 0) atomicAdd(loss, lsum);
}

// Adam on the FP32 master parameters; refreshes their BF16 copy
__global__ void adam_kernel(float* __restrict__ w, __nv_bfloat16* __restrict__ wb, const float* __restrict__ g,
                            float* __restrict__ m, float* __restrict__ v, float lr, float b1, float b2, float eps,
                            float c1, float c2) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= kMlpParams) return;
    const float gk = g[k];
    const float mk = b1 * m[k] + (1.f - b1) * gk;
    const float vk = b2 * v[k] + (1.f - b2) * gk * gk;
    m[k] = mk;
    v[k] = vk;
    w[k] -= lr * (mk / c1) / (sqrtf(vk / c2) + eps);
    wb[k] = __float2bfloat16_rn(w[k]);
}

__global__ void to_bf16_kernel(const float* __restrict__ w, __nv_bfloat16* __restrict__ wb, int n) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) wb[k] = __float2bfloat16_rn(w[k]);
}

size_t grad_smem() { return sizeof(float) * ((kMlpParams + 3) & ~3) + sizeof(Stage) * kTrainWarps; }

// Xavier-uniform start; the output bias makes softplus(z) = 1 (plain Smagorinsky)
void init_params(uint64_t seed, float* w) {
    std::mt19937_64 g(seed);
    auto fill = [&](int off, int n, int fan_in, int fan_out) {
        const double a = std::sqrt(6.0 / (fan_in + fan_out));
        std::uniform_real_distribution<double> d(-a, a);
        for (int k = 0; k < n; k++) w[off + k] = float(d(g));
    };
    fill(kMlpW1, kMlpHid * kMlpIn, kMlpIn, kMlpHid);
    fill(kMlpW2, kMlpHid * kMlpHid, kMlpHid, kMlpHid);
    fill(kMlpW3, kMlpHid, kMlpHid, 1);
    for (int k = 0; k < kMlpHid; k++) { w[kMlpB1 + k] = 0.f; w[kMlpB2 + k] = 0.f; }
    for (int k = 0; k < kMlpHid; k++) w[kMlpW3 + k] *= 0.1f;
    w[kMlpB3] = float(std::log(std::expm1(1.0)));
}

// one multiplier per feature row: path 0 = the warp tensor-core form of the
// stream-collide, 1 = the per-thread FP32 form (mlp_forward).  Rows past n run
// with zero features so that every warp is complete.
__global__ void __launch_bounds__(128) closure_infer_kernel(const uint32_t* __restrict__ pack,
                                                            const __nv_bfloat16* __restrict__ pw,
                                                            const float* __restrict__ feat, size_t n, int path,
                                                            float* __restrict__ out) {
    __shared__ __align__(16) uint32_t s_pack[kPackWords];
    __shared__ __align__(16) uint32_t s_stage[4][kStageWords];
    for (int k = threadIdx.x; k < kPackWords; k += blockDim.x) s_pack[k] = pack[k];
    __syncthreads();
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    float x[kMlpIn];
#pragma unroll
    for (int k = 0; k < kMlpIn; k++) x[k] = i < n ? feat[i * kMlpIn + k] : 0.f;
    const float m = path == 0 ? mlp_forward_warp(s_pack, s_stage[threadIdx.x >> 5], x) : mlp_forward(pw, x);
    if (i < n) out[i] = m;
}

struct DevBuf {
    void* p = nullptr;
    ~DevBuf() { cudaFree(p); }
};

}  // namespace
}  // namespace lbl

using namespace lbl;

extern "C" {

int lbl_closure_generate(const lbl_config* fine, int filter, int spinup, int n_snapshots, int spacing, int device,
                         float* features, float* targets, size_t capacity, size_t* n_samples, char* err,
                         size_t err_cap) {
    if (!fine || !features || !targets || !n_samples || filter < 2 || n_snapshots < 1 || spacing < 1 || spinup < 0) {
        set_err(err, err_cap, "bad argument");
        return LBL_ERR_ARG;
    }
    if (fine->nx % filter || fine->ny % filter) { set_err(err, err_cap, "filter must divide the grid"); return LBL_ERR_ARG; }
    const int nxc = fine->nx / filter, nyc = fine->ny / filter;
    const size_t nc = size_t(nxc) * nyc;
    const size_t need = nc * size_t(fine->n_ens) * n_snapshots;
    if (capacity < need) { set_err(err, err_cap, "capacity below n_ens * snapshots * coarse cells"); return LBL_ERR_ARG; }
    lbl_config cfg = *fine;
    cfg.mode = LBL_MODE_NATURE;
    lbl_ctx* ctx = nullptr;
    int rc = lbl_create(&cfg, device, &ctx);
    if (rc == LBL_OK) rc = lbl_init(ctx, 0);
    int t = 0;
    if (rc == LBL_OK && spinup > 0) rc = lbl_update(ctx, t, spinup);
    t += spinup;
    if (rc != LBL_OK) {
        set_err(err, err_cap, ctx ? lbl_last_error(ctx) : "lbl_create failed");
        lbl_destroy(ctx);
        return rc;
    }
    // the coarse grid's own spacing (the engine's dx for ny/filter points) scales the
    // features; the filtered field's cells are filter fine cells apart
    const float h = float(filter) * ctx->P.dx;
    cudaStream_t st = ctx->stream;
    ClosureScales sc{float(cfg.h_ref / double(nyc - 1)), ctx->P.nu, float(cfg.h_ref / 255.0)};
    DevBuf filt, df, dt;
    cudaError_t ce = cudaMalloc(&filt.p, sizeof(float) * 5 * nc);
    if (ce == cudaSuccess) ce = cudaMalloc(&df.p, sizeof(float) * kMlpIn * nc);
    if (ce == cudaSuccess) ce = cudaMalloc(&dt.p, sizeof(float) * nc);
    size_t at = 0;
    for (int s = 0; s < n_snapshots && ce == cudaSuccess && rc == LBL_OK; s++) {
        rc = lbl_update(ctx, t, spacing);
        t += spacing;
        if (rc != LBL_OK) break;
        for (int m = 0; m < cfg.n_ens && ce == cudaSuccess; m++) {
            const float* mac = ctx->mac[ctx->cur] + size_t(m) * 3 * ctx->P.nxy;
            box_filter_kernel<<<int((nc + 255) / 256), 256, 0, st>>>(mac, cfg.nx, cfg.ny, filter,
                                                                      static_cast<float*>(filt.p), nxc, nyc);
            closure_sample_kernel<<<int((nc + 255) / 256), 256, 0, st>>>(static_cast<float*>(filt.p), nxc, nyc, h,
                                                                          float(cfg.cs), sc, static_cast<float*>(df.p),
                                                                          static_cast<float*>(dt.p));
            ce = cudaMemcpyAsync(features + at * kMlpIn, df.p, sizeof(float) * kMlpIn * nc, cudaMemcpyDeviceToHost, st);
            if (ce == cudaSuccess)
                ce = cudaMemcpyAsync(targets + at, dt.p, sizeof(float) * nc, cudaMemcpyDeviceToHost, st);
            if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
            at += nc;
        }
    }
    if (rc == LBL_OK && ce != cudaSuccess) { set_err(err, err_cap, cudaGetErrorString(ce)); rc = LBL_ERR_CUDA; }
    if (rc != LBL_OK && ce == cudaSuccess) set_err(err, err_cap, lbl_last_error(ctx));
    lbl_destroy(ctx);
    *n_samples = at;
    return rc;
}

int lbl_closure_grad(const float* params, const float* features, const float* targets, size_t n, int device,
                     float* grad, float* loss) {
    if (!params || !features || !targets || !grad || n == 0 || n > (size_t(1) << 31)) return LBL_ERR_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return LBL_ERR_CUDA;
    DevBuf w, wb, f, t, g, l;
    if (cudaMalloc(&w.p, sizeof(float) * kMlpParams) != cudaSuccess ||
        cudaMalloc(&wb.p, sizeof(__nv_bfloat16) * kMlpParams) != cudaSuccess ||
        cudaMalloc(&f.p, sizeof(float) * kMlpIn * n) != cudaSuccess || cudaMalloc(&t.p, sizeof(float) * n) != cudaSuccess ||
        cudaMalloc(&g.p, sizeof(float) * kMlpParams) != cudaSuccess || cudaMalloc(&l.p, sizeof(float)) != cudaSuccess)
        return LBL_ERR_CUDA;
    CLOSURE_CK(cudaMemcpy(w.p, params, sizeof(float) * kMlpParams, cudaMemcpyHostToDevice));
    CLOSURE_CK(cudaMemcpy(f.p, features, sizeof(float) * kMlpIn * n, cudaMemcpyHostToDevice));
    CLOSURE_CK(cudaMemcpy(t.p, targets, sizeof(float) * n, cudaMemcpyHostToDevice));
    CLOSURE_CK(cudaMemset(g.p, 0, sizeof(float) * kMlpParams));
    CLOSURE_CK(cudaMemset(l.p, 0, sizeof(float)));
    to_bf16_kernel<<<(kMlpParams + 255) / 256, 256>>>(static_cast<float*>(w.p), static_cast<__nv_bfloat16*>(wb.p),
                                                      kMlpParams);
    CLOSURE_CK(cudaFuncSetAttribute(mlp_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(grad_smem())));
    const int blocks = int(std::min<size_t>(148 * 4, (n + 32 * kTrainWarps - 1) / (32 * kTrainWarps)));
    mlp_grad_kernel<<<blocks, 32 * kTrainWarps, grad_smem()>>>(static_cast<__nv_bfloat16*>(wb.p),
                                                                static_cast<float*>(f.p), static_cast<float*>(t.p), n,
                                                                int(n), 0, static_cast<float*>(g.p),
                                                                static_cast<float*>(l.p));
    if (cudaDeviceSynchronize() != cudaSuccess) return LBL_ERR_CUDA;
    CLOSURE_CK(cudaMemcpy(grad, g.p, sizeof(float) * kMlpParams, cudaMemcpyDeviceToHost));
    if (loss) {
        float ls = 0;
        CLOSURE_CK(cudaMemcpy(&ls, l.p, sizeof(float), cudaMemcpyDeviceToHost));
        *loss = ls / float(n);
    }
    return cudaGetLastError() == cudaSuccess ? LBL_OK : LBL_ERR_CUDA;
}

int lbl_closure_train(const float* features, const float* targets, size_t n, int iters, int batch, float lr,
                      uint64_t seed, int device, const float* init, float* params, float* loss_curve) {
    if (!features || !targets || !params || n == 0 || iters < 1 || batch < 32 || !(lr > 0)) return LBL_ERR_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return LBL_ERR_CUDA;
    std::vector<float> w0(kMlpParams);
    if (init) std::copy(init, init + kMlpParams, w0.begin());
    else init_params(seed, w0.data());
    DevBuf w, wb, f, t, g, m, v, l;
    if (cudaMalloc(&w.p, sizeof(float) * kMlpParams) != cudaSuccess ||
        cudaMalloc(&wb.p, sizeof(__nv_bfloat16) * kMlpParams) != cudaSuccess ||
        cudaMalloc(&f.p, sizeof(float) * kMlpIn * n) != cudaSuccess || cudaMalloc(&t.p, sizeof(float) * n) != cudaSuccess ||
        cudaMalloc(&g.p, sizeof(float) * kMlpParams) != cudaSuccess ||
        cudaMalloc(&m.p, sizeof(float) * kMlpParams) != cudaSuccess ||
        cudaMalloc(&v.p, sizeof(float) * kMlpParams) != cudaSuccess ||
        cudaMalloc(&l.p, sizeof(float) * iters) != cudaSuccess)
        return LBL_ERR_CUDA;
    CLOSURE_CK(cudaMemcpy(w.p, w0.data(), sizeof(float) * kMlpParams, cudaMemcpyHostToDevice));
    CLOSURE_CK(cudaMemcpy(f.p, features, sizeof(float) * kMlpIn * n, cudaMemcpyHostToDevice));
    CLOSURE_CK(cudaMemcpy(t.p, targets, sizeof(float) * n, cudaMemcpyHostToDevice));
    CLOSURE_CK(cudaMemset(m.p, 0, sizeof(float) * kMlpParams));
    CLOSURE_CK(cudaMemset(v.p, 0, sizeof(float) * kMlpParams));
    CLOSURE_CK(cudaMemset(l.p, 0, sizeof(float) * iters));
    to_bf16_kernel<<<(kMlpParams + 255) / 256, 256>>>(static_cast<float*>(w.p), static_cast<__nv_bfloat16*>(wb.p),
                                                      kMlpParams);
    CLOSURE_CK(cudaFuncSetAttribute(mlp_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(grad_smem())));
    const int blocks = int(std::min<int>(148 * 4, (batch + 32 * kTrainWarps - 1) / (32 * kTrainWarps)));
    const float b1 = 0.9f, b2 = 0.999f;
    double p1 = 1, p2 = 1;
    for (int it = 0; it < iters; it++) {
        CLOSURE_CK(cudaMemsetAsync(g.p, 0, sizeof(float) * kMlpParams));
        mlp_grad_kernel<<<blocks, 32 * kTrainWarps, grad_smem()>>>(
            static_cast<__nv_bfloat16*>(wb.p), static_cast<float*>(f.p), static_cast<float*>(t.p), n, batch,
            seed * 1000003ull + uint64_t(it) + 1, static_cast<float*>(g.p), static_cast<float*>(l.p) + it);
        p1 *= b1;
        p2 *= b2;
        adam_kernel<<<(kMlpParams + 255) / 256, 256>>>(static_cast<float*>(w.p), static_cast<__nv_bfloat16*>(wb.p),
                                                       static_cast<float*>(g.p), static_cast<float*>(m.p),
                                                       static_cast<float*>(v.p), lr, b1, b2, 1e-8f,
                                                       float(1 - p1), float(1 - p2));
    }
    if (cudaDeviceSynchronize() != cudaSuccess || cudaGetLastError() != cudaSuccess) return LBL_ERR_CUDA;
    CLOSURE_CK(cudaMemcpy(params, w.p, sizeof(float) * kMlpParams, cudaMemcpyDeviceToHost));
    if (loss_curve) {
        CLOSURE_CK(cudaMemcpy(loss_curve, l.p, sizeof(float) * iters, cudaMemcpyDeviceToHost));
        for (int it = 0; it < iters; it++) loss_curve[it] /= float(batch);
    }
    return LBL_OK;
}

}  // extern "C"

extern "C" {

int lbl_set_closure(lbl_ctx* ctx, const float* params, double nu_ref, double dx_ref) {
    if (!ctx) return LBL_ERR_ARG;
    if (cudaSetDevice(ctx->device) != cudaSuccess) return LBL_ERR_CUDA;
    if (params) {
        if (ctx->slab_ny) {
            ctx->err = "a y-slab runs the Smagorinsky closure only";
            return LBL_ERR_UNSUPPORTED;
        }
        if (ctx->P.nx % 32 != 0) {  // whole warps of cells
            ctx->err = "the learned closure needs nx a multiple of 32";
            return LBL_ERR_UNSUPPORTED;
        }
        if (ctx->use_tma) {
            ctx->err = "the learned closure runs in the direct-load stream-collide (lbm_variant AUTO or DIRECT)";
            return LBL_ERR_UNSUPPORTED;
        }
        for (int k = 0; k < kMlpParams; k++)
            if (!std::isfinite(params[k])) { ctx->err = "closure parameters must be finite"; return LBL_ERR_ARG; }
    }
    // graphs captured with the other stream-collide variant are rebuilt on demand
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess || cudaStreamSynchronize(ctx->side) != cudaSuccess)
        return LBL_ERR_CUDA;
    for (auto& g : ctx->graphs) cudaGraphExecDestroy(g.second);
    ctx->graphs.clear();
    ctx->ty_tuned = 0;  // a strip height tuned for the other variant does not carry over
    if (!params) {
        ctx->closure = false;
        ctx->ty_default = lbm_strip_rows(ctx);
        return LBL_OK;
    }
    std::vector<uint32_t> pack(kPackWords);
    closure_pack(params, pack.data());
    if (!ctx->d_closure && cudaMalloc(&ctx->d_closure, sizeof(uint32_t) * kPackWords) != cudaSuccess) {
        ctx->err = "cudaMalloc(closure parameters) failed";
        return LBL_ERR_CUDA;
    }
    if (cudaMemcpy(ctx->d_closure, pack.data(), sizeof(uint32_t) * kPackWords, cudaMemcpyHostToDevice) != cudaSuccess)
        return LBL_ERR_CUDA;
    ctx->closure_sc.dx = ctx->P.dx;
    ctx->closure_sc.nu_ref = nu_ref > 0 ? float(nu_ref) : ctx->P.nu;
    ctx->closure_sc.dx_ref = dx_ref > 0 ? float(dx_ref) : float(ctx->cfg.h_ref / 255.0);
    ctx->closure = true;
    ctx->ty_default = lbm_strip_rows(ctx);
    ctx->ty_held = ctx->closure_every > 1 ? lbm_strip_rows_held(ctx) : 0;
    return LBL_OK;
}

int lbl_set_closure_refresh(lbl_ctx* ctx, int steps) {
    if (!ctx) return LBL_ERR_ARG;
    if (steps < 1 || steps > 1000) {
        ctx->err = "the closure refresh interval must lie in [1, 1000] steps";
        return LBL_ERR_ARG;
    }
    if (steps > 1 && ctx->P.nx > 1024) {
        ctx->err = "holding the closure multiplier between evaluations needs nx <= 1024";
        return LBL_ERR_UNSUPPORTED;
    }
    if (cudaSetDevice(ctx->device) != cudaSuccess) return LBL_ERR_CUDA;
    if (cudaStreamSynchronize(ctx->stream) != cudaSuccess || cudaStreamSynchronize(ctx->side) != cudaSuccess)
        return LBL_ERR_CUDA;
    for (auto& g : ctx->graphs) cudaGraphExecDestroy(g.second);  // captured with the old schedule
    ctx->graphs.clear();
    if (steps > 1 && !ctx->d_mclos) {
        const cudaError_t e = cudaMalloc(&ctx->d_mclos, sizeof(float) * size_t(ctx->P.M) * ctx->P.nxy);
        if (e != cudaSuccess) {
            ctx->err = std::string("cudaMalloc(closure multipliers): ") + cudaGetErrorString(e);
            cudaGetLastError();
            return e == cudaErrorMemoryAllocation ? LBL_ERR_NOMEM : LBL_ERR_CUDA;
        }
    }
    if (steps == 1 && ctx->d_mclos) {
        cudaFree(ctx->d_mclos);
        ctx->d_mclos = nullptr;
    }
    ctx->closure_every = steps;
    ctx->ty_held = steps > 1 ? lbm_strip_rows_held(ctx) : 0;
    return LBL_OK;
}

int lbl_closure_infer(const float* params, const float* features, size_t n, int path, int device, float* out) {
    if (!params || !features || !out || n == 0 || (path != 0 && path != 1)) return LBL_ERR_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return LBL_ERR_CUDA;
    std::vector<uint32_t> pack(kPackWords);
    closure_pack(params, pack.data());
    DevBuf w, wb, pk, f, o;
    if (cudaMalloc(&w.p, sizeof(float) * kMlpParams) != cudaSuccess ||
        cudaMalloc(&wb.p, sizeof(__nv_bfloat16) * kMlpParams) != cudaSuccess ||
        cudaMalloc(&pk.p, sizeof(uint32_t) * kPackWords) != cudaSuccess ||
        cudaMalloc(&f.p, sizeof(float) * kMlpIn * n) != cudaSuccess || cudaMalloc(&o.p, sizeof(float) * n) != cudaSuccess)
        return LBL_ERR_CUDA;
    CLOSURE_CK(cudaMemcpy(w.p, params, sizeof(float) * kMlpParams, cudaMemcpyHostToDevice));
    CLOSURE_CK(cudaMemcpy(pk.p, pack.data(), sizeof(uint32_t) * kPackWords, cudaMemcpyHostToDevice));
    CLOSURE_CK(cudaMemcpy(f.p, features, sizeof(float) * kMlpIn * n, cudaMemcpyHostToDevice));
    to_bf16_kernel<<<(kMlpParams + 255) / 256, 256>>>(static_cast<float*>(w.p), static_cast<__nv_bfloat16*>(wb.p),
                                                      kMlpParams);
    closure_infer_kernel<<<int((n + 127) / 128), 128>>>(static_cast<uint32_t*>(pk.p),
                                                          static_cast<__nv_bfloat16*>(wb.p),
                                                          static_cast<float*>(f.p), n, path, static_cast<float*>(o.p));
    if (cudaDeviceSynchronize() != cudaSuccess || cudaGetLastError() != cudaSuccess) return LBL_ERR_CUDA;
    return cudaMemcpy(out, o.p, sizeof(float) * n, cudaMemcpyDeviceToHost) == cudaSuccess ? LBL_OK : LBL_ERR_CUDA;
}

}  // extern "C"
