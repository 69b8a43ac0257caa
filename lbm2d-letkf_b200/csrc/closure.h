// closure.h -- the learned eddy-viscosity closure shared by the stream-collide
// (inference) and the closure data/training kernels.
//
// A 6 -> 32 -> 32 -> 1 MLP (GELU hidden layers, softplus output, 1313 parameters)
// maps invariants of the resolved velocity gradient to a multiplier m >= 0 of the
// Smagorinsky viscosity: nu_t = m (Cs dx)^2 |S|, so m = 1 is the plain Smagorinsky
// closure the model falls back to.
//
// Arithmetic contract (the same in training and in the stream-collide): parameters
// are BF16 values.  The three matrix products run on FP16 tensor-core operands: the
// weights W1, W2, W3 and the first layer's bias (a weight on a constant input) are
// those BF16 values carried in FP16 (exact for |w| >= 2^-14), and the inputs -- the
// features and both hidden activations -- are rounded to FP16.  Every sum is
// accumulated in FP32; b2, b3 and softplus are FP32.  GELU is FP32 (tanhf) in
// training and in the per-thread form; the stream-collide evaluates it on pairs in
// FP16 arithmetic with the MUFU tanh (about 1e-3 relative).
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cstdint>
#include <cstring>

namespace lbl {

constexpr int kMlpIn = 6;
constexpr int kMlpHid = 32;
// parameter layout: W1[32][6], b1[32], W2[32][32], b2[32], W3[32], b3
constexpr int kMlpW1 = 0;
constexpr int kMlpB1 = kMlpW1 + kMlpHid * kMlpIn;
constexpr int kMlpW2 = kMlpB1 + kMlpHid;
constexpr int kMlpB2 = kMlpW2 + kMlpHid * kMlpHid;
constexpr int kMlpW3 = kMlpB2 + kMlpHid;
constexpr int kMlpB3 = kMlpW3 + kMlpHid;
constexpr int kMlpParams = kMlpB3 + 1;  // 1313

// Scales of the features: dx of the grid the closure runs on, the molecular
// viscosity as the reference rate, and the reference grid spacing of the training.
struct ClosureScales {
    float dx, nu_ref, dx_ref;
};

// The six inputs from the velocity gradient (ux = du/dx, uy = du/dy, ...):
//   x0 = log(1 + dx^2 |S| / nu_ref),  |S| = sqrt(2 S:S)
//   x1 = log(1 + dx^2 |W| / nu_ref),  |W| = sqrt(2 W:W)
//   x2 = (W:W - S:S) / (W:W + S:S)    strain / rotation balance
//   x3 = (S11 + S22) / sqrt(S:S)      divergence relative to strain
//   x4 = dx / dx_ref                  grid scale
//   x5 = asinh(dx^2 omega / nu_ref)   signed vorticity, omega = vx - uy
// Returns |S|.
__host__ __device__ inline float closure_features(float ux, float uy, float vx, float vy, const ClosureScales& c,
                                                  float* x) {
    const float s11 = ux, s22 = vy, s12 = 0.5f * (uy + vx), w12 = 0.5f * (uy - vx);
    const float ss = s11 * s11 + 2.f * s12 * s12 + s22 * s22;
    const float ww = 2.f * w12 * w12;
    const float smag = sqrtf(2.f * ss), wmag = sqrtf(2.f * ww);
    const float k = c.dx * c.dx / c.nu_ref;
    x[0] = log1pf(k * smag);
    x[1] = log1pf(k * wmag);
    x[2] = (ww - ss) / (ww + ss + 1e-30f);
    x[3] = (s11 + s22) / sqrtf(ss + 1e-30f);
    x[4] = c.dx / c.dx_ref;
    x[5] = asinhf(k * (vx - uy));
    return smag;
}

#ifdef __CUDACC__
// the hardware's approximate square root (sqrt.approx.f32)
__device__ __forceinline__ float closure_sqrt(float x) {
    float r;
    asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
// The same features with the hardware log / reciprocal / square root (a few ulp;
// the features are rounded to FP16 before use): the stream-collide's form.
__device__ __forceinline__ float closure_features_fast(float ux, float uy, float vx, float vy,
                                                       const ClosureScales& c, float* x) {
    const float s11 = ux, s22 = vy, s12 = 0.5f * (uy + vx), w12 = 0.5f * (uy - vx);
    const float ss = fmaf(s11, s11, fmaf(2.f * s12, s12, s22 * s22));
    const float ww = 2.f * w12 * w12;
    const float smag = closure_sqrt(2.f * ss), wmag = closure_sqrt(2.f * ww);
    const float k = c.dx * c.dx / c.nu_ref;
    const float y = k * (vx - uy);
    x[0] = __logf(fmaf(k, smag, 1.f));
    x[1] = __logf(fmaf(k, wmag, 1.f));
    x[2] = __fdividef(ww - ss, ww + ss + 1e-30f);
    x[3] = (s11 + s22) * rsqrtf(ss + 1e-30f);
    x[4] = c.dx / c.dx_ref;
    x[5] = copysignf(__logf(fabsf(y) + closure_sqrt(fmaf(y, y, 1.f))), y);
    return smag;
}
#endif

// GELU, tanh form: 0.5 x (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3)))
constexpr float kGeluK = 0.7978845608f, kGeluC = 0.044715f;
__host__ __device__ inline float mlp_gelu(float x) {
    const float t = tanhf(kGeluK * (x + kGeluC * x * x * x));
    return 0.5f * x * (1.f + t);
}
__host__ __device__ inline float mlp_softplus(float z) { return z > 20.f ? z : log1pf(expf(z)); }
__host__ __device__ inline float f16_round(float x) { return __half2float(__float2half_rn(x)); }
// a parameter as the network uses it: BF16, and for W1, b1, W2 and W3 also FP16
__host__ __device__ inline float param_value(const __nv_bfloat16* p, int k) {
    const float w = __bfloat162float(p[k]);
    return (k < kMlpB2 || (k >= kMlpW3 && k < kMlpB3)) ? f16_round(w) : w;
}

// forward pass under the contract above (one cell): the Smagorinsky multiplier
__device__ inline float mlp_forward(const __nv_bfloat16* __restrict__ p, const float* x_in) {
    float x[kMlpIn], a1[kMlpHid];
#pragma unroll
    for (int k = 0; k < kMlpIn; k++) x[k] = f16_round(x_in[k]);
#pragma unroll 4
    for (int i = 0; i < kMlpHid; i++) {
        float h = param_value(p, kMlpB1 + i);
#pragma unroll
        for (int k = 0; k < kMlpIn; k++) h = fmaf(param_value(p, kMlpW1 + i * kMlpIn + k), x[k], h);
        a1[i] = f16_round(mlp_gelu(h));
    }
    float z = param_value(p, kMlpB3);
    for (int i = 0; i < kMlpHid; i++) {
        float h = param_value(p, kMlpB2 + i);
#pragma unroll
        for (int j = 0; j < kMlpHid; j++) h = fmaf(param_value(p, kMlpW2 + i * kMlpHid + j), a1[j], h);
        z = fmaf(param_value(p, kMlpW3 + i), f16_round(mlp_gelu(h)), z);
    }
    return mlp_softplus(z);
}

// ---------------------------------------------------------------------------
// Warp-cooperative inference on the tensor cores (mma.sync m16n8k16, FP16 in,
// FP32 accumulate): the 32 lanes of a warp hold 32 cells, the warp evaluates the
// network for all of them at once and returns each lane its own multiplier.
//
// The parameters are prepared once (closure_pack) in the fragment order of the
// m16n8k16 operands, so that lane t reads its share with vector loads:
//   u32 B1[32][4]   layer-1 B fragments (k = feature, n = hidden), one per n-tile, FP16x2;
//                   k = 6 is a constant 1 input whose weight is b1
//   u32 B2[32][16]  layer-2 B fragments, [n-tile][k-step][2], FP16x2 of W2 / 2
//   u32 B3[32][4]   layer-3 B fragments, [k-step][2]: W3 / 2 in all 8 columns, so
//                   that every lane's accumulators end up holding its rows' outputs
//                   (the halves take the doubled GELU of gelu2_f16x2)
//   f32 C[32][8]    b2 at the accumulator columns of lane t, [n-tile][2]
//   f32 b3
// ---------------------------------------------------------------------------
constexpr int kPackB1 = 0;                   // u32 offset of B1
constexpr int kPackB2 = 32 * 4;              // u32 offset of B2
constexpr int kPackB3f = kPackB2 + 32 * 16;  // u32 offset of B3
constexpr int kPackC = kPackB3f + 32 * 4;    // f32 offset of the per-lane b2
constexpr int kPackB3 = kPackC + 32 * 8;
constexpr int kPackWords = kPackB3 + 4;      // 1028 words = 4112 B
constexpr int kStageWords = 128;           // per-warp feature staging (32 lanes x 4 words)

// round-to-nearest-even BF16 value of a finite float (host side of the packing)
inline float bf16_value(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    u = ((u + 0x7FFFu + ((u >> 16) & 1u)) >> 16) << 16;
    float r;
    std::memcpy(&r, &u, 4);
    return r;
}
// FP16 bits of scale times the BF16 value of f (a matrix weight as the tensor cores
// take it; scale is 1 or the exact 1/2 that undoes the doubled GELU of the inputs)
inline uint32_t weight_bits(float f, float scale = 1.f) {
    const __half h = __float2half_rn(scale * bf16_value(f));
    uint16_t b;
    std::memcpy(&b, &h, 2);
    return b;
}

// FP32 parameters (layout above) -> the fragment-ordered pack
inline void closure_pack(const float* w, uint32_t* out) {
    auto pk = [&](int lo, int hi) { return weight_bits(w[lo]) | (weight_bits(w[hi]) << 16); };
    auto pk_half = [&](int lo, int hi) { return weight_bits(w[lo], 0.5f) | (weight_bits(w[hi], 0.5f) << 16); };
    float* cf = reinterpret_cast<float*>(out);
    for (int t = 0; t < 32; t++) {
        const int g = t >> 2, c = t & 3;
        for (int nt = 0; nt < 4; nt++) {
            const int n = 8 * nt + g;  // hidden unit = the fragment's n column
            out[kPackB1 + t * 4 + nt] = (2 * c < kMlpIn) ? pk(kMlpW1 + n * kMlpIn + 2 * c, kMlpW1 + n * kMlpIn + 2 * c + 1)
                                                         : weight_bits(w[kMlpB1 + n]);  // k = 6, 7: (b1, 0)
            for (int ks = 0; ks < 2; ks++) {
                const int k0 = kMlpW2 + n * kMlpHid + 16 * ks + 2 * c;
                out[kPackB2 + t * 16 + (nt * 2 + ks) * 2 + 0] = pk_half(k0, k0 + 1);
                out[kPackB2 + t * 16 + (nt * 2 + ks) * 2 + 1] = pk_half(k0 + 8, k0 + 9);
            }
            for (int e = 0; e < 2; e++)  // accumulator column 8 nt + 2 c + e of lane t
                cf[kPackC + t * 8 + nt * 2 + e] = bf16_value(w[kMlpB2 + 8 * nt + 2 * c + e]);
        }
        for (int ks = 0; ks < 2; ks++) {
            const int k0 = kMlpW3 + 16 * ks + 2 * c;
            out[kPackB3f + t * 4 + ks * 2 + 0] = pk_half(k0, k0 + 1);
            out[kPackB3f + t * 4 + ks * 2 + 1] = pk_half(k0 + 8, k0 + 9);
        }
    }
    cf[kPackB3] = bf16_value(w[kMlpB3]);
    out[kPackB3 + 1] = out[kPackB3 + 2] = out[kPackB3 + 3] = 0u;
}

#ifdef __CUDACC__
__device__ __forceinline__ uint32_t pack_f16x2(float lo, float hi) {
    const __half2 v = __floats2half2_rn(lo, hi);  // .x (lo) is the low half
    return *reinterpret_cast<const uint32_t*>(&v);
}
__device__ __forceinline__ __half2 as_h2(uint32_t u) { return *reinterpret_cast<const __half2*>(&u); }
__device__ __forceinline__ uint32_t as_u32(__half2 h) { return *reinterpret_cast<const uint32_t*>(&h); }
// Twice the GELU of a pair, x (1 + tanh(...)), in FP16 arithmetic with the MUFU tanh
// (PTX tanh.approx.f16x2); the next layer's weights carry the 1/2 (exactly), which
// saves a multiply per pair, and doubling commutes with the FP16 rounding.  Past
// |x| = 256, x^2 overflows to inf, tanh gives +-1 and the result is 2x or 0, the
// function's own limits.
__device__ __forceinline__ uint32_t gelu2_f16x2(uint32_t xu) {
    const __half2 x = as_h2(xu);
    const __half2 inner = __hfma2(__hmul2(x, x), __float2half2_rn(kGeluK * kGeluC), __float2half2_rn(kGeluK));
    const uint32_t yu = as_u32(__hmul2(x, inner));
    uint32_t tu;
    asm("tanh.approx.f16x2 %0, %1;" : "=r"(tu) : "r"(yu));
    return as_u32(__hfma2(x, as_h2(tu), x));
}
// D += A (16x16, row) * B (16x8, col), FP16 operands, FP32 accumulators
__device__ __forceinline__ void mma_f16_16816(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                              uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// The warp's 32 lanes each bring the features of one cell; every lane gets back its
// cell's multiplier.  Rows of the m16 tiles are cells: tile mt row r = lane 16 mt + r.
// pk: closure_pack output (shared or global memory, 16-byte aligned); stage: this
// warp's kStageWords words of shared memory.  All 32 lanes must call it together.
__device__ __forceinline__ float mlp_forward_warp(const uint32_t* __restrict__ pk, uint32_t* __restrict__ stage,
                                                  const float* x) {
    const int lane = threadIdx.x & 31, g = lane >> 2, c = lane & 3;
    __syncwarp();
    reinterpret_cast<uint4*>(stage)[lane] =
        make_uint4(pack_f16x2(x[0], x[1]), pack_f16x2(x[2], x[3]), pack_f16x2(x[4], x[5]), 0x3C00u /* (1, 0) */);
    __syncwarp();
    uint32_t xa[2][2];
#pragma unroll
    for (int mt = 0; mt < 2; mt++) {
        xa[mt][0] = stage[(16 * mt + g) * 4 + c];
        xa[mt][1] = stage[(16 * mt + g + 8) * 4 + c];
    }
    const uint4* w1v = reinterpret_cast<const uint4*>(pk + kPackB1);
    const uint4* w2v = reinterpret_cast<const uint4*>(pk + kPackB2 + lane * 16);
    const uint4* w3v = reinterpret_cast<const uint4*>(pk + kPackB3f);
    const float2* b2v = reinterpret_cast<const float2*>(pk + kPackC + lane * 8);
    const float b3 = reinterpret_cast<const float*>(pk)[kPackB3];
    float z[2][4];
    // one m-tile (16 cells) at a time through the three layers keeps few registers live
#pragma unroll
    for (int mt = 0; mt < 2; mt++) {
        // layer 1 (K = 6 features + the constant 1 of the bias, of 16) and GELU in FP16
        // pairs: the accumulators of n-tiles 2ks, 2ks+1 are the A fragment of layer 2's
        // k-step ks
        const uint4 w1 = w1v[lane];
        const uint32_t w1f[4] = {w1.x, w1.y, w1.z, w1.w};
        uint32_t a2[2][4];
#pragma unroll
        for (int nt = 0; nt < 4; nt++) {
            float h[4] = {0.f, 0.f, 0.f, 0.f};
            mma_f16_16816(h, xa[mt][0], xa[mt][1], 0u, 0u, w1f[nt], 0u);
            a2[nt >> 1][2 * (nt & 1) + 0] = gelu2_f16x2(pack_f16x2(h[0], h[1]));
            a2[nt >> 1][2 * (nt & 1) + 1] = gelu2_f16x2(pack_f16x2(h[2], h[3]));
        }
        // layer 2 and GELU, laid out the same way as the A fragment of layer 3
        uint32_t a3[2][4];
#pragma unroll
        for (int nt = 0; nt < 4; nt++) {
            const uint4 w2 = w2v[nt];  // {ks0 b0, ks0 b1, ks1 b0, ks1 b1}
            const float2 b2 = b2v[nt];
            float o[4] = {b2.x, b2.y, b2.x, b2.y};
            mma_f16_16816(o, a2[0][0], a2[0][1], a2[0][2], a2[0][3], w2.x, w2.y);
            mma_f16_16816(o, a2[1][0], a2[1][1], a2[1][2], a2[1][3], w2.z, w2.w);
            a3[nt >> 1][2 * (nt & 1) + 0] = gelu2_f16x2(pack_f16x2(o[0], o[1]));
            a3[nt >> 1][2 * (nt & 1) + 1] = gelu2_f16x2(pack_f16x2(o[2], o[3]));
        }
        // layer 3: W3 fills every column of B, so each lane's accumulators hold z of
        // its rows g (z[mt][0]) and g + 8 (z[mt][2]) of the tile
        const uint4 w3 = w3v[lane];
        z[mt][0] = z[mt][1] = z[mt][2] = z[mt][3] = b3;
        mma_f16_16816(z[mt], a3[0][0], a3[0][1], a3[0][2], a3[0][3], w3.x, w3.y);
        mma_f16_16816(z[mt], a3[1][0], a3[1][1], a3[1][2], a3[1][3], w3.z, w3.w);
    }
    // lane 4 g + (2 mt + hh) of quad g offers row g + 8 hh of tile mt
    const float offer = (c == 0) ? z[0][0] : (c == 1) ? z[0][2] : (c == 2) ? z[1][0] : z[1][2];
    const int r = lane & 15;
    const float zz = __shfl_sync(0xffffffffu, offer, 4 * (r & 7) + 2 * (lane >> 4) + (r >> 3));
    return zz > 20.f ? zz : __logf(1.f + __expf(zz));
}
#endif

}  // namespace lbl
