// gram_tc.cu -- the localised Gram of the LETKF analysis on the tcgen05 tensor cores.
//
// For every grid point the analysis needs Q - (M-1)/beta I = dY^T R^-1 dY over the point's
// observation window (letkf_solver.h:252-254, a cublasSgemmStridedBatched pair in the
// reference, cu_matrix_cublas_wrapper.hpp:163-195).  All p x p points of an observation
// block share one window C [nobs x M] (the sites of letkf.cu:164-181 depend on i/p and j/p
// only); they differ only in the R^-1 x Gaspari-Cohn weights w_pt of the slots
// (letkf.cu:97-113, a pattern per (i mod p, j mod p)).  So
//
//     Q_pt - (M-1)/beta I = (diag(w_pt) C)^T C,
//
// and one CTA per block computes the p^2 Grams as MMAs with the shared B = C:
//   * A tile: 128 rows = 128/MP points x MP members, K = the window slots (padded to 8);
//     row (s, k) of point pt = t*128/MP + s holds w_pt[o] C[o][k];
//   * B: MP + 16 rows x K: the unweighted window (rows l < MP, member l), then the
//     innovations dyo of the slots (row MP), then zeros;
//   * D: 128 x (MP + 16) fp32 in tensor memory: row (s, k) holds row k of point pt's Gram in
//     columns l < MP and c_k = (dY^T R^-1 dyo)_k (letkf_solver.h:298-300) in column MP.
// FP32 accuracy from TF32 operands: every operand x = x_hi + x_lo with x_hi = tf32(x) and
// x_lo = tf32(x - x_hi), and D = A_hi B_hi + A_hi B_lo + A_lo B_hi (kind::tf32, FP32
// accumulation); the dropped A_lo B_lo and the rounding of x_lo are about 2^-22 relative.
// Both operands are K-major in the canonical no-swizzle layout: core matrices of 8 rows x
// 16 bytes, contiguous along K (LBO = 128 B) and K/4 core matrices apart between 8-row
// groups (SBO = 32 K bytes).  256 threads build A (two per row, one half of K each); one
// thread issues the MMAs, commits them to an mbarrier and polls it (bounded) while the
// others wait at the CTA barrier; warps 0-3 read D back with tcgen05.ld (warp w: lanes
// 32w..32w+31)
// and writes Q without the diagonal term to Qout[point][MP][MP] (row k, column l) and c to
// Cout[point][MP].  Only the CTA's own shared memory is read by the tensor cores; there is
// no multicast.
#include <cstdint>

#include "lbl_internal.h"

namespace lbl {
namespace {

constexpr int kTcRows = 128;          // MMA M
constexpr int kTcThreads = 256;       // two threads per A row (each half of K); warps 0-3 = TMEM lane quadrants
constexpr long long kTcWaitLimit = 1ll << 22;

__device__ __forceinline__ uint32_t saddr(const void* p) { return uint32_t(__cvta_generic_to_shared(p)); }

// shared-memory matrix descriptor (tcgen05): start, leading (K) and stride (8-row group)
// byte offsets >> 4, version 1, no swizzle
__device__ __forceinline__ uint64_t mat_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return uint64_t((addr >> 4) & 0x3FFFu) | (uint64_t((lbo >> 4) & 0x3FFFu) << 16) |
           (uint64_t((sbo >> 4) & 0x3FFFu) << 32) | (uint64_t(1) << 46);
}
// instruction descriptor of kind::tf32: D F32 (bits 4-5 = 1), A and B TF32 (bits 7-9, 10-12
// = 2), both K-major, N >> 3 at bits 17-22, M >> 4 at bits 24-28
constexpr uint32_t idesc_tf32(int m, int n) {
    return (1u << 4) | (2u << 7) | (2u << 10) | (uint32_t(n >> 3) << 17) | (uint32_t(m >> 4) << 24);
}

__device__ __forceinline__ uint32_t tf32_of(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ void split_tf32(float x, uint32_t& hi, uint32_t& lo) {
    hi = tf32_of(x);
    lo = tf32_of(x - __uint_as_float(hi));
}

__device__ __forceinline__ void mbar_init1(uint64_t* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(saddr(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_done(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(saddr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
    for (long long it = 0; it < kTcWaitLimit; it++)
        if (mbar_done(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ void tc_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void mma_tf32(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}" ::"r"(d),
        "l"(a), "l"(b), "r"(idesc), "r"(acc));
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(saddr(bar))
                 : "memory");
}
// 16 consecutive 32-bit columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// byte offset of element (row r, k) of a K-major no-swizzle operand with kpad columns
__device__ __forceinline__ uint32_t canon(int r, int k, int kpad) {
    return uint32_t((r >> 3) * (kpad * 32) + (k >> 2) * 128 + (r & 7) * 16 + (k & 3) * 4);
}

template <int MP>
__global__ void __launch_bounds__(kTcThreads, 1) gram_tc_kernel(const float* __restrict__ dY,
                                                                  const float* __restrict__ dyo,
                                                                  const float* __restrict__ wdense,
                                                                  float* __restrict__ Qout, float* __restrict__ Cout,
                                                                  GramTcParams G, int* __restrict__ err) {
    constexpr int PPT = kTcRows / MP;           // points per A tile
    constexpr int NB = MP + 16;                  // B rows = MMA N: members, innovations, zeros
    constexpr uint32_t NCOL = NB <= 32 ? 32 : (NB <= 64 ? 64 : 128);  // TMEM columns (a power of two)
    extern __shared__ __align__(1024) unsigned char smem[];
    const int kpad = G.kpad;
    const uint32_t a_bytes = uint32_t(kTcRows) * kpad * 4, b_bytes = uint32_t(NB) * kpad * 4;
    unsigned char* sA_hi = smem;
    unsigned char* sA_lo = sA_hi + a_bytes;
    unsigned char* sB_hi = sA_lo + a_bytes;
    unsigned char* sB_lo = sB_hi + b_bytes;
    float* sC = reinterpret_cast<float*>(sB_lo + b_bytes);  // [kpad][MP] window
    float* sD = sC + kpad * MP;                               // [kpad] innovations of the slots
    float* sW = sD + kpad;                                    // [p*p][kpad] weights
    uint64_t* bar = reinterpret_cast<uint64_t*>(sW + G.p * G.p * kpad);
    uint32_t* s_taddr = reinterpret_cast<uint32_t*>(bar + 1);
    int* s_fail = reinterpret_cast<int*>(s_taddr + 1);  // the poller's verdict, for the whole CTA

    const int tid = threadIdx.x, warp = tid >> 5;
    const int bi = blockIdx.x % G.nsx, bj = blockIdx.x / G.nsx;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(s_taddr)),
                     "r"(NCOL));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        mbar_init1(bar);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // the block's window: slot o = a + nox b + var nox^2 at site (bi + a - nl_off, bj + b - nl_off)
    const int nox2 = G.nox * G.nox;
#pragma unroll 4
    for (int e = tid; e < kpad * MP; e += kTcThreads) {
        const int o = e / MP, k = e - o * MP;
        float v = 0.f;
        if (o < G.nobs && k < G.M) {
            const int var = o / nox2, ab = o - var * nox2, b = ab / G.nox, a = ab - b * G.nox;
            int si = (bi + a - G.nl_off) % G.nsx;
            si += si < 0 ? G.nsx : 0;
            int sj = (bj + b - G.nl_off) % G.nsy;
            sj += sj < 0 ? G.nsy : 0;
            v = __ldg(dY + (size_t(var) * G.nsites + si + size_t(G.nsx) * sj) * G.M + k);
        }
        sC[e] = v;
    }
    for (int o = tid; o < kpad; o += kTcThreads) {
        float v = 0.f;
        if (o < G.nobs) {
            const int var = o / nox2, ab = o - var * nox2, b = ab / G.nox, a = ab - b * G.nox;
            int si = (bi + a - G.nl_off) % G.nsx;
            si += si < 0 ? G.nsx : 0;
            int sj = (bj + b - G.nl_off) % G.nsy;
            sj += sj < 0 ? G.nsy : 0;
            v = __ldg(dyo + size_t(var) * G.nsites + si + size_t(G.nsx) * sj);
        }
        sD[o] = v;
    }
    for (int e = tid; e < G.p * G.p * kpad; e += kTcThreads) sW[e] = __ldg(wdense + e);
    __syncthreads();
    // B = [C | dyo | 0] as [l][o], hi and lo
    for (int e = tid; e < NB * (kpad >> 2); e += kTcThreads) {
        const int l = e % NB, c4 = e / NB;
        uint32_t hi[4], lo[4];
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const int o = 4 * c4 + i;
            split_tf32(l < MP ? sC[o * MP + l] : (l == MP ? sD[o] : 0.f), hi[i], lo[i]);
        }
        const uint32_t off = canon(l, 4 * c4, kpad);
        *reinterpret_cast<uint4*>(sB_hi + off) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
        *reinterpret_cast<uint4*>(sB_lo + off) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
    }
    tc_before();
    __syncthreads();
    tc_after();
    const uint32_t taddr = *s_taddr;
    constexpr uint32_t idesc = idesc_tf32(kTcRows, NB);
    const uint32_t sbo_a = uint32_t(kpad) * 32, sbo_b = uint32_t(kpad) * 32;

    const int r = tid & (kTcRows - 1);    // this thread's A row (and, for warps 0-3, TMEM lane)
    const int half = tid >> 7;            // which half of the K chunks this thread builds
    const int s = r / MP, k = r - s * MP; // point within the tile, member
    const int ntiles = G.p * G.p / PPT;
    const int nch = kpad >> 2, c_lo = half * (nch >> 1), c_hi = c_lo + (nch >> 1);
    uint32_t phase = 0;
    bool failed = false;  // uniform: a commit that never arrived stops the CTA's MMAs
    for (int t = 0; t < ntiles && !failed; t++) {
        const int pat = t * PPT + s;
        const float* w = sW + pat * kpad;
        for (int c4 = c_lo; c4 < c_hi; c4++) {
            const float4 w4 = *reinterpret_cast<const float4*>(w + 4 * c4);
            const float wv[4] = {w4.x, w4.y, w4.z, w4.w};
            uint32_t hi[4], lo[4];
#pragma unroll
            for (int i = 0; i < 4; i++) split_tf32(wv[i] * sC[(4 * c4 + i) * MP + k], hi[i], lo[i]);
            const uint32_t off = canon(r, 4 * c4, kpad);
            *reinterpret_cast<uint4*>(sA_hi + off) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
            *reinterpret_cast<uint4*>(sA_lo + off) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
        }
        // the generic-proxy stores must be visible to the tensor cores' async proxy
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        tc_before();
        __syncthreads();
        tc_after();
        if (tid == 0) {
            const uint32_t a_lo = saddr(sA_lo), a_hi = saddr(sA_hi), b_hi = saddr(sB_hi), b_lo = saddr(sB_lo);
            const uint32_t aa[3] = {a_hi, a_hi, a_lo}, bb[3] = {b_hi, b_lo, b_hi};
            uint32_t acc = 0;
            for (int pr = 0; pr < 3; pr++)
                for (int ks = 0; ks < (kpad >> 3); ks++) {  // K = 8 per MMA: two core matrices along K
                    mma_tf32(taddr, mat_desc(aa[pr] + ks * 256, 128, sbo_a), mat_desc(bb[pr] + ks * 256, 128, sbo_b),
                             idesc, acc);
                    acc = 1;
                }
            mma_commit(bar);
        }
        // one thread polls the barrier; the others sleep at the CTA barrier meanwhile
        if (tid == 0) {
            *s_fail = mbar_wait_bounded(bar, phase) ? 0 : 1;
            tc_before();
        }
        __syncthreads();
        phase ^= 1;
        tc_after();
        if (*s_fail) {  // leave the tile unread; the MMAs may still be in flight
            failed = true;
            break;
        }
        // row r of D: this thread's lane (warp w reads lanes 32w..32w+31): the Gram row in
        // columns [0, MP), c_k in column MP
        const int pi = pat % G.p, pj = pat / G.p;
        const size_t point = size_t(bi * G.p + pi) + size_t(G.nx) * (bj * G.p + pj);
        float* q = Qout + (point * MP + k) * MP;
#pragma unroll
        for (int c0 = 0; half == 0 && c0 < MP; c0 += 16) {
            uint32_t v[16];
            tmem_ld16(taddr + (uint32_t(32 * warp) << 16) + uint32_t(c0), v);
            tmem_wait_ld();
#pragma unroll
            for (int i = 0; i < 16; i += 4)
                *reinterpret_cast<float4*>(q + c0 + i) = make_float4(__uint_as_float(v[i]), __uint_as_float(v[i + 1]),
                                                                     __uint_as_float(v[i + 2]),
                                                                     __uint_as_float(v[i + 3]));
        }
        if (half == 0) {
            uint32_t v[16];
            tmem_ld16(taddr + (uint32_t(32 * warp) << 16) + uint32_t(MP), v);
            tmem_wait_ld();
            Cout[point * MP + k] = __uint_as_float(v[0]);
        }
        tc_before();
        __syncthreads();  // the next tile rewrites A and the accumulator
        tc_after();
    }
    if (failed) {
        // code 4: the Gram's MMA wait gave up.  Wait once more (bounded) for the commit before
        // the accumulator is released; its rows of Q are not written.
        if (tid == 0) {
            atomicCAS(err, 0, 4);
            mbar_wait_bounded(bar, phase ^ 1);
        }
        __syncthreads();
    }
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(NCOL));
}

template <int MP>
size_t gram_tc_smem_mp(int kpad, int p) {
    // operands, window, weights, barrier + TMEM address.  Every address an MMA forms stays
    // inside its operand (rows < 128 or MP, K steps < kpad/8), and would under either reading
    // of the two strides: (kpad/8 - 1) 256 + 15 x 128 + 32 kpad + 127 < 128 kpad x 4.
    return size_t(2) * kTcRows * kpad * 4 + size_t(2) * (MP + 16) * kpad * 4 + size_t(kpad) * MP * 4 + size_t(kpad) * 4 +
           size_t(p) * p * kpad * 4 + 32;
}

}  // namespace

bool gram_tc_supported(int M, int p, int nobs) {
    const int mp = M <= 16 ? 16 : (M <= 32 ? 32 : 64);
    const int kpad = (nobs + 7) & ~7;
    return M >= 2 && M <= 64 && p >= 1 && (p * p) % (kTcRows / mp) == 0 && gram_tc_smem(M, p, nobs) <= 227 * 1024 &&
           kpad <= 256;
}

size_t gram_tc_smem(int M, int p, int nobs) {
    const int kpad = (nobs + 7) & ~7;
    if (M <= 16) return gram_tc_smem_mp<16>(kpad, p);
    if (M <= 32) return gram_tc_smem_mp<32>(kpad, p);
    return gram_tc_smem_mp<64>(kpad, p);
}

int gram_tc_prepare() {
    const int lim = 227 * 1024;
    int rc = int(cudaFuncSetAttribute(gram_tc_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
    rc |= int(cudaFuncSetAttribute(gram_tc_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
    rc |= int(cudaFuncSetAttribute(gram_tc_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
    return rc;
}

void launch_gram_tc(const GramTcParams& G, const float* dY, const float* dyo, const float* wdense, float* Qout,
                    float* Cout, int* err, cudaStream_t s) {
    const int blocks = G.nsx * G.nsy;
    const size_t sm = gram_tc_smem(G.M, G.p, G.nobs);
    if (G.M <= 16)
        gram_tc_kernel<16><<<blocks, kTcThreads, sm, s>>>(dY, dyo, wdense, Qout, Cout, G, err);
    else if (G.M <= 32)
        gram_tc_kernel<32><<<blocks, kTcThreads, sm, s>>>(dY, dyo, wdense, Qout, Cout, G, err);
    else
        gram_tc_kernel<64><<<blocks, kTcThreads, sm, s>>>(dY, dyo, wdense, Qout, Cout, G, err);
}

}  // namespace lbl
