// letkf_kernels.cu -- LETKF analysis kernels for sm_100a (FP32, IEEE division/sqrt).
//
// The reference (letkf.cu:120-360, util/letkf_solver.h:235-349) builds, per grid
// point, a 75-row observation window out of every member's H(x), multiplies it
// with a dense 75x75 R^-1 through cuBLAS, eigen-decomposes Q with cuSOLVER
// syevjBatched, and applies W through more cuBLAS calls, with MPI alltoalls in
// between.  Here the whole ensemble is resident, so:
//
//   obs_ensemble_kernel  H(x) = (u, v, rho) of every member at every observation
//                        site, minus the member mean  -> dY[var][site][member],
//                        and the innovation yo - mean -> dyo[var][site]
//                        (pack_yk letkf.cu:148-187, set_yo :230-269, ybar/dY/dyo
//                        letkf_solver.h:239-243).  Mean over members depends only
//                        on the site, so it is computed once per site.
//   analysis_kernel<MP>  one group of MP lanes (lane = member) per grid point:
//                        gather the localised window (R^-1 x Gaspari-Cohn weights
//                        from a per-(i mod p, j mod p) table, zero-weight slots
//                        dropped), Gram Q = (M-1)/beta I + dY^T R^-1 dY,
//                        one-sided (Hestenes) Jacobi eigensolver in registers with
//                        xor-pair parallel ordering, then
//                        Xa = xbar + dX V (sqrt(M-1) Lambda^-1/2 V^T + Lambda^-1 V^T dY^T R^-1 dyo 1^T)
//                        written straight into the member-major populations, plus
//                        the lbm2euler macros (letkf.cu:336-357).
#include <cmath>

#include "lbl_internal.h"

namespace lbl {
namespace {

__host__ __device__ constexpr int exq(int q) { return (q % 3) - 1; }
__host__ __device__ constexpr int eyq(int q) { return (q / 3) - 1; }

struct AnaParams {
    int nx, ny, nxy, M;
    int p, nsx, nsy, nsites;
    int n_pat_max;          // window slots = entries per pattern row of the weight table
    int nox;                // window sites per row
    int nl_off;             // n_obs_local - obs_offset (window origin, in sites)
    float diag;             // (M-1)/beta
    float sqrt_m1;          // sqrt(M-1)
    float tol;              // Jacobi off-diagonal tolerance: pairs below tol are not rotated
    float stop;             // sqrt(tol): a sweep whose worst relative off-diagonal is below it ends the
                            // iteration, since the sweep's own rotations leave about stop^2 = tol
    int max_sweeps;
    const float* qin;       // Q - (M-1)/beta I per point from the tensor-core Gram, or null
    const float* cin;       // with it, c = dY^T R^-1 dyo per point (cin + n mpq, member k)
    int mpq;                // its member padding: Q of point n at qin + n mpq^2, row k, column l
    float c;                // lattice speed for the macros
    int write_v;            // 0 reproduces the reference's stale v after analysis
    int tile_y0;            // first tile row (0 for the whole grid)
};

// Matrix dump of one chunk of whole rows [j0, j1) (the batch of one reference rank):
// every matrix of letkf_solver.h:243-345 per point b = point - point0, column-major
// with the point slowest, as cu_matrix::save lays them out.
struct DumpPtrs {
    float *dYf, *dyo, *Q, *V, *Xf, *dXf, *Pa, *dWa, *Xa, *Wa, *AI, *Z, *Lambda, *Wma;
    int j0, j1, point0;
};

// ---------------------------------------------------------------------------
// H(x) at every observation site for every member, centred on the member mean.
// One warp per site; lanes stride over members.
// ---------------------------------------------------------------------------
__global__ void obs_ensemble_kernel(const float* __restrict__ f, const float* __restrict__ yo,
                                    float* __restrict__ dY, float* __restrict__ dyo, AnaParams A) {
    const int lane = threadIdx.x & 31;
    const int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (s >= A.nsites) return;
    const int si = s % A.nsx, sj = s / A.nsx;
    const int ij = si * A.p + A.nx * (sj * A.p);
    constexpr int kPer = 2;  // members per lane (M <= 64)
    float H[3][kPer];
    float sum[3] = {0.f, 0.f, 0.f};
#pragma unroll
    for (int t = 0; t < kPer; t++) {
        const int m = lane + 32 * t;
        H[0][t] = H[1][t] = H[2][t] = 0.f;
        if (m < A.M) {
            float fc[kQ];
#pragma unroll
            for (int q = 0; q < kQ; q++) fc[q] = __ldg(f + (size_t(m) * kQ + q) * A.nxy + ij);
            float r = 0, mu = 0, mv = 0;
#pragma unroll
            for (int q = 0; q < kQ; q++) r += fc[q];
#pragma unroll
            for (int q = 0; q < kQ; q++) { mu += fc[q] * A.c * exq(q); mv += fc[q] * A.c * eyq(q); }
            H[0][t] = mu / r;  // u
            H[1][t] = mv / r;  // v
            H[2][t] = r;       // rho
            sum[0] += H[0][t]; sum[1] += H[1][t]; sum[2] += H[2][t];
        }
    }
#pragma unroll
    for (int v = 0; v < 3; v++)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) sum[v] += __shfl_xor_sync(0xffffffffu, sum[v], o);
#pragma unroll
    for (int v = 0; v < 3; v++) {
        const float mean = sum[v] / float(A.M);
#pragma unroll
        for (int t = 0; t < kPer; t++) {
            const int m = lane + 32 * t;
            if (m < A.M) dY[(size_t(v) * A.nsites + s) * A.M + m] = H[v][t] - mean;
        }
        if (lane == 0) dyo[size_t(v) * A.nsites + s] = yo[size_t(v) * A.nsites + s] - mean;
    }
}

// square root for the Jacobi rotation angle: t only picks the angle, and cs = (1 + t^2)^-1/2
// makes the rotation orthogonal for any t, so the hardware approximation serves
__device__ __forceinline__ float sqrt_approx(float x) {
    float r;
    asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

template <int MP>
__device__ __forceinline__ float group_sum(float v) {
#pragma unroll
    for (int o = MP / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// ---------------------------------------------------------------------------
// The local analysis.  MP = member lanes per grid point (power of two >= M).
// A group of MP lanes walks a CW x CH tile of neighbouring grid points in snake
// order.  The unweighted observation window of the current p x p block is cached
// in shared memory, and every point's Jacobi starts from the previous point's
// eigenvectors (A = Q V_prev), which leaves little to rotate.
// Weight table entry (int4): x = window slot (a + nox*b + var*nox^2), y = variable,
// z = sqrt(w) bits (the tensor-core Gram's row weight; zero in tables that serve only
// analysis_kernel), w = weight bits (sigma^-2 x Gaspari-Cohn), only w > 0, per pattern
// (i mod p, j mod p).
// ---------------------------------------------------------------------------
constexpr int kCW = 4, kCH = 2;  // chain tile (points in x, points in y)

// The Jacobi ends after a sweep whose largest rotated relative off-diagonal stayed below
// sqrt(tol), counting on quadratic convergence to bring the sweep's rotations down to tol.
// That holds while every late rotation is small.  A pair of (nearly) equal column norms
// turns by up to 45 degrees even for a tiny off-diagonal (the products of other pairs'
// residues suffice once they pass tol), which remixes residues the sweep had already
// removed and makes convergence linear: with p = 1 (three observations, a 13-fold
// eigenvalue (M-1)/beta at M = 16) the increments then kept errors of about sqrt(tol)
// (8e-4 of the largest increment against the reference's solver).  So a sweep that meets
// the quadratic stop but turned some pair wider than atan(kWideTurn) is followed by one
// cleanup sweep in which such turns are skipped: the nearly degenerate pairs are already
// orthogonal to about tol, and mixing eigenvectors of (nearly) equal eigenvalues leaves the
// transform as it is, while the other pairs then converge quadratically.  Measured against the
// FP64 oracle with observation errors 0.1 (u, v) and 0.01 (rho): 4.3e-4 of the largest increment without the
// cleanup at 256^2 x 16, 9.8e-6 with it (3.0 -> 3.4 mean sweeps); at 512^2 x 64, 6.2e-4 and
// 2.8e-5 (2.4 -> 3.3 mean sweeps).
constexpr float kWideTurn = 0.1f;
// the wide analysis walks taller tiles: fewer cold starts, and its many waves hide
// the longer CTAs (512^2, M = 64: 58.7 ms at 4 x 8, 59.3 at 4 x 4, 62.8 at 4 x 2;
// 16 members' kernel is fastest at 4 x 2 on 256^2)
constexpr int kWCW = 4, kWCH = 8;

// DUMP = true recomputes the tiles that cover the rows of D and, instead of writing
// the analysis, writes every intermediate matrix of those rows (need_save_mat).
template <int MP, bool DUMP>
__global__ void __launch_bounds__(128) analysis_kernel(const float* __restrict__ fin, float* __restrict__ fout,
                                                       float* __restrict__ mac, const float* __restrict__ dY,
                                                       const float* __restrict__ dyo,
                                                       const int4* __restrict__ wtab,
                                                       const int* __restrict__ wcnt, int* __restrict__ stats,
                                                       AnaParams A, DumpPtrs D) {
    constexpr int GPW = 32 / MP;
    extern __shared__ float smem[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int grp = lane / MP;
    const int k = lane % MP;
    const int gbase = lane - k;
    const int M = A.M;
    const bool real_k = k < M;
    const int nobs = A.n_pat_max;  // window slots (3 * nox * nox)
    const int nox2 = nobs / 3;

    // per-group shared memory
    // every block below is a multiple of 4 floats, so all float4 accesses stay 16-B aligned
    const int nobs_pad = (nobs + 3) & ~3;
    const int per_grp = nobs * MP + nobs_pad + MP * MP + kQ * MP + 2 * MP + 12;
    float* base = smem + size_t(warp * GPW + grp) * per_grp;
    float* sW = base;                          // [nobs][MP] window dY (unweighted)
    float* sDyo = sW + nobs * MP;              // [nobs]     window innovations (padded to 4)
    float* sQ = sDyo + nobs_pad;               // [MP][MP] Q columns, then V
    float* sDX = sQ + MP * MP;                 // [9][MP]  dX, then D = dX V in place
    float* sS = sDX + kQ * MP;                 // [MP]     sqrt(M-1)/sqrt(lambda)
    float* sY = sS + MP;                       // [MP]     Lambda^-1 V^T c
    float* sXbar = sY + MP;                    // [9]      ensemble mean (12 reserved)

    const int tiles_x = (A.nx + kCW - 1) / kCW;
    const int tile = (blockIdx.x * (blockDim.x >> 5) + warp) * GPW + grp;
    const int x0 = (tile % tiles_x) * kCW;
    const int y0 = (A.tile_y0 + tile / tiles_x) * kCH;
    const unsigned gmask = (MP == 32) ? 0xffffffffu : (((1u << MP) - 1u) << gbase);

    float vv[MP];  // eigenvectors (column k), carried from point to point
#pragma unroll
    for (int l = 0; l < MP; l++) vv[l] = (l == k) ? 1.f : 0.f;
    int cached_bi = -1, cached_bj = -1;
    int max_sweeps = 0, noconv = 0, total_sweeps = 0;
    bool bad = false;

    for (int idx = 0; idx < kCW * kCH; idx++) {
        const int r = idx / kCW;
        const int cc = (r & 1) ? (kCW - 1 - idx % kCW) : (idx % kCW);
        const int i = x0 + cc, j = y0 + r;
        const bool active = (i < A.nx) && (j < A.ny);  // uniform within the group
        const int point = active ? i + A.nx * j : 0;
        const bool real_m = active && real_k;
        const bool dump = DUMP && active && j >= D.j0 && j < D.j1;
        const size_t b = dump ? size_t(point - D.point0) : 0;

        // 1. forecast ensemble at the point: X, xbar, dX (letkf_solver.h:278-280)
        {
            float xq[kQ];
#pragma unroll
            for (int q = 0; q < kQ; q++) xq[q] = real_m ? __ldg(fin + (size_t(k) * kQ + q) * A.nxy + point) : 0.f;
#pragma unroll
            for (int q = 0; q < kQ; q++) {
                const float xb = group_sum<MP>(xq[q]) / float(M);
                sDX[q * MP + k] = real_m ? xq[q] - xb : 0.f;
                if (k == 0) sXbar[q] = xb;
                if (DUMP && dump && real_k) {
                    D.Xf[q + kQ * (k + M * b)] = xq[q];
                    D.dXf[q + kQ * (k + M * b)] = xq[q] - xb;
                }
            }
        }

        // 2. observation window of the point's p x p block (pack_yk/set_yo geometry,
        //    letkf.cu:148-269), gathered once per block from the site ensemble
        const int bi = i / A.p, bj = j / A.p;
        if ((DUMP || !A.qin) && (bi != cached_bi || bj != cached_bj)) {  // the tensor-core Gram needs no window
            for (int b = 0; b < A.nox; b++) {
                int sj = (bj + b - A.nl_off) % A.nsy;
                sj += sj < 0 ? A.nsy : 0;
                for (int a = 0; a < A.nox; a++) {
                    int si = (bi + a - A.nl_off) % A.nsx;
                    si += si < 0 ? A.nsx : 0;
                    const int site = si + A.nsx * sj;
#pragma unroll
                    for (int var = 0; var < 3; var++) {
                        const int sl = a + A.nox * b + var * nox2;
                        sW[sl * MP + k] = real_k ? __ldg(dY + (size_t(var) * A.nsites + site) * M + k) : 0.f;
                        if (k == 0) sDyo[sl] = __ldg(dyo + size_t(var) * A.nsites + site);
                    }
                }
            }
            cached_bi = bi;
            cached_bj = bj;
        }
        __syncwarp();
        if (DUMP && dump) {
            if (real_k)
                for (int sl = 0; sl < nobs; sl++) D.dYf[sl + size_t(nobs) * (k + M * b)] = sW[sl * MP + k];
            for (int sl = k; sl < nobs; sl += MP) D.dyo[sl + nobs * b] = sDyo[sl];
        }

        // 3. Gram: column k of Q = (M-1)/beta I + dY^T R^-1 dY (letkf_solver.h:252-254),
        //    and c_k = (dY^T R^-1 dyo)_k
        const int pat = (i % A.p) + A.p * (j % A.p);
        const int cnt = wcnt[pat];
        const int4* ent = wtab + size_t(pat) * nobs;
        float qv[MP];
#pragma unroll
        for (int l = 0; l < MP; l++) qv[l] = 0.f;
        float ck = 0.f;
        if (!DUMP && A.qin) {  // Q and c from the tensor-core Gram (gram_tc.cu)
            ck = real_m ? __ldg(A.cin + size_t(point) * A.mpq + k) : 0.f;
            const float* qrow = A.qin + (size_t(point) * A.mpq + k) * A.mpq;
#pragma unroll
            for (int l = 0; l < MP; l += 4) {
                const float4 q4 = real_m ? __ldg(reinterpret_cast<const float4*>(qrow + l)) : make_float4(0.f, 0.f, 0.f, 0.f);
                qv[l] = q4.x;
                qv[l + 1] = q4.y;
                qv[l + 2] = q4.z;
                qv[l + 3] = q4.w;
            }
        }
        for (int o = 0; (DUMP || !A.qin) && o < cnt; o++) {
            const int4 e = ent[o];
            const float* row = sW + e.x * MP;
            const float ek = __int_as_float(e.w) * row[k];
            ck = fmaf(ek, sDyo[e.x], ck);
#pragma unroll
            for (int l = 0; l < MP; l += 4) {
                const float4 r4 = *reinterpret_cast<const float4*>(row + l);
                qv[l + 0] = fmaf(ek, r4.x, qv[l + 0]);
                qv[l + 1] = fmaf(ek, r4.y, qv[l + 1]);
                qv[l + 2] = fmaf(ek, r4.z, qv[l + 2]);
                qv[l + 3] = fmaf(ek, r4.w, qv[l + 3]);
            }
        }
#pragma unroll
        for (int l = 0; l < MP; l++)
            if (l == k && k < M) qv[l] += A.diag;
        if (DUMP && dump && real_k)
            for (int l = 0; l < M; l++) D.Q[l + M * (k + M * b)] = qv[l];

        // 4. warm start: A = Q V_prev (column k = sum_l Q_:l V_prev[l][k])
        if (idx > 0) {
#pragma unroll
            for (int l = 0; l < MP; l++) sQ[k * MP + l] = qv[l];
            __syncwarp();
            float av[MP];
#pragma unroll
            for (int l = 0; l < MP; l++) av[l] = 0.f;
#pragma unroll
            for (int l = 0; l < MP; l++) {
                const float vl = vv[l];
#pragma unroll
                for (int t = 0; t < MP; t += 4) {
                    const float4 q4 = *reinterpret_cast<const float4*>(sQ + l * MP + t);
                    av[t + 0] = fmaf(q4.x, vl, av[t + 0]);
                    av[t + 1] = fmaf(q4.y, vl, av[t + 1]);
                    av[t + 2] = fmaf(q4.z, vl, av[t + 2]);
                    av[t + 3] = fmaf(q4.w, vl, av[t + 3]);
                }
            }
            __syncwarp();
#pragma unroll
            for (int l = 0; l < MP; l++) qv[l] = av[l];
        }

        // 5. one-sided Jacobi: rotate column pairs (k, k^r) of A = Q V until mutually
        //    orthogonal.  V is not accumulated: for SPD Q, A with orthogonal columns is
        //    V Lambda (A^T A = V^T Q^2 V diagonal makes V diagonalise Q), so column k of
        //    V is a_k / |a_k| and lambda_k = |a_k|.  A sweep whose largest relative
        //    off-diagonal |g|/sqrt(a b) stayed below sqrt(tol) ends the iteration:
        //    convergence is quadratic, so that sweep's rotations leave about tol, the
        //    relative off-diagonal norm at which the reference's syevj stops.
        //    Rotations are applied with a lazy column scale: column k is sc * qv, so a
        //    rotation cs a + sn b becomes qv += (sn / cs)(sc_b / sc) pq_b, sc *= cs: one
        //    FMA per element instead of a multiply and an FMA.  The scale is folded back
        //    into qv at the start of every sweep.
        int sweeps = 0;
        bool converged = false;
        bool cleanup = false;  // this sweep turns no nearly degenerate pair (see kWideTurn)
        const float tol2 = A.tol * A.tol, stop2 = A.stop * A.stop;  // the tests below compare squares
        float sc = 1.f;
        for (int sw = 0; sw < A.max_sweeps; sw++) {
#pragma unroll
            for (int l = 0; l < MP; l++) qv[l] *= sc;
            sc = 1.f;
            float a0 = 0.f, a1 = 0.f;
#pragma unroll
            for (int l = 0; l < MP; l += 2) { a0 = fmaf(qv[l], qv[l], a0); a1 = fmaf(qv[l + 1], qv[l + 1], a1); }
            float a = a0 + a1;
            bool rot = false, wide = false;
            float worst = 0.f;  // largest g^2 / (a b) of the sweep
// three rounds per loop body: the 256^2 x 16 analysis phase 0.637 against 0.643 ms (one round:
            // run-time loop control; all fifteen: 0.720 ms, the body no longer fits the instruction cache)
#pragma unroll 3
            for (int rr = 1; rr < MP; rr++) {
                float pq[MP];
#pragma unroll
                for (int l = 0; l < MP; l++) pq[l] = __shfl_xor_sync(0xffffffffu, qv[l], rr);
                const float sp = __shfl_xor_sync(0xffffffffu, sc, rr);
                float g0 = 0.f, g1 = 0.f;
#pragma unroll
                for (int l = 0; l < MP; l += 2) { g0 = fmaf(qv[l], pq[l], g0); g1 = fmaf(qv[l + 1], pq[l + 1], g1); }
                const float g = (g0 + g1) * (sc * sp);
                const float b = __shfl_xor_sync(0xffffffffu, a, rr);
                const bool low = k < (k ^ rr);
                const float alo = low ? a : b, ahi = low ? b : a;
                // |g| > tol sqrt(alo ahi), on squares
                const float p2 = alo * ahi, g2 = g * g;
                bool apply = false;
                if (g2 > tol2 * p2) {
                    // any exact rotation converges; cs^2 + sn^2 = 1 keeps the columns' span
                    // t = sign(zeta) / (|zeta| + sqrt(1 + zeta^2)), zeta = d / e, multiplied through by |e|:
                    // one reciprocal on the critical path instead of two
                    const float d = ahi - alo, e = 2.f * g;
                    const float t = __fdividef(copysignf(fabsf(e), d * e), fabsf(d) + sqrt_approx(fmaf(d, d, e * e)));
                    const bool wt = fabsf(t) > kWideTurn;  // both lanes of the pair agree
                    apply = !(cleanup && wt);
                    if (apply) {
                        worst = fmaxf(worst, __fdividef(g2, p2));
                        wide |= wt;
                        const float cs = rsqrtf(fmaf(t, t, 1.f));
                        // low: cs a - sn b; high: sn a + cs b (sn = cs t), with the scales
                        const float rho = (low ? -t : t) * __fdividef(sp, sc);
#pragma unroll
                        for (int l = 0; l < MP; l++) qv[l] = fmaf(rho, pq[l], qv[l]);
                        sc *= cs;
                        a = low ? a - t * g : a + t * g;
                    }
                }
                rot |= apply;
            }
            // group max of the sweep's relative off-diagonal
#pragma unroll
            for (int o = MP / 2; o > 0; o >>= 1) worst = fmaxf(worst, __shfl_xor_sync(0xffffffffu, worst, o));
            // the quadratic stop; after a sweep with a wide turn, one cleanup sweep first
            const bool quad = (__ballot_sync(0xffffffffu, rot) & gmask) == 0u || worst < stop2;
            const bool any_wide = (__ballot_sync(0xffffffffu, wide) & gmask) != 0u;
            bool done;
            if (cleanup) {
                done = quad;
                cleanup = false;
            } else {
                done = quad && !any_wide;
                cleanup = quad && any_wide;
            }
            const unsigned ballot = __ballot_sync(0xffffffffu, !done && active);
            if (!converged) {
                sweeps = sw + 1;
                if ((ballot & gmask) == 0u) converged = true;
            }
            if (ballot == 0u) break;
        }

        // 6. eigenpair of column k: lambda_k = |a_k|, v_k = a_k / lambda_k (padding
        //    columns are zero and keep the unit vector); transform (letkf_solver.h:288-316)
#pragma unroll
        for (int l = 0; l < MP; l++) qv[l] *= sc;
        float lam = 0.f;
        {
            float n0 = 0.f, n1 = 0.f;
#pragma unroll
            for (int l = 0; l < MP; l += 2) { n0 = fmaf(qv[l], qv[l], n0); n1 = fmaf(qv[l + 1], qv[l + 1], n1); }
            const float n2 = n0 + n1;
            if (n2 > 0.f) {
                lam = sqrtf(n2);
                const float inv = 1.f / lam;
#pragma unroll
                for (int l = 0; l < MP; l++) vv[l] = qv[l] * inv;
            } else {
#pragma unroll
                for (int l = 0; l < MP; l++) vv[l] = (l == k) ? 1.f : 0.f;
            }
        }
#pragma unroll
        for (int l = 0; l < MP; l++) sQ[k * MP + l] = vv[l];
        float vc = 0.f;  // (V^T c)_k
#pragma unroll
        for (int l = 0; l < MP; l++) vc = fmaf(vv[l], __shfl_sync(0xffffffffu, ck, gbase + l), vc);
        sY[k] = real_k ? vc / lam : 0.f;
        sS[k] = real_k ? A.sqrt_m1 / sqrtf(lam) : 0.f;
        __syncwarp();
        if (DUMP) {
            // V, Lambda; P = V Lambda^-1 V^T, dW = sqrt(M-1) V Lambda^-1/2 V^T, w = V Lambda^-1 V^T c,
            // W = dW + w 1^T, Z = W - I, Wma = w 1^T (letkf_solver.h:263-345); column k per lane
            float lamj[MP];
#pragma unroll
            for (int jj = 0; jj < MP; jj++) lamj[jj] = __shfl_sync(0xffffffffu, lam, gbase + jj);
            if (dump && real_k) {
                const size_t o = size_t(M) * (k + M * b);
                for (int l = 0; l < M; l++) {
                    float pa = 0.f, dw = 0.f, w = 0.f;
                    for (int jj = 0; jj < M; jj++) {
                        const float vl = sQ[jj * MP + l], vk = sQ[jj * MP + k];
                        pa = fmaf(vl * vk, 1.f / lamj[jj], pa);
                        dw = fmaf(vl * vk, 1.f / sqrtf(lamj[jj]), dw);
                        w = fmaf(vl, sY[jj], w);
                    }
                    dw *= A.sqrt_m1;
                    D.V[o + l] = vv[l];
                    D.Lambda[o + l] = (l == k) ? lam : 0.f;
                    D.Pa[o + l] = pa;
                    D.dWa[o + l] = dw;
                    D.Wa[o + l] = dw + w;
                    D.Z[o + l] = dw + w - ((l == k) ? 1.f : 0.f);
                    D.Wma[o + l] = w;
                }
            }
        }
        {
            float dsum[kQ];
#pragma unroll
            for (int q = 0; q < kQ; q++) {
                dsum[q] = 0.f;
#pragma unroll
                for (int l = 0; l < MP; l++) dsum[q] = fmaf(sDX[q * MP + l], vv[l], dsum[q]);
            }
            __syncwarp();  // every lane has read dX before D overwrites it
#pragma unroll
            for (int q = 0; q < kQ; q++) sDX[q * MP + k] = dsum[q];
        }
        __syncwarp();
        float acc[kQ];
#pragma unroll
        for (int q = 0; q < kQ; q++) acc[q] = 0.f;
#pragma unroll 4
        for (int jj = 0; jj < MP; jj++) {
            const float z = fmaf(sS[jj], sQ[jj * MP + k], sY[jj]);
#pragma unroll
            for (int q = 0; q < kQ; q++) acc[q] = fmaf(sDX[q * MP + jj], z, acc[q]);
        }

        // 7. write the analysis member k, refresh its macros (update_xk + lbm2euler)
        if (DUMP) {
            if (dump && real_k)
#pragma unroll
                for (int q = 0; q < kQ; q++) {
                    const float xa = sXbar[q] + acc[q];
                    const float xf = __ldg(fin + (size_t(k) * kQ + q) * A.nxy + point);
                    D.Xa[q + kQ * (k + M * b)] = xa;
                    D.AI[q + kQ * (k + M * b)] = xa - xf;
                }
        } else if (real_m) {
            float xa[kQ];
#pragma unroll
            for (int q = 0; q < kQ; q++) {
                xa[q] = sXbar[q] + acc[q];
                bad |= !(xa[q] == xa[q]);
                fout[(size_t(k) * kQ + q) * A.nxy + point] = xa[q];
            }
            float rsum = 0, mu = 0, mv = 0;
#pragma unroll
            for (int q = 0; q < kQ; q++) rsum += xa[q];
#pragma unroll
            for (int q = 0; q < kQ; q++) { mu += xa[q] * A.c * exq(q); mv += xa[q] * A.c * eyq(q); }
            float* mm = mac + size_t(k) * 3 * A.nxy;
            mm[point] = rsum;
            mm[A.nxy + point] = mu / rsum;
            if (A.write_v) mm[2 * A.nxy + point] = mv / rsum;
        }
        if (active) {
            max_sweeps = max(max_sweeps, sweeps);
            total_sweeps += sweeps;
            noconv += converged ? 0 : 1;
        }
        __syncwarp();
    }
    if (DUMP) return;
    if (bad) atomicOr(stats + 2, 1);
    if (k == 0 && total_sweeps > 0) {
        atomicMax(stats + 0, max_sweeps);
        if (noconv) atomicAdd(stats + 1, noconv);
        atomicAdd(stats + 3, total_sweeps);
    }
}

// ---------------------------------------------------------------------------
// The local analysis for 32 < M <= 64 (the 64-member ensembles; the reference runs them
// through EigenG-Batched).  One CTA of 128 threads walks one kWCW x kWCH tile of points;
// thread t owns rows [32h, 32h + 32) (h = t & 1) of member column k = t >> 1 for the
// Gram, the warm start and the transform; the two halves of a column combine their
// partial sums with one shuffle.  The algorithm is the one above, except that the
// Jacobi hands whole column pairs between quads of threads through shared memory (step 5).
// ---------------------------------------------------------------------------
constexpr int kWide = 64;             // member columns
constexpr int kHalf = 32;             // rows per thread
constexpr int kWideThreads = 2 * kWide;

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
// floats per half column in the exchange matrix sA: 32 rows and 4 of padding, so that
// a stride of 36 = 4 (mod 32) spreads a quarter warp's 16-byte accesses over the bank
// groups.  The (k, h) threads touch eight consecutive half columns at the same chunk
// (eight groups); in the Jacobi a quad's threads read 16-row quarters of one column
// (half columns 2c, 2c + 1 at offsets 0 and 16: groups 2c + {0, 4, 1, 5} mod 8) and the
// two quads of a quarter warp read columns one apart (the other four groups).  A
// thread's chunks sit at fixed offsets from one base address.
constexpr int kHS = kHalf + 4;
// Arrays indexed by member (window rows, dX, the per-column scalars) put the upper half
// 4 floats further on, so that a column's two threads, which read element m and m + 32
// together, hit different bank groups: member m sits at hx(m) of a kHP-float row.
constexpr int kHP = kWide + 4;
__device__ __forceinline__ int hx(int m) { return m + 4 * (m >> 5); }
// float offset of 16-byte chunk c4 (rows 4 c4 .. 4 c4 + 3) of half column hb
__device__ __forceinline__ int sa_chunk(int hb, int c4) { return hb * kHS + 4 * c4; }
// sum of the two halves of a column (adjacent lanes)
__device__ __forceinline__ float pair_sum(float v) { return v + __shfl_xor_sync(0xffffffffu, v, 1); }
// sum over a quad of lanes (4s .. 4s + 3); every lane of the quad gets the same value
__device__ __forceinline__ float quad_sum(float v) {
    v += __shfl_xor_sync(0xffffffffu, v, 1);
    return v + __shfl_xor_sync(0xffffffffu, v, 2);
}
// 16 consecutive floats of shared memory (16-byte aligned) to registers and back
__device__ __forceinline__ void wide_load16(float (&x)[16], const float* p) {
#pragma unroll
    for (int m = 0; m < 16; m += 4) {
        const float4 v = *reinterpret_cast<const float4*>(p + m);
        x[m] = v.x; x[m + 1] = v.y; x[m + 2] = v.z; x[m + 3] = v.w;
    }
}
__device__ __forceinline__ void wide_store16(float* p, const float (&x)[16]) {
#pragma unroll
    for (int m = 0; m < 16; m += 4) *reinterpret_cast<float4*>(p + m) = make_float4(x[m], x[m + 1], x[m + 2], x[m + 3]);
}

// BF16 tensor-core Gram (TC): the point's weighted window C = sqrt(w) dY (one row per
// member, one column per weight-table entry) is staged as BF16 in sA, kCStride
// entries per row (the padding spreads a quarter warp's fragment loads over all 32
// banks), and Q - diag = C C^T is formed by mma.sync m16n8k16 with FP32 accumulators,
// warp w taking rows [16 w, 16 w + 16).  Entries are taken kGramChunk at a time.
constexpr int kGramChunk = 80;  // entries per staged chunk (5 k-steps)
constexpr int kCStride = 88;    // BF16 elements per staged row

__device__ __forceinline__ void mma_bf16_16816(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                               uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

template <bool TC>
// 5 CTAs per SM for the FP32 Gram (96 registers); the tensor-core Gram keeps 4 (its staging
// overwrites sA, so it carries the eigenvectors in registers)
__global__ void __launch_bounds__(kWideThreads, TC ? 4 : 5) analysis_wide_kernel(const float* __restrict__ fin,
                                                                     float* __restrict__ fout, float* __restrict__ mac,
                                                                     const float* __restrict__ dY,
                                                                     const float* __restrict__ dyo,
                                                                     const int4* __restrict__ wtab,
                                                                     const int* __restrict__ wcnt,
                                                                     int* __restrict__ stats, AnaParams A) {
    extern __shared__ float smem[];
    const int t = threadIdx.x;
    const int k = t >> 1, h = t & 1, r0 = kHalf * h;
    const int warp = t >> 5, lane = t & 31;
    const int M = A.M;
    const bool real_k = k < M;
    const int nobs = A.n_pat_max;
    const int nox2 = nobs / 3;
    const int nobs_pad = (nobs + 3) & ~3;
    float* sW = smem;                    // [nobs][kHP] window dY (unweighted), member m at hx(m)
    float* sDyo = sW + nobs * kHP;       // [nobs]      window innovations (padded to 4)
    float* sA = sDyo + nobs_pad;         // [128][kHS]  half columns: Q, the Jacobi's home slots, then V
    float* sDX = sA + 2 * kWide * kHS;   // [9][kHP]    dX, then D = dX V in place
    float* sS = sDX + kQ * kHP;          // [kHP]       sqrt(M-1)/sqrt(lambda)
    float* sY = sS + kHP;                // [kHP]       Lambda^-1 V^T c
    float* sN = sY + kHP;                // [kHP]       squared column norms of A (Jacobi rounds), and
    float* sC = sN;                      //             c = dY^T R^-1 dyo (transform), and
    float* sRed = sN;                    //             per-warp partial sums [4][12] (between those)
    float* sXbar = sN + kHP;             // [12]        ensemble mean

    const int tiles_x = (A.nx + kWCW - 1) / kWCW;
    const int tile = blockIdx.x;
    const int x0 = (tile % tiles_x) * kWCW;
    const int y0 = (A.tile_y0 + tile / tiles_x) * kWCH;

    // rows [r0, r0 + 32) of eigenvector k, carried from point to point: in registers for
    // the tensor-core Gram; for the FP32 Gram in this thread's half column of sA, which
    // nothing between one point's transform and the next point's warm start rewrites
    float vv[kHalf];
#pragma unroll
    for (int l = 0; l < kHalf; l++) vv[l] = (r0 + l == k) ? 1.f : 0.f;
    if constexpr (!TC) {
#pragma unroll
        for (int l = 0; l < kHalf; l += 4)
            *reinterpret_cast<float4*>(sA + sa_chunk(2 * k + h, l >> 2)) = make_float4(vv[l], vv[l + 1], vv[l + 2], vv[l + 3]);
    }
    int cached_bi = -1, cached_bj = -1;
    int max_sweeps = 0, noconv = 0, total_sweeps = 0;
    bool bad = false;

    for (int idx = 0; idx < kWCW * kWCH; idx++) {
        const int rr_ = idx / kWCW;
        const int cc = (rr_ & 1) ? (kWCW - 1 - idx % kWCW) : (idx % kWCW);
        const int i = x0 + cc, j = y0 + rr_;
        const bool active = (i < A.nx) && (j < A.ny);  // uniform within the CTA
        if (!active) continue;
        const int point = i + A.nx * j;

        // 1. X, xbar, dX (letkf_solver.h:278-280); the h = 0 thread of a column loads it
        {
            float xq[kQ];
#pragma unroll
            for (int q = 0; q < kQ; q++) {
                xq[q] = (real_k && h == 0) ? __ldg(fin + (size_t(k) * kQ + q) * A.nxy + point) : 0.f;
                const float part = warp_sum(xq[q]);
                if (lane == 0) sRed[warp * 12 + q] = part;
            }
            __syncthreads();
            if (h == 0)
#pragma unroll
                for (int q = 0; q < kQ; q++) {
                    const float xb = (sRed[q] + sRed[12 + q] + sRed[24 + q] + sRed[36 + q]) / float(M);
                    sDX[q * kHP + hx(k)] = real_k ? xq[q] - xb : 0.f;
                    if (k == 0) sXbar[q] = xb;
                }
        }

        // 2. observation window of the point's p x p block, once per block
        const int bi = i / A.p, bj = j / A.p;
        if ((TC || !A.qin) && (bi != cached_bi || bj != cached_bj)) {  // the tensor-core Gram needs no window
            for (int b = 0; b < A.nox; b++) {
                int sj = (bj + b - A.nl_off) % A.nsy;
                sj += sj < 0 ? A.nsy : 0;
                for (int a = 0; a < A.nox; a++) {
                    int si = (bi + a - A.nl_off) % A.nsx;
                    si += si < 0 ? A.nsx : 0;
                    const int site = si + A.nsx * sj;
                    for (int var = h; var < 3; var += 2) {
                        const int sl = a + A.nox * b + var * nox2;
                        sW[sl * kHP + hx(k)] = real_k ? __ldg(dY + (size_t(var) * A.nsites + site) * M + k) : 0.f;
                        if (k == 0) sDyo[sl] = __ldg(dyo + size_t(var) * A.nsites + site);
                    }
                }
            }
            cached_bi = bi;
            cached_bj = bj;
        }
        __syncthreads();

        // 3. Gram: rows [r0, r0 + 32) of column k, and c_k (letkf_solver.h:252-254)
        const int pat = (i % A.p) + A.p * (j % A.p);
        const int cnt = wcnt[pat];
        const int4* ent = wtab + size_t(pat) * nobs;
        float qv[kHalf];
#pragma unroll
        for (int l = 0; l < kHalf; l++) qv[l] = 0.f;
        float ck = 0.f;
        if constexpr (TC) {
            __nv_bfloat16* sCb = reinterpret_cast<__nv_bfloat16*>(sA);
            const int g = lane >> 2, c4 = lane & 3;
            float acc[8][4];
#pragma unroll
            for (int nt = 0; nt < 8; nt++) acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
            float ckp = 0.f;
            for (int ob = 0; ob < cnt; ob += kGramChunk) {
                // stage: thread (k, h) fills entries [ob + 40 h, ob + 40 h + 40) of row k (unrolled,
                // so that several weight-table and window loads are in flight at once)
#pragma unroll 5
                for (int q2 = 0; q2 < kGramChunk / 4; q2++) {
                    const int o2 = kGramChunk / 2 * h + 2 * q2;
                    float v2[2];
#pragma unroll
                    for (int u = 0; u < 2; u++) {
                        const int o = ob + o2 + u;
                        float val = 0.f;
                        if (o < cnt) {
                            const int4 e = ent[o];
                            const float wv = __int_as_float(e.w);
                            const float y = sW[e.x * kHP + hx(k)];
                            ckp = fmaf(wv * y, sDyo[e.x], ckp);
                            val = __int_as_float(e.z) * y;  // sqrt(w), from the table
                        }
                        v2[u] = val;
                    }
                    *reinterpret_cast<__nv_bfloat162*>(sCb + k * kCStride + o2) = __floats2bfloat162_rn(v2[0], v2[1]);
                }
                __syncthreads();
                const __nv_bfloat16* ra = sCb + (16 * warp + g) * kCStride + 2 * c4;
#pragma unroll
                for (int ks = 0; ks < kGramChunk / 16; ks++) {
                    const uint32_t a0 = *reinterpret_cast<const uint32_t*>(ra + 16 * ks);
                    const uint32_t a1 = *reinterpret_cast<const uint32_t*>(ra + 8 * kCStride + 16 * ks);
                    const uint32_t a2 = *reinterpret_cast<const uint32_t*>(ra + 16 * ks + 8);
                    const uint32_t a3 = *reinterpret_cast<const uint32_t*>(ra + 8 * kCStride + 16 * ks + 8);
#pragma unroll
                    for (int nt = 0; nt < 8; nt++) {
                        const __nv_bfloat16* rb = sCb + (8 * nt + g) * kCStride + 16 * ks + 2 * c4;
                        mma_bf16_16816(acc[nt], a0, a1, a2, a3, *reinterpret_cast<const uint32_t*>(rb),
                                       *reinterpret_cast<const uint32_t*>(rb + 8));
                    }
                }
                __syncthreads();  // the staging is read: the next chunk, or Q, may overwrite it
            }
            ck = pair_sum(ckp);
            // Q into the half-column layout of sA: element (row, col) = Q[col][row] by symmetry
#pragma unroll
            for (int nt = 0; nt < 8; nt++)
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    const int row = 16 * warp + g + 8 * (e >> 1), col = 8 * nt + 2 * c4 + (e & 1);
                    const float d = (row == col && row < M) ? A.diag : 0.f;
                    sA[sa_chunk(2 * row + (col >> 5), (col & 31) >> 2) + (col & 3)] = acc[nt][e] + d;
                }
            __syncthreads();
#pragma unroll
            for (int l = 0; l < kHalf; l += 4) {
                const float4 q4 = *reinterpret_cast<const float4*>(sA + sa_chunk(2 * k + h, l >> 2));
                qv[l] = q4.x; qv[l + 1] = q4.y; qv[l + 2] = q4.z; qv[l + 3] = q4.w;
            }
            __syncthreads();  // the warm start below rewrites sA
        }
        if (!TC && A.qin) {  // Q and c from the tensor-core Gram (gram_tc.cu)
            ck = real_k ? __ldg(A.cin + size_t(point) * A.mpq + k) : 0.f;
            const float* qrow = A.qin + (size_t(point) * A.mpq + k) * A.mpq + r0;
#pragma unroll
            for (int l = 0; l < kHalf; l += 4) {
                const float4 q4 = real_k ? __ldg(reinterpret_cast<const float4*>(qrow + l)) : make_float4(0.f, 0.f, 0.f, 0.f);
                qv[l] = q4.x;
                qv[l + 1] = q4.y;
                qv[l + 2] = q4.z;
                qv[l + 3] = q4.w;
            }
        }
        for (int o = 0; !TC && !A.qin && o < cnt; o++) {
            const int4 e = ent[o];
            const float* row = sW + e.x * kHP;
            const float ek = __int_as_float(e.w) * row[hx(k)];
            ck = fmaf(ek, sDyo[e.x], ck);
#pragma unroll
            for (int l = 0; l < kHalf; l += 4) {
                const float4 r4 = *reinterpret_cast<const float4*>(row + hx(r0) + l);
                qv[l + 0] = fmaf(ek, r4.x, qv[l + 0]);
                qv[l + 1] = fmaf(ek, r4.y, qv[l + 1]);
                qv[l + 2] = fmaf(ek, r4.z, qv[l + 2]);
                qv[l + 3] = fmaf(ek, r4.w, qv[l + 3]);
            }
        }
        if (!TC) {
#pragma unroll
            for (int l = 0; l < kHalf; l++)
                if (r0 + l == k && k < M) qv[l] += A.diag;
        }

        // 4. warm start A = Q V_prev: Q's columns go through sA.  Column k of V_prev is in
        //    the registers of the column's two threads: V[32h + c][k] here, V[32(1-h) + c][k]
        //    one lane over; they meet Q's columns 32h + c (half column 65h + 2c of sA) and
        //    32(1-h) + c (half column 64 - 63h + 2c).
        if (idx > 0) {
            if constexpr (!TC) {  // V_prev from this thread's own half column, before Q replaces it
#pragma unroll
                for (int l = 0; l < kHalf; l += 4) {
                    const float4 v4 = *reinterpret_cast<const float4*>(sA + sa_chunk(2 * k + h, l >> 2));
                    vv[l] = v4.x; vv[l + 1] = v4.y; vv[l + 2] = v4.z; vv[l + 3] = v4.w;
                }
            }
#pragma unroll
            for (int l = 0; l < kHalf; l += 4)
                *reinterpret_cast<float4*>(sA + sa_chunk(2 * k + h, l >> 2)) = make_float4(qv[l], qv[l + 1], qv[l + 2], qv[l + 3]);
            __syncthreads();
#pragma unroll
            for (int l = 0; l < kHalf; l++) qv[l] = 0.f;
            const float* qo = sA + sa_chunk(65 * h, 0);
            const float* qt = sA + sa_chunk(64 - 63 * h, 0);
#pragma unroll
            for (int c = 0; c < kHalf; c++) {
                const float vo = vv[c];
                const float vt = __shfl_xor_sync(0xffffffffu, vo, 1);
#pragma unroll
                for (int l = 0; l < kHalf; l += 4) {
                    const float4 a4 = *reinterpret_cast<const float4*>(qo + 2 * c * kHS + l);
                    const float4 b4 = *reinterpret_cast<const float4*>(qt + 2 * c * kHS + l);
                    qv[l + 0] = fmaf(b4.x, vt, fmaf(a4.x, vo, qv[l + 0]));
                    qv[l + 1] = fmaf(b4.y, vt, fmaf(a4.y, vo, qv[l + 1]));
                    qv[l + 2] = fmaf(b4.z, vt, fmaf(a4.z, vo, qv[l + 2]));
                    qv[l + 3] = fmaf(b4.w, vt, fmaf(a4.w, vo, qv[l + 3]));
                }
            }
            __syncthreads();  // sA holds the Jacobi's home slots next
        }

        // 5. one-sided Jacobi on the columns of A, lazily scaled (see analysis_kernel), with
        //    the columns handed between thread quads.  Quad s (threads 4s .. 4s + 3, thread r
        //    holding rows [16 r, 16 r + 16)) rotates one column pair per round: a thread
        //    holds 16 rows of both columns, and the pair's dot product is one quad reduction.
        //    The pairs follow a recursive block ordering: at level L = 0..5 the columns form
        //    blocks of 2H (H = 32 >> L), each split into a fixed half and a shifting half; for
        //    H rounds fixed column i of a block meets shifting column (i + j) mod H, and
        //    between rounds every shifting column moves to the quad below.  The levels cover
        //    every pair once in 32 + 16 + 8 + 4 + 2 + 1 = 63 rounds.  Every column has a home
        //    slot in sA (its two half columns): the quad that hands a column on writes it
        //    there, only if it changed since it was last written, and the next owner reads it
        //    after one barrier.  Per round a pair reads one column and writes at most one.
        int sweeps = 0;
        bool converged = false;
        const float tol2 = A.tol * A.tol, stop2 = A.stop * A.stop;  // the tests below compare squares
        float* sSc = sS;  // [64] column scales during the Jacobi (sS is written after it)
#pragma unroll
        for (int l = 0; l < kHalf; l += 4)
            *reinterpret_cast<float4*>(sA + sa_chunk(2 * k + h, l >> 2)) = make_float4(qv[l], qv[l + 1], qv[l + 2], qv[l + 3]);
        if (h == 0) sSc[k] = 1.f;
        __syncthreads();
        {
            const int s = t >> 2, r = t & 3;
            const int hoff = (r >> 1) * kHS + 16 * (r & 1);  // rows [16 r, 16 r + 16) of a home slot
            float xa[16], xb[16];
            float sa = 1.f, sb = 1.f, na = 0.f, nb = 0.f;
            bool cleanup = false;  // this sweep turns no nearly degenerate pair (see kWideTurn)
            for (int sw = 0; sw < A.max_sweeps; sw++) {
                bool big = false;   // some rotated pair's relative off-diagonal reached sqrt(tol)
                bool wide = false;  // some rotation turned wider than atan(kWideTurn)
                for (int L = 0; L < 6; L++) {
                    const int H = 32 >> L;
                    const int b = s >> (5 - L), i = s & (H - 1);
                    const int ca = 2 * H * b + i;
                    int cb = 2 * H * b + H + i;
                    wide_load16(xa, sA + 2 * ca * kHS + hoff);
                    wide_load16(xb, sA + 2 * cb * kHS + hoff);
                    sa = sSc[ca];
                    sb = sSc[cb];
                    bool dirty_a = false, dirty_b = false;
                    if (L == 0) {  // fold the scales in and recompute the norms once per sweep
                        float pa = 0.f, pb = 0.f;
#pragma unroll
                        for (int l = 0; l < 16; l++) {
                            xa[l] *= sa;
                            xb[l] *= sb;
                            pa = fmaf(xa[l], xa[l], pa);
                            pb = fmaf(xb[l], xb[l], pb);
                        }
                        sa = sb = 1.f;
                        na = quad_sum(pa);
                        nb = quad_sum(pb);
                        dirty_a = dirty_b = true;
                    } else {
                        na = sN[ca];
                        nb = sN[cb];
                    }
                    for (int j = 0; j < H; j++) {
                        float g0 = 0.f, g1 = 0.f;
#pragma unroll
                        for (int l = 0; l < 16; l += 2) { g0 = fmaf(xa[l], xb[l], g0); g1 = fmaf(xa[l + 1], xb[l + 1], g1); }
                        const float g = quad_sum(g0 + g1) * (sa * sb);
                        const bool alow = ca < cb;
                        const float alo = alow ? na : nb, ahi = alow ? nb : na;
                        // |g| > tol sqrt(alo ahi), on squares
                        const float p2 = alo * ahi, g2 = g * g;
                        float tt = 0.f;
                        bool turn = g2 > tol2 * p2;
                        if (turn) {
                            // tt = sign(zeta) / (|zeta| + sqrt(1 + zeta^2)), zeta = d / e, times |e|
                            const float d = ahi - alo, e = 2.f * g;
                            tt = __fdividef(copysignf(fabsf(e), d * e), fabsf(d) + sqrt_approx(fmaf(d, d, e * e)));
                            const bool wt = fabsf(tt) > kWideTurn;  // the quad agrees
                            turn = !(cleanup && wt);
                            wide |= turn && wt;
                        }
                        if (turn) {
                            big |= g2 >= stop2 * p2;
                            const float cs = rsqrtf(fmaf(tt, tt, 1.f));
                            // low column: cs (lo - tt hi); high column: cs (hi + tt lo), with the scales
                            const float slo = alow ? sa : sb, shi = alow ? sb : sa;
                            const float rlo = -tt * __fdividef(shi, slo), rhi = tt * __fdividef(slo, shi);
                            const float ra = alow ? rlo : rhi, rb = alow ? rhi : rlo;
#pragma unroll
                            for (int l = 0; l < 16; l++) {
                                const float a0 = xa[l];
                                xa[l] = fmaf(ra, xb[l], a0);
                                xb[l] = fmaf(rb, a0, xb[l]);
                            }
                            sa *= cs;
                            sb *= cs;
                            const float tg = tt * g;
                            na = alow ? na - tg : na + tg;
                            nb = alow ? nb + tg : nb - tg;
                            dirty_a = dirty_b = true;
                        }
                        if (j + 1 < H) {  // hand the shifting column down, take the one from above
                            if (dirty_b) {
                                wide_store16(sA + 2 * cb * kHS + hoff, xb);
                                if (r == 0) {
                                    sN[cb] = nb;
                                    sSc[cb] = sb;
                                }
                            }
                            // from level 2 on a block's H <= 8 quads are one warp, and only
                            // they touch its columns until the level ends
                            if (L >= 2)
                                __syncwarp();
                            else
                                __syncthreads();
                            cb = 2 * H * b + H + ((i + j + 1) & (H - 1));
                            wide_load16(xb, sA + 2 * cb * kHS + hoff);
                            nb = sN[cb];
                            sb = sSc[cb];
                            dirty_b = false;
                        }
                    }
                    if (dirty_a) {
                        wide_store16(sA + 2 * ca * kHS + hoff, xa);
                        if (r == 0) {
                            sN[ca] = na;
                            sSc[ca] = sa;
                        }
                    }
                    if (dirty_b) {
                        wide_store16(sA + 2 * cb * kHS + hoff, xb);
                        if (r == 0) {
                            sN[cb] = nb;
                            sSc[cb] = sb;
                        }
                    }
                    __syncthreads();
                }
                sweeps = sw + 1;
                // the quadratic stop; after a sweep with a wide turn, one cleanup sweep first
                const bool any_big = __syncthreads_or(big ? 1 : 0) != 0;
                const bool any_wide = __syncthreads_or(wide ? 1 : 0) != 0;
                if (cleanup) {
                    cleanup = false;
                    if (!any_big) {
                        converged = true;
                        break;
                    }
                } else if (!any_big) {
                    if (!any_wide) {
                        converged = true;
                        break;
                    }
                    cleanup = true;
                }
            }
        }
        // the columns of A back into the (k, h) half columns
#pragma unroll
        for (int l = 0; l < kHalf; l += 4) {
            const float4 q4 = *reinterpret_cast<const float4*>(sA + sa_chunk(2 * k + h, l >> 2));
            qv[l] = q4.x; qv[l + 1] = q4.y; qv[l + 2] = q4.z; qv[l + 3] = q4.w;
        }
        const float sc = sSc[k];

        // 6. eigenpair of column k and the transform (letkf_solver.h:288-316)
#pragma unroll
        for (int l = 0; l < kHalf; l++) qv[l] *= sc;
        float lam = 0.f;
        {
            float n0 = 0.f, n1 = 0.f;
#pragma unroll
            for (int l = 0; l < kHalf; l += 2) { n0 = fmaf(qv[l], qv[l], n0); n1 = fmaf(qv[l + 1], qv[l + 1], n1); }
            const float n2 = pair_sum(n0 + n1);
            if (n2 > 0.f) {
                lam = sqrtf(n2);
                const float inv = 1.f / lam;
#pragma unroll
                for (int l = 0; l < kHalf; l++) qv[l] *= inv;
            } else {
#pragma unroll
                for (int l = 0; l < kHalf; l++) qv[l] = (r0 + l == k) ? 1.f : 0.f;
            }
        }
        // qv holds rows [r0, r0 + 32) of v_k: into sA (kept there for the next warm start
        // with the FP32 Gram), and in registers with the tensor-core Gram
        if constexpr (TC) {
#pragma unroll
            for (int l = 0; l < kHalf; l++) vv[l] = qv[l];
        }
#pragma unroll
        for (int l = 0; l < kHalf; l += 4)
            *reinterpret_cast<float4*>(sA + sa_chunk(2 * k + h, l >> 2)) = make_float4(qv[l], qv[l + 1], qv[l + 2], qv[l + 3]);
        if (h == 0) sC[hx(k)] = ck;
        __syncthreads();
        float vc = 0.f;  // (V^T c)_k
#pragma unroll
        for (int l = 0; l < kHalf; l++) vc = fmaf(qv[l], sC[hx(r0) + l], vc);
        vc = pair_sum(vc);
        float dsum[kQ];
#pragma unroll
        for (int q = 0; q < kQ; q++) {
            float d = 0.f;
#pragma unroll
            for (int l = 0; l < kHalf; l++) d = fmaf(sDX[q * kHP + hx(r0) + l], qv[l], d);
            dsum[q] = pair_sum(d);
        }
        __syncthreads();  // every thread has read dX before D overwrites it
        if (h == 0) {
            sY[hx(k)] = real_k ? vc / lam : 0.f;
            sS[hx(k)] = real_k ? A.sqrt_m1 / sqrtf(lam) : 0.f;
#pragma unroll
            for (int q = 0; q < kQ; q++) sDX[q * kHP + hx(k)] = dsum[q];
        }
        __syncthreads();
        // Xa_k = xbar + sum_jj D[:, jj] z_jj, z_jj = sS[jj] V[k][jj] + sY[jj]; halves split jj,
        // the upper half one step out of phase (its V reads then fall in other bank groups)
        float acc[kQ];
#pragma unroll
        for (int q = 0; q < kQ; q++) acc[q] = 0.f;
#pragma unroll 4
        for (int ii = 0; ii < kHalf; ii++) {
            const int jj = r0 + ((ii + h) & (kHalf - 1));
            const float z = fmaf(sS[hx(jj)], sA[sa_chunk(2 * jj + (k >> 5), (k & 31) >> 2) + (k & 3)], sY[hx(jj)]);
#pragma unroll
            for (int q = 0; q < kQ; q++) acc[q] = fmaf(sDX[q * kHP + hx(jj)], z, acc[q]);
        }
#pragma unroll
        for (int q = 0; q < kQ; q++) acc[q] = pair_sum(acc[q]);

        // 7. the analysis member k and its macros (update_xk + lbm2euler)
        if (real_k && h == 0) {
            float xa[kQ];
#pragma unroll
            for (int q = 0; q < kQ; q++) {
                xa[q] = sXbar[q] + acc[q];
                bad |= !(xa[q] == xa[q]);
                fout[(size_t(k) * kQ + q) * A.nxy + point] = xa[q];
            }
            float rsum = 0, mu = 0, mv = 0;
#pragma unroll
            for (int q = 0; q < kQ; q++) rsum += xa[q];
#pragma unroll
            for (int q = 0; q < kQ; q++) { mu += xa[q] * A.c * exq(q); mv += xa[q] * A.c * eyq(q); }
            float* mm = mac + size_t(k) * 3 * A.nxy;
            mm[point] = rsum;
            mm[A.nxy + point] = mu / rsum;
            if (A.write_v) mm[2 * A.nxy + point] = mv / rsum;
        }
        max_sweeps = max(max_sweeps, sweeps);
        total_sweeps += sweeps;
        noconv += converged ? 0 : 1;
        __syncthreads();  // the next point rewrites sDX, sA, sXbar
    }
    if (bad) atomicOr(stats + 2, 1);
    if (t == 0 && total_sweeps > 0) {
        atomicMax(stats + 0, max_sweeps);
        if (noconv) atomicAdd(stats + 1, noconv);
        atomicAdd(stats + 3, total_sweeps);
    }
}

AnaParams make_params(const lbl_ctx* c) {
    AnaParams A{};  // every field zero unless set below
    A.nx = c->P.nx; A.ny = c->P.ny; A.nxy = c->P.nxy; A.M = c->P.M;
    A.p = c->G.p; A.nsx = c->G.nsx; A.nsy = c->G.nsy; A.nsites = c->G.nsx * c->G.nsy;
    A.n_pat_max = c->G.nobs;
    A.nox = c->G.nox;
    A.nl_off = c->G.nl - c->G.off;
    const double beta = c->cfg.letkf_covinf;
    A.diag = float((c->P.M - 1) / beta);
    A.sqrt_m1 = float(std::sqrt(double(c->P.M - 1)));
    A.tol = float(c->cfg.jacobi_tol);
    A.stop = float(std::sqrt(c->cfg.jacobi_tol));
    A.max_sweeps = c->cfg.jacobi_max_sweeps;
    A.qin = c->cfg.gram == LBL_GRAM_TF32X3 ? c->d_Q : nullptr;
    A.mpq = gram_tc_mp(c->P.M);
    A.cin = A.qin ? A.qin + size_t(c->P.nxy) * A.mpq * A.mpq : nullptr;
    A.c = c->P.c;
    A.write_v = c->cfg.compat_stale_v ? 0 : 1;
    A.tile_y0 = 0;
    return A;
}

int pad_pow2(int M) {
    int mp = 4;
    while (mp < M) mp *= 2;
    return mp;
}

template <int MP>
void launch_analysis_mp(const lbl_ctx* c, const float* fin, float* fout, float* mac, cudaStream_t s) {
    const AnaParams A = make_params(c);
    constexpr int GPW = 32 / MP;
    const int warps = 4;
    const int groups_per_cta = warps * GPW;
    const size_t sm = analysis_smem_bytes(A.M, A.n_pat_max);
    const int tiles = ((A.nx + kCW - 1) / kCW) * ((A.ny + kCH - 1) / kCH);
    const int grid = (tiles + groups_per_cta - 1) / groups_per_cta;
    analysis_kernel<MP, false><<<grid, warps * 32, sm, s>>>(fin, fout, mac, c->d_dY, c->d_dyo,
                                                             reinterpret_cast<const int4*>(c->d_wtab),
                                                             c->d_wtab + size_t(4) * c->G.p * c->G.p * c->G.nobs,
                                                             c->d_stats, A, DumpPtrs{});
}

// the matrices of the rows [j0, j1): the tiles that cover them, recomputed exactly
template <int MP>
void launch_dump_mp(const lbl_ctx* c, const float* fin, const DumpPtrs& D, cudaStream_t s) {
    AnaParams A = make_params(c);
    constexpr int GPW = 32 / MP;
    const int warps = 4;
    const int groups_per_cta = warps * GPW;
    const size_t sm = analysis_smem_bytes(A.M, A.n_pat_max);
    const int ty0 = D.j0 / kCH, ty1 = (D.j1 - 1) / kCH + 1;
    A.tile_y0 = ty0;
    const int tiles = ((A.nx + kCW - 1) / kCW) * (ty1 - ty0);
    const int grid = (tiles + groups_per_cta - 1) / groups_per_cta;
    analysis_kernel<MP, true><<<grid, warps * 32, sm, s>>>(fin, nullptr, nullptr, c->d_dY, c->d_dyo,
                                                            reinterpret_cast<const int4*>(c->d_wtab),
                                                            c->d_wtab + size_t(4) * c->G.p * c->G.p * c->G.nobs,
                                                            c->d_stats, A, D);
}

}  // namespace

int analysis_supported(int M) { return M >= 2 && M <= kMaxAnalysisMembers; }

// dynamic shared memory of one analysis CTA (4 warps) for M members and a window of nobs slots
size_t analysis_smem_bytes(int M, int nobs) {
    if (M > 32)  // analysis_wide_kernel: one 64-thread CTA
        return sizeof(float) * (size_t(nobs) * kHP + ((nobs + 3) & ~3) + 2 * kWide * kHS + kQ * kHP + 3 * kHP + 12);
    const int mp = pad_pow2(M);
    const int per_grp = nobs * mp + ((nobs + 3) & ~3) + mp * mp + kQ * mp + 2 * mp + 12;
    return sizeof(float) * size_t(per_grp) * 4 * (32 / mp);
}

// opt in to large dynamic shared memory once per device (not allowed during capture)
int analysis_prepare() {
    const int lim = 200 * 1024;
    int rc = 0;
    rc |= int(cudaFuncSetAttribute(analysis_kernel<4, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
    rc |= int(cudaFuncSetAttribute(analysis_kernel<8, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
    rc |= int(cudaFuncSetAttribute(analysis_kernel<16, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
    rc |= int(cudaFuncSetAttribute(analysis_kernel<32, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
    rc |= int(cudaFuncSetAttribute(analysis_kernel<4, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
    rc |= int(cudaFuncSetAttribute(analysis_kernel<8, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
    rc |= int(cudaFuncSetAttribute(analysis_kernel<16, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
    rc |= int(cudaFuncSetAttribute(analysis_kernel<32, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
    rc |= int(cudaFuncSetAttribute(analysis_wide_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
    rc |= int(cudaFuncSetAttribute(analysis_wide_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
    return rc;
}

void launch_obs_ensemble(const lbl_ctx* c, const float* f, cudaStream_t s) {
    const AnaParams A = make_params(c);
    const int threads = 256;
    const long long total = (long long)A.nsites * 32;
    const int grid = int((total + threads - 1) / threads);
    obs_ensemble_kernel<<<grid, threads, 0, s>>>(f, c->d_yo, c->d_dY, c->d_dyo, A);
}

// sizes (floats) of the 14 dumped matrices for nb points, in the order of kDumpLabels
void dump_sizes(int M, int nobs, size_t nb, size_t* sz) {
    const size_t e = size_t(M), o = size_t(nobs);
    const size_t per[kDumpCount] = {o * e, o, e * e, e * e, kQ * e, kQ * e, e * e, e * e, kQ * e, e * e, kQ * e,
                                    e * e, e * e, e * e};
    for (int i = 0; i < kDumpCount; i++) sz[i] = per[i] * nb;
}

void launch_analysis_dump(const lbl_ctx* c, const float* fin, float* buf, int j0, int j1, cudaStream_t s) {
    const size_t nb = size_t(j1 - j0) * c->P.nx;
    size_t sz[kDumpCount];
    dump_sizes(c->P.M, c->G.nobs, nb, sz);
    float* ptr[kDumpCount];
    for (int i = 0; i < kDumpCount; i++) { ptr[i] = buf; buf += sz[i]; }
    DumpPtrs D{ptr[0], ptr[1], ptr[2], ptr[3], ptr[4], ptr[5], ptr[6], ptr[7], ptr[8], ptr[9], ptr[10], ptr[11],
               ptr[12], ptr[13], j0, j1, j0 * c->P.nx};
    switch (pad_pow2(c->P.M)) {
        case 4: launch_dump_mp<4>(c, fin, D, s); break;
        case 8: launch_dump_mp<8>(c, fin, D, s); break;
        case 16: launch_dump_mp<16>(c, fin, D, s); break;
        case 32: launch_dump_mp<32>(c, fin, D, s); break;
        default: break;
    }
}

void launch_analysis_wide(const lbl_ctx* c, const float* fin, float* fout, float* mac, cudaStream_t s) {
    const AnaParams A = make_params(c);
    const int tiles = ((A.nx + kWCW - 1) / kWCW) * ((A.ny + kWCH - 1) / kWCH);
    const size_t sm = analysis_smem_bytes(A.M, A.n_pat_max);
    const int4* wt = reinterpret_cast<const int4*>(c->d_wtab);
    const int* wc = c->d_wtab + size_t(4) * c->G.p * c->G.p * c->G.nobs;
    if (c->cfg.gram == LBL_GRAM_BF16)
        analysis_wide_kernel<true><<<tiles, kWideThreads, sm, s>>>(fin, fout, mac, c->d_dY, c->d_dyo, wt, wc,
                                                                    c->d_stats, A);
    else
        analysis_wide_kernel<false><<<tiles, kWideThreads, sm, s>>>(fin, fout, mac, c->d_dY, c->d_dyo, wt, wc,
                                                                     c->d_stats, A);
}

void launch_analysis(const lbl_ctx* c, const float* fin, float* fout, float* mac, cudaStream_t s) {
    if (c->cfg.gram == LBL_GRAM_TF32X3) {  // every point's Q on the tensor cores first
        GramTcParams G{};
        G.nx = c->P.nx; G.ny = c->P.ny; G.M = c->P.M; G.p = c->G.p;
        G.nsx = c->G.nsx; G.nsy = c->G.nsy; G.nsites = c->G.nsx * c->G.nsy;
        G.nox = c->G.nox; G.nl_off = c->G.nl - c->G.off; G.nobs = c->G.nobs; G.kpad = (c->G.nobs + 7) & ~7;
        const int mpq = gram_tc_mp(c->P.M);
        launch_gram_tc(G, c->d_dY, c->d_dyo, c->d_wdense, c->d_Q, c->d_Q + size_t(c->P.nxy) * mpq * mpq, c->d_err, s);
    }
    if (c->P.M > 32) {
        launch_analysis_wide(c, fin, fout, mac, s);
        return;
    }
    switch (pad_pow2(c->P.M)) {
        case 4: launch_analysis_mp<4>(c, fin, fout, mac, s); break;
        case 8: launch_analysis_mp<8>(c, fin, fout, mac, s); break;
        case 16: launch_analysis_mp<16>(c, fin, fout, mac, s); break;
        case 32: launch_analysis_mp<32>(c, fin, fout, mac, s); break;
        default: break;
    }
}

namespace {
AnaParams params_from_args(const AnalysisArgs& a) {
    AnaParams A{};  // every field zero unless set below
    A.nx = a.nx; A.ny = a.ny; A.nxy = a.nx * a.ny; A.M = a.M;
    A.p = a.p; A.nsx = a.nx / a.p; A.nsy = a.ny / a.p; A.nsites = A.nsx * A.nsy;
    A.n_pat_max = a.nobs;
    A.nox = a.nox;
    A.nl_off = a.nl_off;
    A.diag = a.diag;
    A.sqrt_m1 = a.sqrt_m1;
    A.tol = a.tol;
    A.stop = std::sqrt(a.tol);
    A.max_sweeps = a.max_sweeps;
    A.qin = nullptr;
    A.cin = nullptr;
    A.mpq = 16;
    A.c = a.c;
    A.write_v = a.write_v;
    A.tile_y0 = 0;
    return A;
}

template <int MP>
void launch_analysis_args_mp(const AnalysisArgs& a, cudaStream_t s) {
    const AnaParams A = params_from_args(a);
    constexpr int GPW = 32 / MP;
    const int warps = 4;
    const int groups_per_cta = warps * GPW;
    const size_t sm = analysis_smem_bytes(A.M, A.n_pat_max);
    const int tiles = ((A.nx + kCW - 1) / kCW) * ((A.ny + kCH - 1) / kCH);
    const int grid = (tiles + groups_per_cta - 1) / groups_per_cta;
    analysis_kernel<MP, false><<<grid, warps * 32, sm, s>>>(a.f_in, a.f_out, a.mac_out, a.dY, a.dyo,
                                                             reinterpret_cast<const int4*>(a.wtab),
                                                             a.wtab + size_t(4) * a.p * a.p * a.nobs, a.stats, A,
                                                             DumpPtrs{});
}
}  // namespace

void launch_obs_ensemble_args(const AnalysisArgs& a, cudaStream_t s) {
    const AnaParams A = params_from_args(a);
    const int threads = 256;
    const long long total = (long long)A.nsites * 32;
    const int grid = int((total + threads - 1) / threads);
    obs_ensemble_kernel<<<grid, threads, 0, s>>>(a.f_in, a.yo, a.dY, a.dyo, A);
}

void launch_analysis_args(const AnalysisArgs& a, cudaStream_t s) {
    switch (pad_pow2(a.M)) {
        case 4: launch_analysis_args_mp<4>(a, s); break;
        case 8: launch_analysis_args_mp<8>(a, s); break;
        case 16: launch_analysis_args_mp<16>(a, s); break;
        case 32: launch_analysis_args_mp<32>(a, s); break;
        default: break;
    }
}

}  // namespace lbl
