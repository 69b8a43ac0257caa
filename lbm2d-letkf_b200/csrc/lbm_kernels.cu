// lbm_kernels.cu -- D2Q9 BGK + Smagorinsky forecast kernels for sm_100a.
//
// This translation unit is compiled with -use_fast_math, like the reference
// (config/makefile.compiler.in:42), so that the forcing sin/cos, the Smagorinsky
// sqrt and the float divisions take the same hardware paths as the reference's
// kernels.  Expressions are written in the reference's evaluation order
// (float / double promotions included) for the same reason.
//
// Kernels
//   ic_velocity_kernel  stream-function initial velocity (data.cu:76-110)
//   force_chunk_kernel  Watanabe-97 random forcing for a chunk of steps (data.cu:317-348)
//   lbm_step_kernel     fused pull streaming + macros + Smagorinsky + BGK + force
//                       (lbm.cu:24-160, lbm.h:31-109, lbm_collision_srt.h:8-16)
//   macros_kernel       rho,u,v moments of f (lbm.h:72-109)
#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <type_traits>

#include "lbl_internal.h"

namespace lbl {
namespace {

__host__ __device__ constexpr int ex_q(int q) { return (q % 3) - 1; }  // config.h:257
__host__ __device__ constexpr int ey_q(int q) { return (q / 3) - 1; }  // config.h:258
__host__ __device__ constexpr float w_q(int q) {                       // config.h:260-263
    return (ex_q(q) * ex_q(q) + ey_q(q) * ey_q(q)) == 0   ? float(4. / 9.)
           : (ex_q(q) * ex_q(q) + ey_q(q) * ey_q(q)) == 1 ? float(1. / 9.)
                                                           : float(1. / 36.);
}

__device__ __forceinline__ float w_q_rt(int q) {
    return q == 4 ? float(4. / 9.) : ((q & 1) ? float(1. / 9.) : float(1. / 36.));
}

// ---------------------------------------------------------------------------
// Population storage: FP32 values, or FP16 deviations f - w_q from the lattice
// weights (the precision form): every load widens to FP32 and every store narrows
// after the FP32 collide, so only the bytes in HBM change.
// ---------------------------------------------------------------------------
template <typename T>
struct Store;
template <>
struct Store<float> {
    static __device__ __forceinline__ float ld(const float* p, float) { return __ldg(p); }
    static __device__ __forceinline__ void st(float* p, float v, float) { *p = v; }
};
template <>
struct Store<__half> {
    static __device__ __forceinline__ float ld(const __half* p, float w) { return w + __half2float(__ldg(p)); }
    static __device__ __forceinline__ void st(__half* p, float v, float w) { *p = __float2half_rn(v - w); }
};

// The D2Q9 helpers below skip the e = 0 terms at compile time (x*0 cannot be folded
// under IEEE rules, yet adding it never changes a finite result), and turn the
// divisions by the constants c, c*c and cs2 into multiplications by host-rounded
// reciprocals, which round identically under -use_fast_math.

// u*ex + v*ey for the lattice direction q
template <int q>
__device__ __forceinline__ float edot(float u, float v) {
    constexpr int ex = ex_q(q), ey = ey_q(q);
    if (ex == 0 && ey == 0) return 0.f;
    if (ex == 0) return ey > 0 ? v : -v;
    if (ey == 0) return ex > 0 ? u : -u;
    return (ex > 0 ? u : -u) + (ey > 0 ? v : -v);
}

// feq (lbm.h:31-39)
template <int q>
__device__ __forceinline__ float feq_q(float rho, float u, float v, float uu0, const Phys& P) {
    const float uc0 = edot<q>(u, v) * P.inv_c;
    return rho * w_q(q) * (float(1.) + float(3.) * uc0 + float(4.5) * uc0 * uc0 - float(1.5) * uu0);
}

// ---------------------------------------------------------------------------
// Arithmetic of the stream-collide.  Every operation below is one explicitly rounded
// IEEE operation (__fadd_rn, __fmul_rn, __fmaf_rn, ...) in a fixed order, so the
// rounding sequence is the one written here rather than a compiler's choice of
// contractions; divisions and square roots follow -use_fast_math, and the relaxation
// time is computed in FP64.  (V is the lane type; the kernels use float.)
// ---------------------------------------------------------------------------
__device__ __forceinline__ float vadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float vsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float vmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float vfma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
template <typename V> __device__ __forceinline__ V splat(float s);
template <> __device__ __forceinline__ float splat<float>(float s) { return s; }
__device__ __forceinline__ float vdiv(float a, float b) { return a / b; }
__device__ __forceinline__ float vneg(float a) { return -a; }

// (u ex + v ey) * s for direction q, the signs folded into the constant
template <int q, typename V>
__device__ __forceinline__ V edot_s(V u, V v, float s) {
    constexpr int ex = ex_q(q), ey = ey_q(q);
    if (ex == 0 && ey == 0) return splat<V>(0.f);
    if (ex == 0) return vmul(v, splat<V>(ey * s));
    if (ey == 0) return vmul(u, splat<V>(ex * s));
    if (ex == ey) return vmul(vadd(u, v), splat<V>(ex * s));
    return vmul(vsub(u, v), splat<V>(ex * s));
}

// rho, u, v of a pulled row (lbm.h:72-109): rho = f0 + f1 + ..., u = sum f c ex / rho
template <typename V>
__device__ __forceinline__ void macros_v(const V (&f)[kQ], V& r, V& u, V& v, float c) {
    r = f[0];
#pragma unroll
    for (int q = 1; q < kQ; q++) r = vadd(r, f[q]);
    V su = vmul(f[0], splat<V>(c * ex_q(0)));  // q = 0, 2, 3, 5, 6, 8 have ex != 0
    su = vfma(f[2], splat<V>(c * ex_q(2)), su);
    su = vfma(f[3], splat<V>(c * ex_q(3)), su);
    su = vfma(f[5], splat<V>(c * ex_q(5)), su);
    su = vfma(f[6], splat<V>(c * ex_q(6)), su);
    su = vfma(f[8], splat<V>(c * ex_q(8)), su);
    V sv = vmul(f[0], splat<V>(c * ey_q(0)));  // q = 0, 1, 2, 6, 7, 8 have ey != 0
    sv = vfma(f[1], splat<V>(c * ey_q(1)), sv);
    sv = vfma(f[2], splat<V>(c * ey_q(2)), sv);
    sv = vfma(f[6], splat<V>(c * ey_q(6)), sv);
    sv = vfma(f[7], splat<V>(c * ey_q(7)), sv);
    sv = vfma(f[8], splat<V>(c * ey_q(8)), sv);
    u = vdiv(su, r);
    v = vdiv(sv, r);
}

// Smagorinsky relaxation rate from the post-stream velocity stencil (lbm.cu:42-60,
// 132-139): S from central differences, nu_t = cs^2 dx^2 sqrt(2 S:S) in double from
// the float S, tau = 0.5 + 3 nu / c / c / dt as one FP64 FMA with the precomputed
// 3/c/c/dt, omega = 1/tau correctly rounded in float.
__device__ __forceinline__ float omega_of(float ss2, const Phys& P) {
    const float ss = sqrtf(ss2);
    const float nus = float(P.les_k * double(ss));
    const float nu = P.nu + nus;
    const float tau = float(fma(double(nu), P.tau_k, 0.5));
    return __frcp_rn(tau);
}
template <typename V>
__device__ __forceinline__ V les_omega_v(V ue, V uw, V ve, V vw, V un, V us, V vn, V vs, const Phys& P) {
    const V k2 = splat<V>(P.inv_two_dx);
    const V ux = vmul(vsub(ue, uw), k2);  // s00
    const V uy = vmul(vsub(un, us), k2);
    const V vx = vmul(vsub(ve, vw), k2);
    const V vy = vmul(vsub(vn, vs), k2);  // s11
    const V s01 = vmul(splat<V>(.5f), vadd(uy, vx));
    V t = vmul(ux, ux);
    t = vfma(s01, s01, t);  // s01 s10
    t = vfma(s01, s01, t);  // s10 s01
    t = vfma(vy, vy, t);
    t = vmul(splat<V>(2.f), t);
    return omega_of(t, P);
}

// BGK toward feq (lbm.h:31-39, lbm_collision_srt.h:8-16) plus the first-order force
// with friction (lbm.h:41-70, lbm.cu:142-147): fx = (fx_ - friction/dt u) dt, ...
// feq_q = rho w_q (1 + 3 uc + 4.5 uc^2 - 1.5 uu0) with uc = e_q.u / c.  Opposite
// directions q and 8 - q share w and see -uc, so each pair evaluates the even part
// E = (1 - 1.5 uu0) + 4.5 uc^2 and the odd part O = 3 uc once, and its force terms
// differ only in sign.
template <int q, typename V>
__device__ __forceinline__ void collide_pair(V& fq, V& fqb, V rw, V u, V v, V c0, V nomega, V gx, V gy,
                                             const Phys& P) {
    const V uc = edot_s<q>(u, v, P.inv_c);
    const V e = vfma(vmul(splat<V>(4.5f), uc), uc, c0);
    const V o = vmul(splat<V>(3.f), uc);
    const V feq = vmul(rw, vadd(e, o)), feqb = vmul(rw, vsub(e, o));
    fq = vfma(nomega, vsub(fq, feq), fq);
    fqb = vfma(nomega, vsub(fqb, feqb), fqb);
    const V fe = edot_s<q>(gx, gy, P.inv_cs2);
    fq = vfma(fe, rw, fq);
    fqb = vfma(vneg(fe), rw, fqb);
}
template <typename V>
__device__ __forceinline__ void collide_v(V (&f)[kQ], V rho, V u, V v, V omega, float fxc, float fyc,
                                          const Phys& P) {
    const V uu0 = vmul(vfma(u, u, vmul(v, v)), splat<V>(P.inv_c2));
    const V c0 = vfma(splat<V>(-1.5f), uu0, splat<V>(1.f));
    const V fx = vmul(vfma(splat<V>(-P.fr_dt), u, splat<V>(fxc)), splat<V>(P.dt));
    const V fy = vmul(vfma(splat<V>(-P.fr_dt), v, splat<V>(fyc)), splat<V>(P.dt));
    const V gx = vmul(splat<V>(P.u_ref), fx), gy = vmul(splat<V>(P.u_ref), fy);
    const V nomega = vneg(omega);
    const V rw_axis = vmul(rho, splat<V>(w_q(1))), rw_diag = vmul(rho, splat<V>(w_q(0)));
    collide_pair<0>(f[0], f[8], rw_diag, u, v, c0, nomega, gx, gy, P);
    collide_pair<1>(f[1], f[7], rw_axis, u, v, c0, nomega, gx, gy, P);
    collide_pair<2>(f[2], f[6], rw_diag, u, v, c0, nomega, gx, gy, P);
    collide_pair<3>(f[3], f[5], rw_axis, u, v, c0, nomega, gx, gy, P);
    const V feq4 = vmul(vmul(rho, splat<V>(w_q(4))), c0);  // uc = 0 at rest
    f[4] = vfma(nomega, vsub(f[4], feq4), f[4]);
}

// the one-member forms the scalar kernels call
__device__ __forceinline__ void collide(float (&f)[kQ], float rho, float u, float v, float omega, float fxc,
                                        float fyc, const Phys& P) {
    collide_v<float>(f, rho, u, v, omega, fxc, fyc, P);
}
__device__ __forceinline__ float les_omega(float ue, float uw, float ve, float vw, float un, float us, float vn,
                                           float vs, const Phys& P) {
    return les_omega_v<float>(ue, uw, ve, vw, un, us, vn, vs, P);
}

// Learned closure: the same central differences as les_omega_v give the features,
// the warp's tensor cores evaluate the MLP for its 32 cells, and the multiplier m
// scales the Smagorinsky eddy viscosity: nu_t = m cs^2 dx^2 |S|.  The strain, |S| and
// the relaxation time are explicitly rounded operations shared by the evaluating and
// the held form, so that every kernel running them (one column or two per thread)
// rounds alike, whatever contractions the compiler would choose.
struct ClosureStrain {
    float ux, uy, vx, vy;
};
__device__ __forceinline__ ClosureStrain closure_strain(float ue, float uw, float ve, float vw, float un, float us,
                                                        float vn, float vs, const Phys& P) {
    return {__fmul_rn(__fsub_rn(ue, uw), P.inv_two_dx), __fmul_rn(__fsub_rn(un, us), P.inv_two_dx),
            __fmul_rn(__fsub_rn(ve, vw), P.inv_two_dx), __fmul_rn(__fsub_rn(vn, vs), P.inv_two_dx)};
}
// |S| = sqrt(2 S:S)
__device__ __forceinline__ float closure_smag(const ClosureStrain& g) {
    const float s12 = __fmul_rn(0.5f, __fadd_rn(g.uy, g.vx));
    const float ss = __fmaf_rn(g.ux, g.ux, __fmaf_rn(__fmul_rn(2.f, s12), s12, __fmul_rn(g.vy, g.vy)));
    return closure_sqrt(__fmul_rn(2.f, ss));
}
// omega = 1/tau, tau = 0.5 + 3 (nu + m nu_smag) / c^2 / dt
__device__ __forceinline__ float closure_relax(float m, float smag, const Phys& P) {
    const float nus = __fmul_rn(m, float(P.les_k * double(smag)));
    const float tau = float(fma(double(__fadd_rn(P.nu, nus)), P.tau_k, 0.5));
    return __frcp_rn(tau);
}
__device__ __forceinline__ float closure_omega(float ue, float uw, float ve, float vw, float un, float us, float vn,
                                               float vs, const Phys& P, const ClosureScales& csc,
                                               const uint32_t* pack, uint32_t* stage, float& m) {
    const ClosureStrain g = closure_strain(ue, uw, ve, vw, un, us, vn, vs, P);
    float feat[kMlpIn];
    closure_features_fast(g.ux, g.uy, g.vx, g.vy, csc, feat);
    m = mlp_forward_warp(pack, stage, feat);
    return closure_relax(m, closure_smag(g), P);
}
// The closure between two evaluations of the network (lbl_set_closure_refresh): the
// cell's multiplier m from the last evaluation, |S| of this step.
__device__ __forceinline__ float closure_omega_held(float ue, float uw, float ve, float vw, float un, float us,
                                                    float vn, float vs, const Phys& P, float m) {
    return closure_relax(m, closure_smag(closure_strain(ue, uw, ve, vw, un, us, vn, vs, P)), P);
}

// ---------------------------------------------------------------------------
// initial velocity from the stream-function modes (data.cu:76-110).  The sum is
// accumulated in a float that receives each FP64 term, exactly like `real utmp`.
// ---------------------------------------------------------------------------
__global__ void ic_velocity_kernel(const double* __restrict__ modes, int n, int nx, int ny,
                                   float* __restrict__ u, float* __restrict__ v) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y;
    if (i >= nx || j >= ny) return;
    const double* kxa = modes;
    const double* kya = modes + n;
    const double* pa = modes + 2 * n;
    const double* tha = modes + 3 * n;
    float utmp = 0, vtmp = 0;
    for (int k = 0; k < n; k++) {
        const double kx = kxa[k], ky = kya[k];
        const float p = float(pa[k]), th = float(tha[k]);
        const double cs = cos(kx * i + ky * j + th);
        utmp += p * ky * cs;
        vtmp += p * -kx * cs;
    }
    u[i + nx * j] = utmp;
    v[i + nx * j] = vtmp;
}

// the global row of local row j: the row itself for a whole grid, shifted and wrapped for a y-slab
__device__ __forceinline__ int global_row(int j, const Phys& P) { return (j + P.y0g) % P.nyg; }

// ---------------------------------------------------------------------------
// Watanabe-97 forcing for `nsteps` consecutive steps (data.cu:317-348).  The
// field does not depend on the member, so it is computed once per step for the
// whole ensemble.  sched[s] is the offset, in the normal pool, of the 4*n normals
// that step s uses (the reference's force_theta_d[i_rand_outdated]).
// ---------------------------------------------------------------------------
__global__ void force_chunk_kernel(const float* __restrict__ pool, const int* __restrict__ sched,
                                   const float* __restrict__ modes, const double* __restrict__ amps, int n,
                                   float* __restrict__ force, int slot0, int cap, Phys P) {
    extern __shared__ double s_amp[];  // ax[n], ay[n] (double), then kx[n], ky[n], r[4n] (float)
    float* s_mode = reinterpret_cast<float*>(s_amp + 2 * n);
    const int s = blockIdx.y;
    const float* rnd = pool + sched[s];
    for (int k = threadIdx.x; k < 2 * n; k += blockDim.x) s_amp[k] = amps[k];
    for (int k = threadIdx.x; k < 2 * n; k += blockDim.x) s_mode[k] = modes[k];
    for (int k = threadIdx.x; k < 4 * n; k += blockDim.x) s_mode[2 * n + k] = rnd[k];
    __syncthreads();
    const int ij = blockIdx.x * blockDim.x + threadIdx.x;
    if (ij >= P.nxy) return;
    const int nx = P.nx;
    const int i = ij % nx, j = global_row(ij / nx, P);
    const float x = float(i - nx / 2) * P.inv_nx;
    const float y = float(j - P.nyg / 2) * P.inv_ny;
    const float* force_kx = s_mode;
    const float* force_ky = s_mode + n;
    const float* force_rand = s_mode + 2 * n;
    float f_x = 0;
    float f_y = 0;
    for (int k = 0; k < n; k++) {
        const float kx = force_kx[k];
        const float ky = force_ky[k];
        const float theta = 2 * M_PI * (kx * x + ky * y);
        const float sine = sin(theta);
        const float cosi = cos(theta);
        const float r[4] = {force_rand[k + 0 * n], force_rand[k + 1 * n], force_rand[k + 2 * n],
                            force_rand[k + 3 * n]};
        // amp*2*M_PI*ky (and *(-kx)) are per-mode FP64 products, precomputed on the host
        // with the same IEEE operations the reference evaluates per cell
        const float inner = (r[0] * kx + r[1] * ky) * sine + (r[2] * kx + r[3] * ky) * cosi;
        f_x += s_amp[k] * inner;
        f_y += s_amp[n + k] * inner;
    }
    float* F = force + size_t((slot0 + s) % cap) * 2 * P.nxy;
    F[ij] = f_x;
    F[P.nxy + ij] = f_y;
}

// ---------------------------------------------------------------------------
// DA_NUDGING (nudging.cu:40-143, DA_OBS_RUV or DA_OBS_UV): every member's f relaxes
// in place toward feq of the observed rho, u, v, f = alpha feq_obs + (1 - alpha) f.
// With DA_XYPRUNE p > 1 the site observations are interpolated bilinearly, the
// weights in FP64 as in the reference; DA_QUADRA restricts the nudged quadrant.
// yo holds the site observations [u, v, rho][site]; mac the current macros (rho is
// taken from the model under DA_OBS_UV).  The macros are not refreshed, as there.
// ---------------------------------------------------------------------------
template <int q, typename T>
__device__ __forceinline__ void nudge_q(T* fm, int nxy, float rho, float u, float v, float uu0, float alpha,
                                        const Phys& P) {
    const float f_calc = Store<T>::ld(fm + q * nxy, w_q(q));
    const float f_obse = feq_q<q>(rho, u, v, uu0, P);
    Store<T>::st(fm + q * nxy, alpha * f_obse + (1 - alpha) * f_calc, w_q(q));
}

template <typename T>
__global__ void nudging_kernel(T* __restrict__ f, const float* __restrict__ mac, const float* __restrict__ yo,
                               Phys P, int p, int nsx, int nsy, float alpha, int quadra, int ruv) {
    const int ij = blockIdx.x * blockDim.x + threadIdx.x;
    const int m = blockIdx.y;
    if (ij >= P.nxy) return;
    const int nx = P.nx, ny = P.ny, nxy = P.nxy;
    const int i = ij % nx, j = ij / nx;
    if (quadra % 2 == 1 && !(i < nx / 2)) return;  // skip_east (nudging.cu:26, 93)
    if (quadra >= 2 && !(j < ny / 2)) return;      // skip_north (nudging.cu:27, 95)
    const int ns = nsx * nsy;
    const float* du = yo;
    const float* dv = yo + ns;
    const float* dr = yo + 2 * ns;
    float u_obse = 0, v_obse = 0, rho_obse = 0;
    if (p == 1) {
        u_obse = du[ij];
        v_obse = dv[ij];
        if (ruv) rho_obse = dr[ij];
    } else {
        // corners (iw, js) .. (iw + p, js + p), periodic: sites of the p-lattice
        const int iw = (i / p) * p, js = (j / p) * p;
        const int sw = iw / p, se = (sw + 1) % nsx, ss = js / p, sn = (ss + 1) % nsy;
        const int ij0 = sw + nsx * ss, ije = se + nsx * ss, ijn = sw + nsx * sn, ijen = se + nsx * sn;
        const float ir = (i - iw) / float(p);
        const float jr = (j - js) / float(p);
        u_obse = (1. - ir) * (1. - jr) * du[ij0] + ir * (1. - jr) * du[ije] + (1. - ir) * jr * du[ijn] +
                 ir * jr * du[ijen];
        v_obse = (1. - ir) * (1. - jr) * dv[ij0] + ir * (1. - jr) * dv[ije] + (1. - ir) * jr * dv[ijn] +
                 ir * jr * dv[ijen];
        if (ruv)
            rho_obse = (1. - ir) * (1. - jr) * dr[ij0] + ir * (1. - jr) * dr[ije] + (1. - ir) * jr * dr[ijn] +
                       ir * jr * dr[ijen];
    }
    if (!ruv) rho_obse = mac[size_t(m) * 3 * nxy + ij];  // DA_OBS_UV: rho_calc (nudging.cu:128-131)
    const float uu0 = (u_obse * u_obse + v_obse * v_obse) * P.inv_c2;
    T* fm = f + size_t(m) * kQ * nxy + ij;
    nudge_q<0>(fm, nxy, rho_obse, u_obse, v_obse, uu0, alpha, P);
    nudge_q<1>(fm, nxy, rho_obse, u_obse, v_obse, uu0, alpha, P);
    nudge_q<2>(fm, nxy, rho_obse, u_obse, v_obse, uu0, alpha, P);
    nudge_q<3>(fm, nxy, rho_obse, u_obse, v_obse, uu0, alpha, P);
    nudge_q<4>(fm, nxy, rho_obse, u_obse, v_obse, uu0, alpha, P);
    nudge_q<5>(fm, nxy, rho_obse, u_obse, v_obse, uu0, alpha, P);
    nudge_q<6>(fm, nxy, rho_obse, u_obse, v_obse, uu0, alpha, P);
    nudge_q<7>(fm, nxy, rho_obse, u_obse, v_obse, uu0, alpha, P);
    nudge_q<8>(fm, nxy, rho_obse, u_obse, v_obse, uu0, alpha, P);
}

// x rounded to the nearest float (ties to even), kept in FP64: the FP64 -> FP32 -> FP64
// round trip of a float accumulator.  C = 1.5 * 2^(e+29), with 2^e <= |x| < 2^(e+1)
// taken from x's exponent field, puts x + C in a binade whose ulp is x's float ulp;
// C is a multiple of that ulp with an even significand, so the FP64 addition rounds
// x to float precision with ties to even, and subtracting C back is exact.  Valid
// for finite x with |x| in the normal float range or zero (partial force sums are
// O(1e-3..1)).
__device__ __forceinline__ double round_to_float(double x) {
    const int c_hi = (__double2hiint(x) & 0x7FF00000) + 0x01D80000;  // exponent + 29, significand 1.5
    const double c = __hiloint2double(c_hi, 0);
    return __dadd_rn(__dadd_rn(x, c), -c);
}

// The same forcing with the step loop inside the thread.  theta, sin and cos depend
// only on the cell and the mode, so each thread evaluates them once for its cell and
// keeps them in registers (at most kRegModes modes); the per-step random
// combinations (r0 kx + r1 ky, r2 kx + r3 ky) are staged in shared memory for the
// CTA's steps, and the FP64 amplitudes travel as kernel parameters (constant-bank
// operands).  Two steps advance together for instruction-level parallelism.  Every
// expression keeps the reference's shape and the accumulators keep its float
// rounding after each mode, so the field is the one above.
constexpr int kRegModes = 32;
constexpr int kForceSteps = 4;  // steps a thread advances together (256^2 x 16 analysis phase 0.630 against 0.632 ms with 2)
struct ForceAmps {
    double ax[kRegModes], ay[kRegModes];  // amp*2*pi*ky, amp*2*pi*(-kx)
};

template <int NS>
__device__ __forceinline__ void force_steps(const float2* __restrict__ ab, int n, const float (&sn)[kRegModes],
                                            const float (&cn)[kRegModes], const ForceAmps& A, double (&fx)[NS],
                                            double (&fy)[NS]) {
#pragma unroll
    for (int t = 0; t < NS; t++) fx[t] = fy[t] = 0;
#pragma unroll
    for (int k = 0; k < kRegModes; k++) {
        if (k < n) {
#pragma unroll
            for (int t = 0; t < NS; t++) {
                const float2 c = ab[t * n + k];
                const float inner = c.x * sn[k] + c.y * cn[k];
                fx[t] = round_to_float(fx[t] + A.ax[k] * inner);
                fy[t] = round_to_float(fy[t] + A.ay[k] * inner);
            }
        }
    }
}

__global__ void __launch_bounds__(256) force_chunk_reg_kernel(const float* __restrict__ pool,
                                                              const int* __restrict__ sched,
                                                              const float* __restrict__ modes, const ForceAmps amps,
                                                              int n, int nsteps, int steps_per_cta,
                                                              float* __restrict__ force, int slot0, int cap, Phys P) {
    extern __shared__ float2 s_ab[];  // (A, B)[steps_per_cta][n]
    const int s0 = blockIdx.y * steps_per_cta;
    const int ns = min(steps_per_cta, nsteps - s0);
    for (int e = threadIdx.x; e < ns * n; e += blockDim.x) {
        const int ls = e / n, k = e - ls * n;
        const float* r = pool + sched[s0 + ls];
        const float kx = modes[k], ky = modes[n + k];
        const float a = r[k] * kx + r[n + k] * ky;
        const float b = r[2 * n + k] * kx + r[3 * n + k] * ky;
        s_ab[e] = make_float2(a, b);
    }
    __syncthreads();
    const int ij = blockIdx.x * blockDim.x + threadIdx.x;
    if (ij >= P.nxy) return;
    const int nx = P.nx;
    const int i = ij % nx, j = global_row(ij / nx, P);
    const float x = float(i - nx / 2) * P.inv_nx;
    const float y = float(j - P.nyg / 2) * P.inv_ny;
    float sn[kRegModes], cn[kRegModes];
#pragma unroll
    for (int k = 0; k < kRegModes; k++) {
        if (k < n) {
            const float kx = modes[k];
            const float ky = modes[n + k];
            const float theta = 2 * M_PI * (kx * x + ky * y);
            sn[k] = sin(theta);
            cn[k] = cos(theta);
        }
    }
    int ls = 0;
    for (; ls + kForceSteps - 1 < ns; ls += kForceSteps) {
        double fx[kForceSteps], fy[kForceSteps];
        force_steps<kForceSteps>(s_ab + ls * n, n, sn, cn, amps, fx, fy);
#pragma unroll
        for (int t = 0; t < kForceSteps; t++) {
            float* F = force + size_t((slot0 + s0 + ls + t) % cap) * 2 * P.nxy;
            F[ij] = float(fx[t]);
            F[P.nxy + ij] = float(fy[t]);
        }
    }
    for (; ls < ns; ls++) {
        double fx[1], fy[1];
        force_steps<1>(s_ab + ls * n, n, sn, cn, amps, fx, fy);
        float* F = force + size_t((slot0 + s0 + ls) % cap) * 2 * P.nxy;
        F[ij] = float(fx[0]);
        F[P.nxy + ij] = float(fy[0]);
    }
}

// ---------------------------------------------------------------------------
// Fused LBM step.  One CTA = one member x one strip of TY rows, one thread per
// column x.  Each thread marches up its column: it pulls row j+2 (prefetched one
// row ahead), computes that row's post-stream macros, shares u,v through a 3-row
// shared-memory ring for the x+-1 neighbours, and finalises row j (Smagorinsky
// from the post-stream u,v stencil, BGK toward feq, first-order force with
// friction) straight from registers.  Rows j0-1 and j1 are pulled as halo so that
// the whole step is one pass over f: 72 B/cell of compulsory traffic in FP32.
// NX > 0 fixes the (square) grid at compile time so that plane and row offsets are
// immediates; NX < 0 fixes only nx = -NX (a y-slab's band: ny and the plane stride from
// P); NX = 0 reads nx, ny from P.
// ---------------------------------------------------------------------------
// (256 threads: the plain kernel is held to 4 CTAs per SM, 64 registers, the closure variant
// to 2, 128 registers)
// CL: the learned closure evaluates its network in every cell (and stores the cell's
// multiplier in mclos when given); CLH: the closure between evaluations, with the
// multipliers held in mclos.
template <bool WRITE_MAC, int MAXT, int NX, typename T, bool CL = false, bool CLU = false, bool CLH = false>
__global__ void __launch_bounds__(MAXT, MAXT == 256 ? (CL ? 2 : 4) : 1)
    lbm_step_kernel(const T* __restrict__ fin, T* __restrict__ fout, const float* __restrict__ force,
                    float* __restrict__ mac, Phys P, int TY, const uint32_t* __restrict__ cpack, ClosureScales csc,
                    float* __restrict__ mclos) {
    // CLU: rows wider than one CTA.  The cluster's CTAs (blockIdx.z = chunk) each take
    // blockDim.x columns of the same strip and read the (u, v) of the neighbour
    // columns across a chunk edge from the neighbour CTA's ring (distributed shared
    // memory); the per-row barrier becomes a cluster barrier.
    extern __shared__ float s_uv[];  // [3][2][W]; CL: + packed closure + per-warp staging
    // Programmatic dependent launch (a no-op for an ordinary launch): the previous
    // step's grid is complete, its populations written, before any is read or written
    // here; then the next step's CTAs may start launching into the slots this grid
    // frees, so the launch gap between steps overlaps this grid's tail.
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" :::);
    const int nx = NX ? (NX < 0 ? -NX : NX) : P.nx, ny = NX > 0 ? NX : P.ny, nxy = NX > 0 ? NX * NX : P.nxy;
    const int W = CLU ? int(blockDim.x) : nx;  // columns of this CTA
    const int xl = threadIdx.x;
    const int x = CLU ? int(blockIdx.z) * W + xl : xl;
    uint32_t* s_pack = reinterpret_cast<uint32_t*>(s_uv + 6 * W);
    uint32_t* s_stage = s_pack + kPackWords + (xl >> 5) * kStageWords;
    if (CL) {
        for (int k = xl; k < kPackWords; k += W) s_pack[k] = cpack[k];
        // made visible by the barrier of the first row
    }
    // ring columns of the x-1 / x+1 neighbours and the cluster ranks that hold them
    int lxm = xl == 0 ? W - 1 : xl - 1, lxp = xl == W - 1 ? 0 : xl + 1;
    unsigned rank_m = 0, rank_p = 0;
    if (CLU) {
        const unsigned C = gridDim.z, r = blockIdx.z;
        rank_m = xl == 0 ? (r + C - 1) % C : r;
        rank_p = xl == W - 1 ? (r + 1) % C : r;
    }
    const int m = blockIdx.y;
    const int j0 = blockIdx.x * TY;
    const int j1 = min(j0 + TY, ny);
    const T* __restrict__ fm = fin + size_t(m) * kQ * nxy;
    T* __restrict__ fo = fout + size_t(m) * kQ * nxy + x;
    const int xm = (x == 0) ? nx - 1 : x - 1;
    const int xp = (x == nx - 1) ? 0 : x + 1;
    const float* __restrict__ Fx = force + x;
    const float* __restrict__ Fy = force + nxy + x;

    // running row offsets (row*nx) of rows jj-1, jj, jj+1 for the row jj being pulled
    auto wrap_row = [&](int r) { return (r < 0 ? r + ny : (r >= ny ? r - ny : r)) * nx; };
    int o_m = wrap_row(j0 - 2), o_0 = wrap_row(j0 - 1), o_p = wrap_row(j0);
    auto advance = [&]() {
        o_m = o_0;
        o_0 = o_p;
        o_p = (o_p + nx == nxy) ? 0 : o_p + nx;
    };
    // pull streaming: fc[q] = f[(i-ex, j-ey)] periodic (lbm.cu:82-87)
    auto pull = [&](float (&fc)[kQ]) {
#pragma unroll
        for (int q = 0; q < kQ; q++) {
            const int col = ex_q(q) == -1 ? xp : (ex_q(q) == 0 ? x : xm);
            const int row = ey_q(q) == -1 ? o_p : (ey_q(q) == 0 ? o_0 : o_m);
            fc[q] = Store<T>::ld(fm + q * nxy + row + col, w_q(q));
        }
    };
    // Three row slots rotate roles (A = row being finalised, B = next row, C = the row
    // after, prefetched); the march is unrolled by three so that the rotation is a
    // renaming of registers, not a copy.  Slot k's (u, v) also lives in the shared
    // ring s_uv[k]; u[c], v[c] hold the row below A (the previous A).
    float f[3][kQ], r[3], u[3], v[3];
    {  // halo row below the strip: only its u,v (own column) are needed
        pull(f[2]);
        float rr;
        macros_v(f[2], rr, u[2], v[2], P.c);
    }
    advance();
    pull(f[0]);  // row j0
    macros_v(f[0], r[0], u[0], v[0], P.c);
    s_uv[xl] = u[0];
    s_uv[W + xl] = v[0];
    advance();
    pull(f[1]);  // row j0+1
    int ij = j0 * nx;

    auto row = [&](float (&fa)[kQ], float (&fb)[kQ], float (&fc)[kQ], float& ra, float& ua, float& va, float& rb,
                   float& ub, float& vb, float uc, float vc, float* sa, float* sb, int jc) {
        advance();
        if (jc + 2 <= j1) pull(fc);  // prefetch the row after next
        macros_v(fb, rb, ub, vb, P.c);
        sb[xl] = ub;
        sb[W + xl] = vb;
        const float* am = sa;
        const float* ap = sa;
        if constexpr (CLU) {
            cooperative_groups::this_cluster().sync();
            am = cooperative_groups::this_cluster().map_shared_rank(sa, rank_m);
            ap = cooperative_groups::this_cluster().map_shared_rank(sa, rank_p);
        } else {
            __syncthreads();
        }
        float omega;
        if constexpr (CL) {
            float mm;
            omega = closure_omega(ap[lxp], am[lxm], ap[W + lxp], am[W + lxm], ub, uc, vb, vc, P, csc, s_pack,
                                  s_stage, mm);
            if (mclos) mclos[size_t(m) * nxy + ij + x] = mm;
        } else if constexpr (CLH) {
            omega = closure_omega_held(ap[lxp], am[lxm], ap[W + lxp], am[W + lxm], ub, uc, vb, vc, P,
                                       __ldg(mclos + size_t(m) * nxy + ij + x));
        } else {
            omega = les_omega(ap[lxp], am[lxm], ap[W + lxp], am[W + lxm], ub, uc, vb, vc, P);
        }
        collide(fa, ra, ua, va, omega, Fx[ij], Fy[ij], P);
#pragma unroll
        for (int q = 0; q < kQ; q++) Store<T>::st(fo + q * nxy + ij, fa[q], w_q(q));
        if (WRITE_MAC) {
            float* mm = mac + size_t(m) * 3 * nxy + x;
            mm[ij] = ra;
            mm[nxy + ij] = ua;
            mm[2 * nxy + ij] = va;
        }
        ij += nx;
    };
    float* s0 = s_uv;
    float* s1 = s_uv + 2 * W;
    float* s2 = s_uv + 4 * W;
    for (int jc = j0; jc < j1; jc += 3) {
        row(f[0], f[1], f[2], r[0], u[0], v[0], r[1], u[1], v[1], u[2], v[2], s0, s1, jc);
        if (jc + 1 < j1) row(f[1], f[2], f[0], r[1], u[1], v[1], r[2], u[2], v[2], u[0], v[0], s1, s2, jc + 1);
        if (jc + 2 < j1) row(f[2], f[0], f[1], r[2], u[2], v[2], r[0], u[0], v[0], u[1], v[1], s2, s0, jc + 2);
    }
    // the neighbours may still read this CTA's ring: leave together
    if constexpr (CLU) cooperative_groups::this_cluster().sync();
}

// ---------------------------------------------------------------------------
// Vector-load stream-collide: lbm_step_kernel's column march with each thread owning
// VW consecutive columns x0 .. x0+VW-1.  Every population row of the pull is one
// VW-wide load of the thread's own columns (FP32 rows: 64 bits at VW = 2, 128 bits
// at VW = 4; FP16 deviations: 32 or 64 bits, widened as Store<__half> does); a direction with
// ex = +1 pulls from x-1, so its VW values shift up by one column in registers and
// the column x0-1 comes in as one scalar load (ex = -1 mirrors that with x0+VW).
// The analysis populations, the macros and the forcing move as VW-wide loads and
// stores too.  The x+-1 stencil of the Smagorinsky term is in registers except at
// the thread's two edge columns, whose (u, v) come through a 3-row shared ring that
// holds one float4 per thread, (u, v) of its first and of its last column.  The
// arithmetic of a cell is lbm_step_kernel's (macros_v, les_omega, collide), so the
// two kernels agree bit for bit.  Row offsets of rows j-2 .. j+1 and the strip
// halos are handled as in lbm_step_kernel.
// ---------------------------------------------------------------------------
template <typename T, int VW>
struct VecIO;
template <>
struct VecIO<float, 2> {
    static __device__ __forceinline__ void ld(const float* p, float (&o)[2], float) {
        const float2 t = __ldg(reinterpret_cast<const float2*>(p));
        o[0] = t.x;
        o[1] = t.y;
    }
    static __device__ __forceinline__ void st(float* p, const float (&o)[2], float) {
        *reinterpret_cast<float2*>(p) = make_float2(o[0], o[1]);
    }
};
template <>
struct VecIO<float, 4> {
    static __device__ __forceinline__ void ld(const float* p, float (&o)[4], float) {
        const float4 t = __ldg(reinterpret_cast<const float4*>(p));
        o[0] = t.x;
        o[1] = t.y;
        o[2] = t.z;
        o[3] = t.w;
    }
    static __device__ __forceinline__ void st(float* p, const float (&o)[4], float) {
        *reinterpret_cast<float4*>(p) = make_float4(o[0], o[1], o[2], o[3]);
    }
};
// FP16 deviations: the values Store<__half> gives, VW at a time (32 or 64 bits)
template <int VW>
struct VecIO<__half, VW> {
    static_assert(VW == 2 || VW == 4, "2 or 4 columns per thread");
    using Word = typename std::conditional<VW == 2, unsigned, uint2>::type;
    static __device__ __forceinline__ void ld(const __half* p, float (&o)[VW], float w) {
        const Word t = __ldg(reinterpret_cast<const Word*>(p));
        const __half2* h = reinterpret_cast<const __half2*>(&t);
#pragma unroll
        for (int k = 0; k < VW / 2; k++) {
            const float2 d = __half22float2(h[k]);
            o[2 * k] = w + d.x;
            o[2 * k + 1] = w + d.y;
        }
    }
    static __device__ __forceinline__ void st(__half* p, const float (&o)[VW], float w) {
        Word t;
        __half2* h = reinterpret_cast<__half2*>(&t);
#pragma unroll
        for (int k = 0; k < VW / 2; k++) h[k] = __halves2half2(__float2half_rn(o[2 * k] - w), __float2half_rn(o[2 * k + 1] - w));
        *reinterpret_cast<Word*>(p) = t;
    }
};

// CLH: the learned closure between two evaluations of its network, each cell's
// multiplier read from mclos (lbm_step_kernel's CLH form, cell for cell)
template <bool WRITE_MAC, int NX, int VW, bool PF, typename T, bool CLH = false>
__global__ void __launch_bounds__(NX ? (NX < 0 ? -NX : NX) / VW : 1024 / VW)
    lbm_step_vec_kernel(const T* __restrict__ fin, T* __restrict__ fout, const float* __restrict__ force,
                        float* __restrict__ mac, Phys P, int TY, const float* __restrict__ mclos) {
    extern __shared__ float4 s_edge[];  // [3][nt]: (u, v) of the first and of the last column
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" :::);
    const int nx = NX ? (NX < 0 ? -NX : NX) : P.nx, ny = NX > 0 ? NX : P.ny, nxy = NX > 0 ? NX * NX : P.nxy;
    const int nt = nx / VW;  // threads of a row
    const int t = threadIdx.x;
    const int x0 = t * VW;
    const int xl = x0 == 0 ? nx - 1 : x0 - 1;    // column x0-1, periodic
    const int xr = x0 + VW == nx ? 0 : x0 + VW;  // column x0+VW, periodic
    const int tm = t == 0 ? nt - 1 : t - 1, tp = t == nt - 1 ? 0 : t + 1;
    const int m = blockIdx.y;
    const int j0 = blockIdx.x * TY;
    const int j1 = min(j0 + TY, ny);
    const T* __restrict__ fm = fin + size_t(m) * kQ * nxy;
    T* __restrict__ fo = fout + size_t(m) * kQ * nxy;

    auto wrap_row = [&](int r) { return (r < 0 ? r + ny : (r >= ny ? r - ny : r)) * nx; };
    int o_m = wrap_row(j0 - 2), o_0 = wrap_row(j0 - 1), o_p = wrap_row(j0);
    auto advance = [&]() {
        o_m = o_0;
        o_0 = o_p;
        o_p = (o_p + nx == nxy) ? 0 : o_p + nx;
    };
    // pull streaming of the thread's VW columns: fc[q][k] = f[(x0+k-ex, j-ey)] (lbm.cu:82-87)
    auto pull = [&](float (&fc)[kQ][VW]) {
#pragma unroll
        for (int q = 0; q < kQ; q++) {
            const int row = ey_q(q) == -1 ? o_p : (ey_q(q) == 0 ? o_0 : o_m);
            const T* b = fm + q * nxy + row;
            float w[VW];
            VecIO<T, VW>::ld(b + x0, w, w_q(q));
            if (ex_q(q) == 0) {
#pragma unroll
                for (int k = 0; k < VW; k++) fc[q][k] = w[k];
            } else if (ex_q(q) == 1) {
                fc[q][0] = Store<T>::ld(b + xl, w_q(q));
#pragma unroll
                for (int k = 1; k < VW; k++) fc[q][k] = w[k - 1];
            } else {
#pragma unroll
                for (int k = 0; k < VW - 1; k++) fc[q][k] = w[k + 1];
                fc[q][VW - 1] = Store<T>::ld(b + xr, w_q(q));
            }
        }
    };
    auto macros_row = [&](const float (&fc)[kQ][VW], float (&r)[VW], float (&u)[VW], float (&v)[VW]) {
#pragma unroll
        for (int k = 0; k < VW; k++) {
            float g[kQ];
#pragma unroll
            for (int q = 0; q < kQ; q++) g[q] = fc[q][k];
            macros_v(g, r[k], u[k], v[k], P.c);
        }
    };
    // finalise row A: Smagorinsky from the ring (A's edge neighbours) and the rows above
    // (B) and below (C), collide, store
    int ij = j0 * nx + x0;
    auto finalise = [&](float (&fa)[kQ][VW], const float (&ra)[VW], const float (&ua)[VW], const float (&va)[VW],
                        const float (&ub)[VW], const float (&vb)[VW], const float (&uc)[VW], const float (&vc)[VW],
                        const float4* sa) {
        const float4 em = sa[tm], ep = sa[tp];  // the neighbours' edge columns of row A
        float fx[VW], fy[VW], mh[VW];
        VecIO<float, VW>::ld(force + ij, fx, 0.f);
        VecIO<float, VW>::ld(force + nxy + ij, fy, 0.f);
        if constexpr (CLH) VecIO<float, VW>::ld(mclos + size_t(m) * nxy + ij, mh, 0.f);
#pragma unroll
        for (int k = 0; k < VW; k++) {
            const float ue = k < VW - 1 ? ua[k + 1] : ep.x, ve = k < VW - 1 ? va[k + 1] : ep.y;
            const float uw = k > 0 ? ua[k - 1] : em.z, vw = k > 0 ? va[k - 1] : em.w;
            float omega;
            if constexpr (CLH)
                omega = closure_omega_held(ue, uw, ve, vw, ub[k], uc[k], vb[k], vc[k], P, mh[k]);
            else
                omega = les_omega(ue, uw, ve, vw, ub[k], uc[k], vb[k], vc[k], P);
            float g[kQ];
#pragma unroll
            for (int q = 0; q < kQ; q++) g[q] = fa[q][k];
            collide(g, ra[k], ua[k], va[k], omega, fx[k], fy[k], P);
#pragma unroll
            for (int q = 0; q < kQ; q++) fa[q][k] = g[q];
        }
#pragma unroll
        for (int q = 0; q < kQ; q++) VecIO<T, VW>::st(fo + q * nxy + ij, fa[q], w_q(q));
        if (WRITE_MAC) {
            float* mm = mac + size_t(m) * 3 * nxy + ij;
            VecIO<float, VW>::st(mm, ra, 0.f);
            VecIO<float, VW>::st(mm + nxy, ua, 0.f);
            VecIO<float, VW>::st(mm + 2 * nxy, va, 0.f);
        }
        ij += nx;
    };
    auto edges = [&](const float (&uu)[VW], const float (&vv)[VW]) {
        return make_float4(uu[0], vv[0], uu[VW - 1], vv[VW - 1]);
    };
    if constexpr (PF) {
        // three row slots rotate roles (A = row being finalised, B = next row, C = the
        // row after, prefetched); the march is unrolled by three so that the rotation is
        // a renaming of registers.  Slot k's edges also live in s_edge[k]; uc, vc hold
        // the row below A.
        float f[3][kQ][VW], r[3][VW], u[3][VW], v[3][VW];
        {  // halo row below the strip: only its u,v are needed
            pull(f[2]);
            float rr[VW];
            macros_row(f[2], rr, u[2], v[2]);
        }
        advance();
        pull(f[0]);  // row j0
        macros_row(f[0], r[0], u[0], v[0]);
        s_edge[t] = edges(u[0], v[0]);
        advance();
        pull(f[1]);  // row j0+1
        auto row = [&](float (&fa)[kQ][VW], float (&fb)[kQ][VW], float (&fc)[kQ][VW], float (&ra)[VW],
                       float (&ua)[VW], float (&va)[VW], float (&rb)[VW], float (&ub)[VW], float (&vb)[VW],
                       const float (&uc)[VW], const float (&vc)[VW], const float4* sa, float4* sb, int jc) {
            advance();
            if (jc + 2 <= j1) pull(fc);  // prefetch the row after next
            macros_row(fb, rb, ub, vb);
            sb[t] = edges(ub, vb);
            __syncthreads();
            finalise(fa, ra, ua, va, ub, vb, uc, vc, sa);
        };
        const float4* s0 = s_edge;
        float4* s1 = s_edge + nt;
        float4* s2 = s_edge + 2 * nt;
        for (int jc = j0; jc < j1; jc += 3) {
            row(f[0], f[1], f[2], r[0], u[0], v[0], r[1], u[1], v[1], u[2], v[2], s0, s1, jc);
            if (jc + 1 < j1) row(f[1], f[2], f[0], r[1], u[1], v[1], r[2], u[2], v[2], u[0], v[0], s1, s2, jc + 1);
            if (jc + 2 < j1) row(f[2], f[0], f[1], r[2], u[2], v[2], r[0], u[0], v[0], u[1], v[1], s2, s_edge, jc + 2);
        }
    } else {
        // two population slots (A, B), no prefetch: row B is pulled in the step that
        // needs its macros.  The march is unrolled by two; the (u, v) of the row below A
        // is a copy, and the ring slot of each row is an index (rows rotate over three).
        float f[2][kQ][VW], r[2][VW], u[2][VW], v[2][VW], uc[VW], vc[VW];
        pull(f[1]);  // halo row below the strip: only its u,v are needed
        macros_row(f[1], r[1], uc, vc);
        advance();
        pull(f[0]);  // row j0
        macros_row(f[0], r[0], u[0], v[0]);
        s_edge[t] = edges(u[0], v[0]);
        int sa = 0;  // ring slot of row A
        auto row = [&](float (&fa)[kQ][VW], float (&fb)[kQ][VW], float (&ra)[VW], float (&ua)[VW],
                       float (&va)[VW], float (&rb)[VW], float (&ub)[VW], float (&vb)[VW]) {
            advance();
            pull(fb);  // row A+1: a strip row or the halo row above
            macros_row(fb, rb, ub, vb);
            const int sb = sa == 2 ? 0 : sa + 1;
            s_edge[sb * nt + t] = edges(ub, vb);
            __syncthreads();
            finalise(fa, ra, ua, va, ub, vb, uc, vc, s_edge + sa * nt);
#pragma unroll
            for (int k = 0; k < VW; k++) {
                uc[k] = ua[k];
                vc[k] = va[k];
            }
            sa = sb;
        };
        for (int jc = j0; jc < j1; jc += 2) {
            row(f[0], f[1], r[0], u[0], v[0], r[1], u[1], v[1]);
            if (jc + 1 < j1) row(f[1], f[0], r[1], u[1], v[1], r[0], u[0], v[0]);
        }
    }
}

// ---------------------------------------------------------------------------
// Batched persistent stream-collide: one launch steps every experiment of a batch
// (own grid, members, buffers, forcing and strip height).  The work items are
// (experiment, member, strip, 128-column chunk); a grid sized to the GPU's resident
// CTA slots takes them from an atomic counter, largest strips first, so uneven
// experiments share one launch per step.  The arithmetic is lbm_step_kernel's.  A
// chunk of a row wider than 128 columns gets the (u, v) of its two edge neighbours
// from its edge threads, which pull and reduce those columns themselves (prefetched
// one row ahead, like the populations); a 128-column row wraps inside the CTA.
// ---------------------------------------------------------------------------
template <bool WRITE_MAC>
__global__ void __launch_bounds__(kBatchW, 8) lbm_batch_step_kernel(const BatchExp* __restrict__ exps, int n_exp,
                                                                int total, int step, int* __restrict__ counter) {
    __shared__ float s_uv[3][2][kBatchW + 2];  // per row slot: u, v with a halo column on each side
    __shared__ int s_item;
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" :::);
    const int xl = threadIdx.x;
    for (;;) {
        __syncthreads();  // the previous item's ring is no longer read
        if (xl == 0) s_item = atomicAdd(counter + step, 1);
        __syncthreads();
        const int item = s_item;
        if (item >= total) break;
        int e = 0;
        while (e + 1 < n_exp && item >= exps[e + 1].item0) e++;
        const BatchExp& E = exps[e];
        const Phys P = E.P;
        const int nx = P.nx, ny = P.ny, nxy = P.nxy, TY = E.ty;
        const int local = item - E.item0;
        const int chunk = local % E.chunks, rest = local / E.chunks;
        const int strip = rest % E.strips, m = rest / E.strips;
        const int x0 = chunk * kBatchW, x = x0 + xl;
        const bool whole = E.chunks == 1;
        // ring slots of the x -1 / x +1 neighbours; edge threads of a chunked row also
        // carry the halo column beside them (hx, at ring slot hs)
        const int lidx = (whole && xl == 0) ? kBatchW : xl;
        const int ridx = (whole && xl == kBatchW - 1) ? 1 : xl + 2;
        const int hx = whole ? -1
                             : (xl == 0 ? (x0 == 0 ? nx - 1 : x0 - 1)
                                        : (xl == kBatchW - 1 ? (x0 + kBatchW == nx ? 0 : x0 + kBatchW) : -1));
        const int hs = xl == 0 ? 0 : kBatchW + 1;
        const int hxm = hx <= 0 ? nx - 1 : hx - 1, hxp = hx == nx - 1 ? 0 : hx + 1;
        const int src = (E.cur + step) & 1;
        const float* __restrict__ fm = E.f[src] + size_t(m) * kQ * nxy;
        float* __restrict__ fo = E.f[src ^ 1] + size_t(m) * kQ * nxy + x;
        float* __restrict__ mac = E.mac[src ^ 1];
        const float* __restrict__ force = E.force + size_t(step) * 2 * nxy;
        const int j0 = strip * TY;
        const int j1 = min(j0 + TY, ny);
        const int xm = (x == 0) ? nx - 1 : x - 1;
        const int xp = (x == nx - 1) ? 0 : x + 1;
        const float* __restrict__ Fx = force + x;
        const float* __restrict__ Fy = force + nxy + x;
        auto wrap_row = [&](int r) { return (r < 0 ? r + ny : (r >= ny ? r - ny : r)) * nx; };
        int o_m = wrap_row(j0 - 2), o_0 = wrap_row(j0 - 1), o_p = wrap_row(j0);
        auto advance = [&]() {
            o_m = o_0;
            o_0 = o_p;
            o_p = (o_p + nx == nxy) ? 0 : o_p + nx;
        };
        auto pull_at = [&](float (&fc)[kQ], int c, int cm, int cp) {
#pragma unroll
            for (int q = 0; q < kQ; q++) {
                const int col = ex_q(q) == -1 ? cp : (ex_q(q) == 0 ? c : cm);
                const int row = ey_q(q) == -1 ? o_p : (ey_q(q) == 0 ? o_0 : o_m);
                fc[q] = Store<float>::ld(fm + q * nxy + row + col, w_q(q));
            }
        };
        float hreg[kQ];  // the halo column's pulled populations, one row ahead
        auto pull = [&](float (&fc)[kQ]) {
            pull_at(fc, x, xm, xp);
            if (hx >= 0) pull_at(hreg, hx, hxm, hxp);
        };
        auto halo = [&](float* sb) {  // the halo column's (u, v) for the row in hreg
            if (hx >= 0) {
                float hr, hu, hv;
                macros_v(hreg, hr, hu, hv, P.c);
                sb[hs] = hu;
                sb[kBatchW + 2 + hs] = hv;
            }
        };
        float f[3][kQ], r[3], u[3], v[3];
        {  // halo row below the strip: only its u,v (own column) are needed
            pull_at(f[2], x, xm, xp);
            float rr;
            macros_v(f[2], rr, u[2], v[2], P.c);
        }
        float* s0 = &s_uv[0][0][0];
        float* s1 = &s_uv[1][0][0];
        float* s2 = &s_uv[2][0][0];
        advance();
        pull(f[0]);  // row j0 (and its halo)
        macros_v(f[0], r[0], u[0], v[0], P.c);
        s0[xl + 1] = u[0];
        s0[kBatchW + 2 + xl + 1] = v[0];
        halo(s0);
        advance();
        pull(f[1]);  // row j0+1
        int ij = j0 * nx;
        auto row = [&](float (&fa)[kQ], float (&fb)[kQ], float (&fc)[kQ], float& ra, float& ua, float& va,
                       float& rb, float& ub, float& vb, float uc, float vc, float* sa, float* sb, int jc) {
            advance();
            halo(sb);  // row B's halo, pulled one row ago, before hreg takes row C's
            if (jc + 2 <= j1) pull(fc);
            macros_v(fb, rb, ub, vb, P.c);
            sb[xl + 1] = ub;
            sb[kBatchW + 2 + xl + 1] = vb;
            __syncthreads();
            const float omega = les_omega(sa[ridx], sa[lidx], sa[kBatchW + 2 + ridx], sa[kBatchW + 2 + lidx], ub, uc, vb,
                                          vc, P);
            collide(fa, ra, ua, va, omega, Fx[ij], Fy[ij], P);
#pragma unroll
            for (int q = 0; q < kQ; q++) Store<float>::st(fo + q * nxy + ij, fa[q], w_q(q));
            if (WRITE_MAC) {
                float* mm = mac + size_t(m) * 3 * nxy + x;
                mm[ij] = ra;
                mm[nxy + ij] = ua;
                mm[2 * nxy + ij] = va;
            }
            ij += nx;
        };
        for (int jc = j0; jc < j1; jc += 3) {
            row(f[0], f[1], f[2], r[0], u[0], v[0], r[1], u[1], v[1], u[2], v[2], s0, s1, jc);
            if (jc + 1 < j1) row(f[1], f[2], f[0], r[1], u[1], v[1], r[2], u[2], v[2], u[0], v[0], s1, s2, jc + 1);
            if (jc + 2 < j1) row(f[2], f[0], f[1], r[2], u[2], v[2], r[0], u[0], v[0], u[1], v[1], s2, s0, jc + 2);
        }
    }
}

// ---------------------------------------------------------------------------
// TMA-fed stream-collide (same arithmetic as lbm_step_kernel).  A producer warp
// streams, for every pulled row jj of the strip (j0-1 .. j1), the nine source rows
// f_q(:, jj - ey_q) into one stage of a shared-memory ring with
// cp.async.bulk.tensor (one bulk copy per plane and 256-column box), signalling a
// `full` mbarrier with the byte count; consumer warps read the pulled populations
// straight from shared memory (x+-1 wrap by index) and release the stage on an
// `empty` mbarrier.  Global loads thus cost one instruction per plane-row instead
// of one per cell.  Every wait is bounded: on timeout the kernel records the stage
// in *err and finishes without touching the ring again.
// ---------------------------------------------------------------------------
constexpr int kStages = 6;
constexpr long long kWaitLimit = 1ll << 22;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.shared::cta.b64 st, [%0];\n}" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n}" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// bounded wait; false (and *err set) when the limit is reached
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err, int code, long long limit) {
    for (long long it = 0; it < limit; it++)
        if (mbar_try_wait(bar, parity)) return true;
    atomicCAS(err, 0, code);
    return false;
}
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void consumer_sync(int nthreads) {
    asm volatile("bar.sync 1, %0;" ::"r"(nthreads) : "memory");
}

template <bool WRITE_MAC, int NX>
__global__ void __launch_bounds__(1024) lbm_step_tma_kernel(const __grid_constant__ CUtensorMap fin_map,
                                                            float* __restrict__ fout,
                                                            const float* __restrict__ force,
                                                            float* __restrict__ mac, Phys P, int TY, int box,
                                                            int* __restrict__ err, int stall) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int nx = NX ? NX : P.nx, ny = NX ? NX : P.ny, nxy = NX ? NX * NX : P.nxy;
    const int ncons = nx;  // consumer threads, one column each
    float* ring = reinterpret_cast<float*>(smem_raw);                 // [kStages][9][nx]
    float* s_uv = ring + size_t(kStages) * kQ * nx;                     // [3][2][nx]
    uint64_t* full = reinterpret_cast<uint64_t*>(s_uv + 6 * nx);        // [kStages]
    uint64_t* empty = full + kStages;                                   // [kStages]
    const int m = blockIdx.y;
    const int j0 = blockIdx.x * TY;
    const int j1 = min(j0 + TY, ny);
    const int nrows = j1 - j0 + 2;  // pulled rows j0-1 .. j1
    const int warp = threadIdx.x >> 5;
    const int nwarps_c = ncons >> 5;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], nwarps_c);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    // stall > 0 (fault injection, lbl_inject): the producer issues no copy and every wait
    // polls at most `stall` times, so the consumers' first waits give up with nothing in flight
    const long long limit = stall > 0 ? stall : kWaitLimit;
    if (warp == nwarps_c) {  // ---------------- producer warp ----------------
        if ((threadIdx.x & 31) == 0) {
            bool ok = true;
            int issued = 0;
            const uint32_t bytes = uint32_t(kQ) * nx * sizeof(float);
            const int rows = stall > 0 ? 0 : nrows;
            for (int i = 0; i < rows && ok; i++) {
                const int s = i % kStages;
                if (i >= kStages) ok = mbar_wait(&empty[s], ((i / kStages) - 1) & 1, err, 1, limit);
                if (!ok) break;
                issued = i + 1;
                mbar_expect_tx(&full[s], bytes);
                const int jj = j0 - 1 + i;
#pragma unroll
                for (int q = 0; q < kQ; q++) {
                    int y = jj - ey_q(q);
                    y += (y < 0) ? ny : 0;
                    y -= (y >= ny) ? ny : 0;
                    float* dst = ring + (size_t(s) * kQ + q) * nx;
                    for (int b = 0; b < nx; b += box) tma_load_3d(dst + b, &fin_map, b, y, m * kQ + q, &full[s]);
                }
            }
            // drain: never leave the CTA with a bulk copy still writing shared memory
            for (int i = max(0, issued - kStages); i < issued; i++)
                mbar_wait(&full[i % kStages], (i / kStages) & 1, err, 2, limit);
        }
        return;
    }

    // ---------------- consumer warps ----------------
    const int x = threadIdx.x;
    const int xm = (x == 0) ? nx - 1 : x - 1;
    const int xp = (x == nx - 1) ? 0 : x + 1;
    float* __restrict__ fo = fout + size_t(m) * kQ * nxy + x;
    const float* __restrict__ Fx = force + x;
    const float* __restrict__ Fy = force + nxy + x;
    bool good = true;
    auto take = [&](int i, float (&fc)[kQ]) {  // pulled populations of ring row i
        const int s = i % kStages;
        if (good) good = mbar_wait(&full[s], (i / kStages) & 1, err, 3, limit);
        const float* st = ring + size_t(s) * kQ * nx;
#pragma unroll
        for (int q = 0; q < kQ; q++) {
            const int col = ex_q(q) == -1 ? xp : (ex_q(q) == 0 ? x : xm);
            fc[q] = st[q * nx + col];
        }
        __syncwarp();
        if ((threadIdx.x & 31) == 0) mbar_arrive(&empty[s]);
    };
    float* s_a = s_uv;
    float* s_b = s_uv + 2 * nx;
    float* s_c = s_uv + 4 * nx;
    float fA[kQ], fB[kQ];
    float rA, uA, vA, rB, uB, vB, uM, vM;
    {
        float t[kQ];
        take(0, t);  // halo row j0-1: u,v only
        float r;
        macros_v(t, r, uM, vM, P.c);
    }
    take(1, fA);  // row j0
    macros_v(fA, rA, uA, vA, P.c);
    s_a[x] = uA;
    s_a[nx + x] = vA;
    int ij = j0 * nx;
    for (int jc = j0; jc < j1; jc++) {
        take(jc - j0 + 2, fB);  // row jc+1
        macros_v(fB, rB, uB, vB, P.c);
        s_b[x] = uB;
        s_b[nx + x] = vB;
        consumer_sync(ncons);

        const float omega = les_omega(s_a[xp], s_a[xm], s_a[nx + xp], s_a[nx + xm], uB, uM, vB, vM, P);
        collide(fA, rA, uA, vA, omega, Fx[ij], Fy[ij], P);
        if (good) {
#pragma unroll
            for (int q = 0; q < kQ; q++) fo[q * nxy + ij] = fA[q];
            if (WRITE_MAC) {
                float* mm = mac + size_t(m) * 3 * nxy + x;
                mm[ij] = rA;
                mm[nxy + ij] = uA;
                mm[2 * nxy + ij] = vA;
            }
        }
        uM = uA; vM = vA;
        rA = rB; uA = uB; vA = vB;
#pragma unroll
        for (int q = 0; q < kQ; q++) fA[q] = fB[q];
        float* t = s_a; s_a = s_b; s_b = s_c; s_c = t;
        ij += nx;
    }
}

// moments of f for every member (lbm2euler-style, letkf.cu:340-355, but with v)
template <typename T>
__global__ void macros_kernel(const T* __restrict__ f, float* __restrict__ mac, Phys P) {
    const int ij = blockIdx.x * blockDim.x + threadIdx.x;
    const int m = blockIdx.y;
    if (ij >= P.nxy) return;
    float fc[kQ];
#pragma unroll
    for (int q = 0; q < kQ; q++) fc[q] = Store<T>::ld(f + (size_t(m) * kQ + q) * P.nxy + ij, w_q(q));
    float r, u, v;
    macros_v(fc, r, u, v, P.c);
    float* mm = mac + size_t(m) * 3 * P.nxy;
    mm[ij] = r;
    mm[P.nxy + ij] = u;
    mm[2 * P.nxy + ij] = v;
}

// The compile-time shape of the plain stream-collide: nx for the square grids it is built
// for, -nx for a y-slab's band of 256 or 512 columns (nx fixed, rows from P), else 0.
int shape_key(const Phys& P) {
    if (P.nx == P.ny) return (P.nx == 64 || P.nx == 128 || P.nx == 256 || P.nx == 512 || P.nx == 1024) ? P.nx : 0;
    return (P.nx == 256 || P.nx == 512) ? -P.nx : 0;
}

// The kernel launch_lbm_step runs for a context (its WRITE_MAC = false form), with its
// block size and dynamic shared memory, for the occupancy query of the strip height.
struct StepKernel {
    const void* fn;
    int threads;
    size_t smem;
};
template <typename T>
StepKernel direct_kernel(const lbl_ctx* c) {
    const Phys& P = c->P;
    const int sq = (P.nx == P.ny) ? P.nx : 0;
    if (P.nx > 1024) {
        const int w = P.nx / cluster_chunks(P.nx);
        const size_t sm = c->closure ? closure_step_smem(w) : sizeof(float) * 6 * w;
        const void* fn = c->closure ? (sq == 2048 ? (const void*)lbm_step_kernel<false, 1024, 2048, T, true, true>
                                                  : (const void*)lbm_step_kernel<false, 1024, 0, T, true, true>)
                                    : (sq == 2048 ? (const void*)lbm_step_kernel<false, 1024, 2048, T, false, true>
                                                  : (const void*)lbm_step_kernel<false, 1024, 0, T, false, true>);
        return {fn, w, sm};
    }
    if (c->closure) {
        const size_t sm = closure_step_smem(P.nx);
        if (sq == 256) return {(const void*)lbm_step_kernel<false, 256, 256, T, true>, P.nx, sm};
        if (P.nx <= 256) return {(const void*)lbm_step_kernel<false, 256, 0, T, true>, P.nx, sm};
        return {(const void*)lbm_step_kernel<false, 1024, 0, T, true>, P.nx, sm};
    }
    const size_t sm = sizeof(float) * 6 * P.nx;
    switch (shape_key(P)) {
        case -256: return {(const void*)lbm_step_kernel<false, 256, -256, T>, P.nx, sm};
        case -512: return {(const void*)lbm_step_kernel<false, 1024, -512, T>, P.nx, sm};
        case 64: return {(const void*)lbm_step_kernel<false, 256, 64, T>, P.nx, sm};
        case 128: return {(const void*)lbm_step_kernel<false, 256, 128, T>, P.nx, sm};
        case 256: return {(const void*)lbm_step_kernel<false, 256, 256, T>, P.nx, sm};
        case 512: return {(const void*)lbm_step_kernel<false, 1024, 512, T>, P.nx, sm};
        case 1024: return {(const void*)lbm_step_kernel<false, 1024, 1024, T>, P.nx, sm};
        default:
            if (P.nx <= 256) return {(const void*)lbm_step_kernel<false, 256, 0, T>, P.nx, sm};
            return {(const void*)lbm_step_kernel<false, 1024, 0, T>, P.nx, sm};
    }
}
template <int VW, bool PF, typename T>
StepKernel vec_kernel_w(const lbl_ctx* c) {
    const Phys& P = c->P;
    const int sq = shape_key(P);
    const void* fn = sq == -256   ? (const void*)lbm_step_vec_kernel<false, -256, VW, PF, T>
                     : sq == -512 ? (const void*)lbm_step_vec_kernel<false, -512, VW, PF, T>
                     : sq == 64   ? (const void*)lbm_step_vec_kernel<false, 64, VW, PF, T>
                     : sq == 128  ? (const void*)lbm_step_vec_kernel<false, 128, VW, PF, T>
                     : sq == 256  ? (const void*)lbm_step_vec_kernel<false, 256, VW, PF, T>
                     : sq == 512  ? (const void*)lbm_step_vec_kernel<false, 512, VW, PF, T>
                     : sq == 1024 ? (const void*)lbm_step_vec_kernel<false, 1024, VW, PF, T>
                                  : (const void*)lbm_step_vec_kernel<false, 0, VW, PF, T>;
    return {fn, P.nx / VW, sizeof(float4) * 3 * (P.nx / VW)};
}
template <typename T>
StepKernel vec_kernel_t(const lbl_ctx* c) {
    if (c->vec == 2) return c->vec_pf ? vec_kernel_w<2, true, T>(c) : vec_kernel_w<2, false, T>(c);
    return c->vec_pf ? vec_kernel_w<4, true, T>(c) : vec_kernel_w<4, false, T>(c);
}
StepKernel vec_kernel(const lbl_ctx* c) { return c->f16 ? vec_kernel_t<__half>(c) : vec_kernel_t<float>(c); }
StepKernel step_kernel(const lbl_ctx* c) {
    const Phys& P = c->P;
    if (c->vec && !c->closure) return vec_kernel(c);
    if (c->use_tma) {
        const int sq = (P.nx == P.ny) ? P.nx : 0;
        const void* fn = sq == 64    ? (const void*)lbm_step_tma_kernel<false, 64>
                         : sq == 128 ? (const void*)lbm_step_tma_kernel<false, 128>
                         : sq == 256 ? (const void*)lbm_step_tma_kernel<false, 256>
                         : sq == 512 ? (const void*)lbm_step_tma_kernel<false, 512>
                                     : (const void*)lbm_step_tma_kernel<false, 0>;
        return {fn, P.nx + 32, lbm_tma_smem(P.nx)};
    }
    return c->f16 ? direct_kernel<__half>(c) : direct_kernel<float>(c);
}

// The closure's held-multiplier steps run the two-column vector-load kernel when the
// context's plain steps do (with the prefetched row, grids up to 256 columns wide), else
// lbm_step_kernel's CLH form.
bool held_vec(const lbl_ctx* c) { return c->vec == 2 && c->vec_pf && c->P.nx <= 256; }
template <typename T>
StepKernel held_kernel_t(const lbl_ctx* c) {
    const Phys& P = c->P;
    const int sq = (P.nx == P.ny) ? P.nx : 0;
    if (held_vec(c))
        return {sq == 256 ? (const void*)lbm_step_vec_kernel<false, 256, 2, true, T, true>
                          : (const void*)lbm_step_vec_kernel<false, 0, 2, true, T, true>,
                P.nx / 2, sizeof(float4) * 3 * (P.nx / 2)};
    const size_t sm = sizeof(float) * 6 * P.nx;
    if (sq == 256) return {(const void*)lbm_step_kernel<false, 256, 256, T, false, false, true>, P.nx, sm};
    if (P.nx <= 256) return {(const void*)lbm_step_kernel<false, 256, 0, T, false, false, true>, P.nx, sm};
    return {(const void*)lbm_step_kernel<false, 1024, 0, T, false, false, true>, P.nx, sm};
}
StepKernel held_kernel(const lbl_ctx* c) { return c->f16 ? held_kernel_t<__half>(c) : held_kernel_t<float>(c); }

// Strip height: fill the GPU's resident CTA slots with as few waves as possible,
// counting the two halo rows each strip pulls.  Queried outside stream capture (at
// context creation and when the closure is switched), for the kernel that runs: an
// occupancy query inside a capture may fail and must not decide the launch shape.
int strip_rows_for(const lbl_ctx* c, const StepKernel& k) {
    const Phys& P = c->P;
    int dev = 0, sms = 148, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k.fn, k.threads, k.smem) != cudaSuccess) {
        (void)cudaGetLastError();
        per_sm = 1;
    }
    const long long slots = (long long)std::max(1, per_sm) * sms;
    int best = 4;
    double best_cost = 1e30;
    for (int ty = 2; ty <= 64; ty++) {
        const long long strips = (long long)P.M * ((P.ny + ty - 1) / ty) * cluster_chunks(P.nx);
        const long long waves = (strips + slots - 1) / slots;
        const double cost = double(waves) * (ty + 1.0);
        if (cost < best_cost - 1e-9) { best_cost = cost; best = ty; }
    }
    return best;
}
int strip_rows(const lbl_ctx* c) { return strip_rows_for(c, step_kernel(c)); }

}  // namespace

void launch_ic_velocity(const double* modes, int n_modes, int nx, int ny, float* u, float* v, cudaStream_t s) {
    dim3 block(128), grid((nx + 127) / 128, ny);
    ic_velocity_kernel<<<grid, block, 0, s>>>(modes, n_modes, nx, ny, u, v);
}

void launch_nudging(const lbl_ctx* c, int buf, const float* mac, cudaStream_t s) {
    const int threads = 256;
    dim3 grid((c->P.nxy + threads - 1) / threads, c->P.M);
    const float alpha = float(c->cfg.da_nud_rate);
    if (c->f16)
        nudging_kernel<__half><<<grid, threads, 0, s>>>(c->h[buf], mac, c->d_yo, c->P, c->G.p, c->G.nsx, c->G.nsy,
                                                        alpha, c->cfg.da_quadra, c->cfg.da_obs_ruv);
    else
        nudging_kernel<float><<<grid, threads, 0, s>>>(c->f[buf], mac, c->d_yo, c->P, c->G.p, c->G.nsx, c->G.nsy,
                                                       alpha, c->cfg.da_quadra, c->cfg.da_obs_ruv);
}

void launch_force_chunk(const lbl_ctx* c, int nsteps, int slot0, cudaStream_t s) {
    const int threads = 256;
    const int cells = (c->P.nxy + threads - 1) / threads;
    const int n = c->n_modes;
    if (n <= kRegModes) {
        // split the steps over enough CTAs to fill the GPU four times over
        int sms = 148, dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const int ys = std::max(1, std::min(nsteps, (4 * sms + cells - 1) / cells));
        const int spc = (nsteps + ys - 1) / ys;
        dim3 grid(cells, (nsteps + spc - 1) / spc);
        const size_t sm = sizeof(float2) * size_t(spc) * n;
        ForceAmps A{};
        for (int k = 0; k < n; k++) { A.ax[k] = c->h_amps[k]; A.ay[k] = c->h_amps[n + k]; }
        force_chunk_reg_kernel<<<grid, threads, sm, s>>>(c->d_pool, c->d_sched, c->d_modes, A, n, nsteps, spc,
                                                         c->d_force, slot0, c->force_cap, c->P);
        return;
    }
    dim3 grid(cells, nsteps);
    const size_t sm = sizeof(double) * 2 * n + sizeof(float) * 6 * n;
    force_chunk_kernel<<<grid, threads, sm, s>>>(c->d_pool, c->d_sched, c->d_modes, c->d_amps, n, c->d_force,
                                                 slot0, c->force_cap, c->P);
}

// one box per row (nx <= 256) or whole 256-column boxes (nx = 512): a partial box would
// write past its plane in the shared ring
bool lbm_tma_supported(int nx) { return (nx >= 32 && nx <= 256 && nx % 32 == 0) || nx == 512; }

size_t lbm_tma_smem(int nx) { return sizeof(float) * (size_t(kStages) * kQ * nx + 6 * nx) + 2 * kStages * sizeof(uint64_t); }

namespace {
template <int NX>
int tma_prepare_nx(int sm) {
    int rc = int(cudaFuncSetAttribute(lbm_step_tma_kernel<false, NX>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
    rc |= int(cudaFuncSetAttribute(lbm_step_tma_kernel<true, NX>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
    return rc;
}

template <int NX>
void launch_tma(const lbl_ctx* c, dim3 grid, int ty, int b, float* fout, const float* force, float* mac_out,
                cudaStream_t s) {
    const Phys& P = c->P;
    const size_t sm = lbm_tma_smem(P.nx);
    const int box = P.nx < 256 ? P.nx : 256;
    if (mac_out)
        lbm_step_tma_kernel<true, NX><<<grid, P.nx + 32, sm, s>>>(c->tmap[b], fout, force, mac_out, P, ty, box, c->d_err,
                                                                   c->inject_tma_stall);
    else
        lbm_step_tma_kernel<false, NX><<<grid, P.nx + 32, sm, s>>>(c->tmap[b], fout, force, nullptr, P, ty, box, c->d_err,
                                                                    c->inject_tma_stall);
}

// a stream-collide launch, with programmatic stream serialization when the previous
// launch on the stream is the previous step (pdl)
template <typename... KArgs, typename... Args>
void launch_step(void (*kernel)(KArgs...), dim3 grid, int threads, size_t sm, cudaStream_t s, bool pdl,
                 Args... args) {
    cudaLaunchConfig_t lc = {};
    lc.gridDim = grid;
    lc.blockDim = dim3(threads);
    lc.dynamicSmemBytes = sm;
    lc.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    lc.attrs = at;
    lc.numAttrs = pdl ? 1 : 0;
    cudaLaunchKernelEx(&lc, kernel, args...);
}

template <int MAXT, int NX, typename T>
void launch_direct_t(const lbl_ctx* c, dim3 grid, int ty, const T* fin, T* fout, const float* force,
                     float* mac_out, cudaStream_t s, bool pdl) {
    const Phys& P = c->P;
    const size_t sm = sizeof(float) * 6 * P.nx;
    if (mac_out)
        launch_step(lbm_step_kernel<true, MAXT, NX, T>, grid, P.nx, sm, s, pdl, fin, fout, force, mac_out, P, ty,
                    static_cast<const uint32_t*>(nullptr), ClosureScales{}, static_cast<float*>(nullptr));
    else
        launch_step(lbm_step_kernel<false, MAXT, NX, T>, grid, P.nx, sm, s, pdl, fin, fout, force,
                    static_cast<float*>(nullptr), P, ty, static_cast<const uint32_t*>(nullptr), ClosureScales{},
                    static_cast<float*>(nullptr));
}

// rows wider than 1024 columns: clusters of cluster_chunks(nx) CTAs per strip
template <bool CL, typename T, int NX>
void launch_cluster_t(const lbl_ctx* c, int strips, int ty, const T* fin, T* fout, const float* force,
                      float* mac_out, cudaStream_t s) {
    const Phys& P = c->P;
    const int C = cluster_chunks(P.nx), W = P.nx / C;
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3(strips, P.M, C);
    lc.blockDim = dim3(W);
    lc.dynamicSmemBytes = CL ? closure_step_smem(W) : sizeof(float) * 6 * W;
    lc.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = 1;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = C;
    lc.attrs = at;
    lc.numAttrs = 1;
    const uint32_t* pk = CL ? c->d_closure : nullptr;
    const ClosureScales sc = CL ? c->closure_sc : ClosureScales{};
    if (mac_out)
        cudaLaunchKernelEx(&lc, lbm_step_kernel<true, 1024, NX, T, CL, true>, fin, fout, force, mac_out, P, ty, pk,
                           sc, static_cast<float*>(nullptr));
    else
        cudaLaunchKernelEx(&lc, lbm_step_kernel<false, 1024, NX, T, CL, true>, fin, fout, force,
                           static_cast<float*>(nullptr), P, ty, pk, sc, static_cast<float*>(nullptr));
}
template <bool CL>
void launch_cluster(const lbl_ctx* c, int strips, int ty, int src, int dst, const float* force, float* mac_out,
                    cudaStream_t s) {
    const bool sq2048 = c->P.nx == 2048 && c->P.ny == 2048;
    if (c->f16) {
        if (sq2048) launch_cluster_t<CL, __half, 2048>(c, strips, ty, c->h[src], c->h[dst], force, mac_out, s);
        else launch_cluster_t<CL, __half, 0>(c, strips, ty, c->h[src], c->h[dst], force, mac_out, s);
    } else {
        if (sq2048) launch_cluster_t<CL, float, 2048>(c, strips, ty, c->f[src], c->f[dst], force, mac_out, s);
        else launch_cluster_t<CL, float, 0>(c, strips, ty, c->f[src], c->f[dst], force, mac_out, s);
    }
}

// learned-closure variant (nx % 32 == 0 and nx <= 1024, checked by lbl_set_closure)
template <int MAXT, int NX, typename T>
void launch_closure_t(const lbl_ctx* c, dim3 grid, int ty, const T* fin, T* fout, const float* force,
                      float* mac_out, cudaStream_t s, bool pdl, bool held) {
    const Phys& P = c->P;
    const uint32_t* pk = c->d_closure;
    float* mc = c->d_mclos;  // null when the network runs every step
    if (held && held_vec(c)) {  // the multipliers of the last evaluation, two columns per thread
        const int nt = P.nx / 2;
        const int tyh = c->ty_held > 0 ? c->ty_held : ty;
        const dim3 gh((P.ny + tyh - 1) / tyh, P.M);
        const size_t sm = sizeof(float4) * 3 * nt;
        if (NX == 256) {
            if (mac_out)
                launch_step(lbm_step_vec_kernel<true, 256, 2, true, T, true>, gh, nt, sm, s, pdl, fin, fout, force,
                            mac_out, P, tyh, static_cast<const float*>(mc));
            else
                launch_step(lbm_step_vec_kernel<false, 256, 2, true, T, true>, gh, nt, sm, s, pdl, fin, fout, force,
                            static_cast<float*>(nullptr), P, tyh, static_cast<const float*>(mc));
        } else {
            if (mac_out)
                launch_step(lbm_step_vec_kernel<true, 0, 2, true, T, true>, gh, nt, sm, s, pdl, fin, fout, force,
                            mac_out, P, tyh, static_cast<const float*>(mc));
            else
                launch_step(lbm_step_vec_kernel<false, 0, 2, true, T, true>, gh, nt, sm, s, pdl, fin, fout, force,
                            static_cast<float*>(nullptr), P, tyh, static_cast<const float*>(mc));
        }
        return;
    }
    if (held) {  // the plain kernel's cost: the multipliers of the last evaluation
        const int tyh = c->ty_held > 0 ? c->ty_held : ty;
        grid = dim3((P.ny + tyh - 1) / tyh, P.M);
        ty = tyh;
        const size_t sm = sizeof(float) * 6 * P.nx;
        if (mac_out)
            launch_step(lbm_step_kernel<true, MAXT, NX, T, false, false, true>, grid, P.nx, sm, s, pdl, fin, fout,
                        force, mac_out, P, ty, pk, c->closure_sc, mc);
        else
            launch_step(lbm_step_kernel<false, MAXT, NX, T, false, false, true>, grid, P.nx, sm, s, pdl, fin, fout,
                        force, static_cast<float*>(nullptr), P, ty, pk, c->closure_sc, mc);
        return;
    }
    const size_t sm = closure_step_smem(P.nx);
    if (mac_out)
        launch_step(lbm_step_kernel<true, MAXT, NX, T, true>, grid, P.nx, sm, s, pdl, fin, fout, force, mac_out, P,
                    ty, pk, c->closure_sc, mc);
    else
        launch_step(lbm_step_kernel<false, MAXT, NX, T, true>, grid, P.nx, sm, s, pdl, fin, fout, force,
                    static_cast<float*>(nullptr), P, ty, pk, c->closure_sc, mc);
}
template <int MAXT, int NX>
void launch_closure(const lbl_ctx* c, dim3 grid, int ty, int src, int dst, const float* force, float* mac_out,
                    cudaStream_t s, bool pdl, bool held) {
    if (c->f16)
        launch_closure_t<MAXT, NX, __half>(c, grid, ty, c->h[src], c->h[dst], force, mac_out, s, pdl, held);
    else
        launch_closure_t<MAXT, NX, float>(c, grid, ty, c->f[src], c->f[dst], force, mac_out, s, pdl, held);
}

// vector-load stream-collide (FP32 storage, nx a multiple of 32 up to 1024)
template <int NX, int VW, bool PF, typename T>
void launch_vec_s(const lbl_ctx* c, dim3 grid, int ty, const T* fin, T* fout, const float* force, float* mac_out,
                  cudaStream_t s, bool pdl) {
    const int nt = c->P.nx / VW;
    const size_t sm = sizeof(float4) * 3 * nt;
    if (mac_out)
        launch_step(lbm_step_vec_kernel<true, NX, VW, PF, T>, grid, nt, sm, s, pdl, fin, fout, force, mac_out, c->P,
                    ty, static_cast<const float*>(nullptr));
    else
        launch_step(lbm_step_vec_kernel<false, NX, VW, PF, T>, grid, nt, sm, s, pdl, fin, fout, force,
                    static_cast<float*>(nullptr), c->P, ty, static_cast<const float*>(nullptr));
}
template <int NX, int VW, bool PF>
void launch_vec_t(const lbl_ctx* c, dim3 grid, int ty, int src, int dst, const float* force, float* mac_out,
                  cudaStream_t s, bool pdl) {
    if (c->f16)
        launch_vec_s<NX, VW, PF, __half>(c, grid, ty, c->h[src], c->h[dst], force, mac_out, s, pdl);
    else
        launch_vec_s<NX, VW, PF, float>(c, grid, ty, c->f[src], c->f[dst], force, mac_out, s, pdl);
}
template <int VW, bool PF>
void launch_vec_w(const lbl_ctx* c, dim3 grid, int ty, int src, int dst, const float* force, float* mac_out,
                  cudaStream_t s, bool pdl) {
    switch (shape_key(c->P)) {
        case -256: launch_vec_t<-256, VW, PF>(c, grid, ty, src, dst, force, mac_out, s, pdl); break;
        case -512: launch_vec_t<-512, VW, PF>(c, grid, ty, src, dst, force, mac_out, s, pdl); break;
        case 64: launch_vec_t<64, VW, PF>(c, grid, ty, src, dst, force, mac_out, s, pdl); break;
        case 128: launch_vec_t<128, VW, PF>(c, grid, ty, src, dst, force, mac_out, s, pdl); break;
        case 256: launch_vec_t<256, VW, PF>(c, grid, ty, src, dst, force, mac_out, s, pdl); break;
        case 512: launch_vec_t<512, VW, PF>(c, grid, ty, src, dst, force, mac_out, s, pdl); break;
        case 1024: launch_vec_t<1024, VW, PF>(c, grid, ty, src, dst, force, mac_out, s, pdl); break;
        default: launch_vec_t<0, VW, PF>(c, grid, ty, src, dst, force, mac_out, s, pdl);
    }
}
void launch_vec(const lbl_ctx* c, dim3 grid, int ty, int src, int dst, const float* force, float* mac_out,
                cudaStream_t s, bool pdl) {
    if (c->vec == 2) {
        if (c->vec_pf) launch_vec_w<2, true>(c, grid, ty, src, dst, force, mac_out, s, pdl);
        else launch_vec_w<2, false>(c, grid, ty, src, dst, force, mac_out, s, pdl);
    } else {
        if (c->vec_pf) launch_vec_w<4, true>(c, grid, ty, src, dst, force, mac_out, s, pdl);
        else launch_vec_w<4, false>(c, grid, ty, src, dst, force, mac_out, s, pdl);
    }
}

template <int MAXT, int NX>
void launch_direct(const lbl_ctx* c, dim3 grid, int ty, int src, int dst, const float* force, float* mac_out,
                   cudaStream_t s, bool pdl) {
    if (c->f16)
        launch_direct_t<MAXT, NX, __half>(c, grid, ty, c->h[src], c->h[dst], force, mac_out, s, pdl);
    else
        launch_direct_t<MAXT, NX, float>(c, grid, ty, c->f[src], c->f[dst], force, mac_out, s, pdl);
}
}  // namespace

int lbm_tma_prepare(int nx) {
    const int sm = int(lbm_tma_smem(nx));
    return tma_prepare_nx<0>(sm) | tma_prepare_nx<64>(sm) | tma_prepare_nx<128>(sm) | tma_prepare_nx<256>(sm) |
           tma_prepare_nx<512>(sm);
}

void launch_lbm_step(const lbl_ctx* c, int src, int dst, const float* force, float* mac_out, cudaStream_t s,
                     bool pdl, int step) {
    const Phys& P = c->P;
    const int sq = (P.nx == P.ny) ? P.nx : 0;

    const int ty = c->ty_tuned > 0 ? c->ty_tuned : (c->ty_default > 0 ? c->ty_default : 4);
    dim3 grid((P.ny + ty - 1) / ty, P.M);
    if (P.nx > 1024) {
        if (c->closure) launch_cluster<true>(c, int(grid.x), ty, src, dst, force, mac_out, s);
        else launch_cluster<false>(c, int(grid.x), ty, src, dst, force, mac_out, s);
        return;
    }
    if (c->use_tma) {
        float* fout = c->f[dst];
        switch (sq) {
            case 64: launch_tma<64>(c, grid, ty, src, fout, force, mac_out, s); break;
            case 128: launch_tma<128>(c, grid, ty, src, fout, force, mac_out, s); break;
            case 256: launch_tma<256>(c, grid, ty, src, fout, force, mac_out, s); break;
            case 512: launch_tma<512>(c, grid, ty, src, fout, force, mac_out, s); break;
            default: launch_tma<0>(c, grid, ty, src, fout, force, mac_out, s); break;
        }
        return;
    }
    if (c->closure) {
        // the network runs on steps 0, k, 2k, ... of a chunk and the multipliers are held between
        const bool held = c->d_mclos && c->closure_every > 1 && step % c->closure_every != 0;
        if (sq == 256) launch_closure<256, 256>(c, grid, ty, src, dst, force, mac_out, s, pdl, held);
        else if (P.nx <= 256) launch_closure<256, 0>(c, grid, ty, src, dst, force, mac_out, s, pdl, held);
        else launch_closure<1024, 0>(c, grid, ty, src, dst, force, mac_out, s, pdl, held);
        return;
    }
    if (c->vec) {
        launch_vec(c, grid, ty, src, dst, force, mac_out, s, pdl);
        return;
    }
    switch (shape_key(P)) {
        case -256: launch_direct<256, -256>(c, grid, ty, src, dst, force, mac_out, s, pdl); break;
        case -512: launch_direct<1024, -512>(c, grid, ty, src, dst, force, mac_out, s, pdl); break;
        case 64: launch_direct<256, 64>(c, grid, ty, src, dst, force, mac_out, s, pdl); break;
        case 128: launch_direct<256, 128>(c, grid, ty, src, dst, force, mac_out, s, pdl); break;
        case 256: launch_direct<256, 256>(c, grid, ty, src, dst, force, mac_out, s, pdl); break;
        case 512: launch_direct<1024, 512>(c, grid, ty, src, dst, force, mac_out, s, pdl); break;
        case 1024: launch_direct<1024, 1024>(c, grid, ty, src, dst, force, mac_out, s, pdl); break;
        default:
            if (P.nx <= 256) launch_direct<256, 0>(c, grid, ty, src, dst, force, mac_out, s, pdl);
            else launch_direct<1024, 0>(c, grid, ty, src, dst, force, mac_out, s, pdl);
    }
}

int lbm_strip_rows(const lbl_ctx* c) { return strip_rows(c); }
int lbm_strip_rows_held(const lbl_ctx* c) { return strip_rows_for(c, held_kernel(c)); }

void launch_batch_step(const BatchExp* exps, int n_exp, int total, int step, int* counter, int grid, bool mac,
                       bool pdl, cudaStream_t s) {
    if (mac)
        launch_step(lbm_batch_step_kernel<true>, dim3(grid), kBatchW, 0, s, pdl, exps, n_exp, total, step, counter);
    else
        launch_step(lbm_batch_step_kernel<false>, dim3(grid), kBatchW, 0, s, pdl, exps, n_exp, total, step, counter);
}

int batch_step_slots() {
    int dev = 0, sms = 148, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lbm_batch_step_kernel<false>, kBatchW, 0) != cudaSuccess) {
        (void)cudaGetLastError();
        per_sm = 1;
    }
    return std::max(1, per_sm) * sms;
}

int cluster_chunks(int nx) {
    if (nx <= 1024) return 1;
    for (int w : {1024, 512, 256})
        if (nx % w == 0 && nx / w <= 8) return nx / w;
    return 0;
}

size_t closure_step_smem(int nx) {
    return sizeof(float) * 6 * nx + sizeof(uint32_t) * (kPackWords + size_t(nx / 32) * kStageWords);
}

// rest state f = w_q rho_ref in every member of both buffers (FP16 storage: deviation 0)
__global__ void rest_kernel(float* f, size_t n, int nxy, float rho) {
    for (size_t e = blockIdx.x * size_t(blockDim.x) + threadIdx.x; e < n; e += size_t(gridDim.x) * blockDim.x)
        f[e] = w_q_rt(int((e / nxy) % kQ)) * rho;
}
void launch_rest_state(const lbl_ctx* c, cudaStream_t s) {
    const size_t n = size_t(c->P.M) * kQ * c->P.nxy;
    for (int b = 0; b < 2; b++) {
        if (c->f16)
            cudaMemsetAsync(c->h[b], 0, sizeof(__half) * n, s);
        else
            rest_kernel<<<4 * 148, 256, 0, s>>>(c->f[b], n, c->P.nxy, float(c->cfg.rho_ref));
    }
}

void launch_macros(const lbl_ctx* c, int buf, float* mac, cudaStream_t s) {
    dim3 grid((c->P.nxy + 255) / 256, c->P.M);
    if (c->f16)
        macros_kernel<__half><<<grid, 256, 0, s>>>(c->h[buf], mac, c->P);
    else
        macros_kernel<float><<<grid, 256, 0, s>>>(c->f[buf], mac, c->P);
}

// FP16 deviation storage <-> FP32 populations over [M][9][ny][nx]: one grid row per
// population plane (q = plane mod 9, so no division per element), eight values per
// thread and iteration (16-byte FP16 and 2 x 16-byte FP32 accesses; nxy is a multiple
// of 256)
__global__ void expand_kernel(const __half* __restrict__ h, float* __restrict__ f, int nxy) {
    const size_t plane = blockIdx.y;
    const float w = w_q_rt(int(plane % kQ));
    const uint4* hp = reinterpret_cast<const uint4*>(h + plane * nxy);
    float4* fp = reinterpret_cast<float4*>(f + plane * nxy);
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nxy / 8; e += gridDim.x * blockDim.x) {
        const uint4 v = __ldg(hp + e);
        const __half2* h2 = reinterpret_cast<const __half2*>(&v);
        float o[8];
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const float2 d = __half22float2(h2[k]);
            o[2 * k] = w + d.x;
            o[2 * k + 1] = w + d.y;
        }
        fp[2 * e] = make_float4(o[0], o[1], o[2], o[3]);
        fp[2 * e + 1] = make_float4(o[4], o[5], o[6], o[7]);
    }
}
__global__ void compress_kernel(const float* __restrict__ f, __half* __restrict__ h, int nxy) {
    const size_t plane = blockIdx.y;
    const float w = w_q_rt(int(plane % kQ));
    const float4* fp = reinterpret_cast<const float4*>(f + plane * nxy);
    uint4* hp = reinterpret_cast<uint4*>(h + plane * nxy);
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nxy / 8; e += gridDim.x * blockDim.x) {
        const float4 a = __ldg(fp + 2 * e), b = __ldg(fp + 2 * e + 1);
        uint4 v;
        __half2* h2 = reinterpret_cast<__half2*>(&v);
        h2[0] = __halves2half2(__float2half_rn(a.x - w), __float2half_rn(a.y - w));
        h2[1] = __halves2half2(__float2half_rn(a.z - w), __float2half_rn(a.w - w));
        h2[2] = __halves2half2(__float2half_rn(b.x - w), __float2half_rn(b.y - w));
        h2[3] = __halves2half2(__float2half_rn(b.z - w), __float2half_rn(b.w - w));
        hp[e] = v;
    }
}

void launch_expand(const lbl_ctx* c, const __half* h, float* f, cudaStream_t s) {
    const int nxy = c->P.nxy;
    dim3 grid(std::max(1, std::min(64, nxy / 8 / 256)), c->P.M * kQ);
    expand_kernel<<<grid, 256, 0, s>>>(h, f, nxy);
}
void launch_compress(const lbl_ctx* c, const float* f, __half* h, cudaStream_t s) {
    const int nxy = c->P.nxy;
    dim3 grid(std::max(1, std::min(64, nxy / 8 / 256)), c->P.M * kQ);
    compress_kernel<<<grid, 256, 0, s>>>(f, h, nxy);
}

}  // namespace lbl
