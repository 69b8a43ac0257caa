// oracle.cpp -- CPU ORACLE (test infrastructure only; never part of the product path).
//
// A plain FP64 C++/OpenMP restatement of the reference's forecast-and-assimilate
// path, used by tests/ to check the CUDA engine, by __graft_entry__.smoke() as the
// checker, and by bench.py as the timed CPU baseline.  Each function cites the
// reference code it follows (paths relative to the reference project):
//
//   initial condition        src/data.cu:25-141   (stdata::init_lbm)
//   forcing mode table       src/data.cu:161-237  (stdata::init_forces)
//   forcing field            src/data.cu:239-350  (update_forces_watanabe97, lambda :317-348)
//   LBM step                 src/lbm.h:16-109, src/lbm.cu:20-160, src/lbm_collision_srt.h:8-16
//   observation noise        src/io.cu:160-246    (OBSERVE branch of output())
//   vorticity                src/io.cu:61-86
//   LETKF analysis           src/letkf.cu:29-118, 120-360; src/util/letkf_solver.h:235-349
//
// The reference stores everything in FP32 `real`; the oracle computes the
// dynamics and the analysis in FP64.  Where the reference does its arithmetic
// on the host in FP32 (initial condition rescale, feq of the IC, OBSERVE noise,
// vorticity), the oracle repeats it in FP32 exactly, because those values are
// inputs to everything else (or must be bit-exact).
//
// The forcing normals come from cuRAND MTGP32 on the device in the reference;
// the oracle takes them as an input array (tests read them from the engine or
// from the golden fixtures made by running the reference itself).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/lbl.h"

namespace {

constexpr int Q = 9;
inline int ex(int q) { return (q % 3) - 1; }   // config.h:257
inline int ey(int q) { return (q / 3) - 1; }   // config.h:258
inline double wq(int q) {                       // config.h:260-263
    const int ee = ex(q) * ex(q) + ey(q) * ey(q);
    return ee == 0 ? 4.0 / 9.0 : ee == 1 ? 1.0 / 9.0 : 1.0 / 36.0;
}
inline float wqf(int q) {
    const int ee = ex(q) * ex(q) + ey(q) * ey(q);
    return ee == 0 ? float(4. / 9.) : ee == 1 ? float(1. / 9.) : float(1. / 36.);
}

struct Derived {
    int nx, ny, M;
    double c, dx, dt, nu, cs, cs2, friction, u_ref, rho_ref;
    float cf, dxf;   // FP32 copies for the host-FP32 parts (IC feq, vorticity)
};

Derived derive(const lbl_config& cfg) {
    Derived d;
    d.nx = cfg.nx; d.ny = cfg.ny; d.M = cfg.n_ens;
    // The physical constants are the reference's constexpr `real` (FP32) values
    // (config.h:153-253), widened to FP64: the oracle solves the same discrete problem.
    const float cf = float(cfg.u_ref) / float(cfg.cfl);              // config.h:248
    const float dxf = float(cfg.h_ref) / float(cfg.ny - 1);          // config.h:250
    const float dtf = dxf / cf;                                       // config.h:251
    d.c = cf;
    d.dx = dxf;
    d.dt = dtf;
    d.nu = float(cfg.tau > 0 ? (cfg.tau - 0.5) * double(cf) * double(cf) * double(dtf) / 3.0 : cfg.nu);
    d.cs = cfg.cs;                                                    // a double in lbm.cu:59
    d.cs2 = cf * cf / 3;                                              // lbm.h:50 (constexpr real)
    d.friction = cfg.friction_rate;
    d.u_ref = cfg.u_ref; d.rho_ref = cfg.rho_ref;
    d.cf = cf;
    d.dxf = dxf;
    return d;
}

// feq in FP32 with the reference's host evaluation order (lbm.h:31-39); used for the IC.
inline float feq_f32(float rho, float u, float v, int q, float c) {
    const float uc0 = (u * float(ex(q)) + v * float(ey(q))) / c;
    const float uu0 = (u * u + v * v) / (c * c);
    return rho * wqf(q) * (1.0f + 3.0f * uc0 + 4.5f * uc0 * uc0 - 1.5f * uu0);
}

inline double feq(double rho, double u, double v, int q, double c) {   // lbm.h:31-39
    const double uc0 = (u * ex(q) + v * ey(q)) / c;
    const double uu0 = (u * u + v * v) / (c * c);
    return rho * wq(q) * (1.0 + 3.0 * uc0 + 4.5 * uc0 * uc0 - 1.5 * uu0);
}

// Gaspari-Cohn 5th-order piecewise rational function (letkf.cu:104-109), support d<=2.
inline double gaspari_cohn(double d) {
    if (d <= 0) return 1.0;
    if (d <= 1) return -d * d * d * d * d / 4. + d * d * d * d / 2. + d * d * d * 5. / 8. - d * d * 5. / 3. + 1;
    if (d <= 2) return d * d * d * d * d / 12. - d * d * d * d / 2. + d * d * d * 5. / 8. + d * d * 5. / 3. - d * 5 + 4 - 2. / 3. / d;
    return 0.0;
}

}  // namespace

struct orc_ctx {
    lbl_config cfg;
    Derived d;
    std::vector<double> f;           // [M][Q][ny][nx]
    std::vector<double> r, u, v;     // [M][ny][nx] post-stream macros of the last step
    std::vector<double> fx, fy;      // [ny][nx] body force of the current step
    std::vector<float> kx, ky, amp;  // forcing mode table
    std::mt19937 obs_engine;         // OBSERVE noise engine (io.cu:321, function-static there)
    bool obs_engine_started = false;
    std::mt19937 baseline_rng;       // normals for baseline timing runs only
    int max_sweeps_seen = 0;
    // learned closure (orc_set_closure): BF16-rounded parameters, feature scales
    std::vector<double> cl_w;
    double cl_nu_ref = 0, cl_dx_ref = 0;
};

namespace {

// ---------------------------------------------------------------------------
// learned closure: the 6-32-32-1 MLP of the engine's closure (parameter layout
// W1[32][6], b1[32], W2[32][32], b2[32], W3[32], b3), evaluated in FP64 under the
// engine's operand contract: BF16 parameter values, FP16 matrix operands (the
// weights W1, W2, W3, the bias b1, the features and both hidden activations).
// No counterpart in the reference (its closure is lbm.cu:42-60).
// ---------------------------------------------------------------------------
double bf16_round(double x) {
    float f = float(x);
    uint32_t u;
    std::memcpy(&u, &f, 4);
    u = ((u + 0x7FFFu + ((u >> 16) & 1u)) >> 16) << 16;
    std::memcpy(&f, &u, 4);
    return f;
}
// nearest FP16 value (ties to even), subnormals included, inf past 65520
double f16_round(double x) {
    if (x == 0 || !std::isfinite(x)) return x;
    const double a = std::fabs(x);
    if (a >= 65520.0) return std::copysign(INFINITY, x);
    int e;
    std::frexp(a, &e);  // a in [2^(e-1), 2^e)
    const double ulp = std::ldexp(1.0, std::max(e - 11, -24));
    return std::copysign(std::nearbyint(a / ulp) * ulp, x);
}
double gelu(double x) { return 0.5 * x * (1 + std::tanh(0.7978845608028654 * (x + 0.044715 * x * x * x))); }

// BF16 values of the parameters, W1, b1, W2 (0..1247) and W3 (1280..1311) also FP16
void contract_params(const float* params, double* w) {
    for (int k = 0; k < 1313; k++) {
        w[k] = bf16_round(params[k]);
        if (k < 1248 || (k >= 1280 && k < 1312)) w[k] = f16_round(w[k]);
    }
}

// w: contract_params output; x: the six features
double mlp_multiplier(const double* w, const double* x) {
    double xb[6], a1[32];
    for (int i = 0; i < 6; i++) xb[i] = f16_round(x[i]);
    for (int i = 0; i < 32; i++) {
        double h = w[192 + i];
        for (int j = 0; j < 6; j++) h += w[i * 6 + j] * xb[j];
        a1[i] = f16_round(gelu(h));
    }
    double z = w[1312];
    for (int i = 0; i < 32; i++) {
        double h = w[1248 + i];
        for (int j = 0; j < 32; j++) h += w[224 + i * 32 + j] * a1[j];
        z += w[1280 + i] * f16_round(gelu(h));
    }
    return z > 20 ? z : std::log1p(std::exp(z));
}

double closure_multiplier(const orc_ctx* o, double ux, double uy, double vx, double vy, double dx) {
    const double s12 = 0.5 * (uy + vx), w12 = 0.5 * (uy - vx);
    const double ss = ux * ux + 2 * s12 * s12 + vy * vy, ww = 2 * w12 * w12;
    const double k = dx * dx / o->cl_nu_ref;
    const double x[6] = {std::log1p(k * std::sqrt(2 * ss)), std::log1p(k * std::sqrt(2 * ww)), (ww - ss) / (ww + ss + 1e-30),
                         (ux + vy) / std::sqrt(ss + 1e-30), dx / o->cl_dx_ref, std::asinh(k * (vx - uy))};
    return mlp_multiplier(o->cl_w.data(), x);
}

// ---------------------------------------------------------------------------
// initial condition: src/data.cu:25-141 (reference spectrum) and the K4EXP variant
// ---------------------------------------------------------------------------
// Fills p (amplitude) and theta (phase) tables in the reference's draw order:
// kj outer, ki inner, one uniform(-1,1) draw per mode (data.cu:48-63).
void ic_tables(const lbl_config& cfg, int seed, std::vector<float>& p, std::vector<float>& theta) {
    const int nk = cfg.nx / 2;
    std::mt19937 eng(seed);
    std::uniform_real_distribution<float> dist(-1, 1);
    p.assign(size_t(nk) * nk, 0.f);
    theta.assign(size_t(nk) * nk, 0.f);
    const float k0 = float(cfg.kf);
    for (int kj = 0; kj < nk; kj++) {
        for (int ki = 0; ki < nk; ki++) {
            const size_t kij = ki + size_t(nk) * kj;
            const float k = std::sqrt(float(ki * ki + kj * kj));
            float pk;
            if (cfg.ic_kind == LBL_IC_REFERENCE) {
                const float dk = 10, sigma = 5;
                pk = (k0 - dk <= k && k <= k0 + dk) ? std::exp(-(k - k0) * (k - k0) / sigma) : 0.f;
            } else {
                // E(k) ~ k^4 exp(-2 (k/kf)^2)  <=>  |psi_k| ~ k^(1/2) exp(-(k/kf)^2); truncated at
                // exp(-(k/kf)^2) < 1e-10 so that both engine and oracle sum the same modes.
                const float s = k / k0;
                pk = (k > 0 && s * s <= 23.0f) ? std::sqrt(k) * std::exp(-s * s) : 0.f;
            }
            p[kij] = pk;
            theta[kij] = float(dist(eng) * M_PI);
        }
    }
}

// u, v from the stream-function sum (data.cu:76-110): FP64 terms added into FP32 sums;
// zero-amplitude modes are skipped (adding +-0 does not change the FP64 sum).
void ic_velocity(const lbl_config& cfg, const std::vector<float>& p, const std::vector<float>& theta,
                 std::vector<float>& u, std::vector<float>& v) {
    const int nx = cfg.nx, ny = cfg.ny, nk = nx / 2;
    struct Mode { double kx, ky, p, th; };
    std::vector<Mode> modes;
    for (int kj = 0; kj < nk; kj++)
        for (int ki = 0; ki < nk; ki++) {
            const size_t kij = ki + size_t(nk) * kj;
            if (p[kij] == 0.f) continue;
            modes.push_back({2 * M_PI * ki / nx, 2 * M_PI * kj / ny, double(p[kij]), double(theta[kij])});
        }
    u.assign(size_t(nx) * ny, 0.f);
    v.assign(size_t(nx) * ny, 0.f);
#pragma omp parallel for schedule(static)
    for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
            float ut = 0, vt = 0;  // `real utmp`: a float receiving FP64 terms
            for (const auto& m : modes) {
                const double cs = std::cos(m.kx * i + m.ky * j + m.th);
                ut += m.p * m.ky * cs;
                vt += m.p * -m.kx * cs;
            }
            u[i + size_t(nx) * j] = ut;
            v[i + size_t(nx) * j] = vt;
        }
}

// Rescale in FP32 on the host exactly like data.cu:113-120 (max speed) or to an rms speed.
void ic_rescale(const lbl_config& cfg, std::vector<float>& u, std::vector<float>& v) {
    const size_t n = u.size();
    if (cfg.ic_kind == LBL_IC_REFERENCE) {
        float vmax = float(1e-30 * cfg.u_ref);
        for (size_t ij = 0; ij < n; ij++) vmax = std::max(vmax, std::sqrt(u[ij] * u[ij] + v[ij] * v[ij]));
        const float s = float(cfg.u_ref) / vmax * float(cfg.ic_amp);
        for (size_t ij = 0; ij < n; ij++) { u[ij] *= s; v[ij] *= s; }
    } else {
        double e = 0;
        for (size_t ij = 0; ij < n; ij++) e += double(u[ij]) * u[ij] + double(v[ij]) * v[ij];
        const float s = float(cfg.ic_amp / std::sqrt(e / double(n) + 1e-300));
        for (size_t ij = 0; ij < n; ij++) { u[ij] *= s; v[ij] *= s; }
    }
}

void ic_member_uv(const lbl_config& cfg, int seed, std::vector<float>& u, std::vector<float>& v) {
    std::vector<float> p, th;
    ic_tables(cfg, seed, p, th);
    ic_velocity(cfg, p, th, u, v);
    ic_rescale(cfg, u, v);
}

}  // namespace

extern "C" {

// The reference's defaults for a run mode at grid nx = 64*SCALER (src/config.h with
// LES and FORCE_TURB on), so that code timing the oracle needs nothing from the
// product library.  OBS_ERROR_* have no default in the reference (config.h:195
// #error); they take run/jserr:146-147's values.
int orc_config_default(lbl_config* c, int mode, int nx, int n_ens) {
    if (!c) return LBL_ERR_ARG;
    std::memset(c, 0, sizeof(*c));
    const int scaler = nx / 64;
    c->abi_version = LBL_ABI_VERSION;
    c->mode = mode;
    c->nx = nx; c->ny = nx;                               // config.h:88-89, 133-134
    c->n_ens = n_ens;                                     // mpiexec -np M
    c->iiter = 5 * (scaler > 0 ? scaler : 1);             // config.h:136
    c->ioprune = 10;                                      // config.h:90-92
    c->daprune = 10;                                      // config.h:55-57
    c->da_xyprune = 1;                                    // config.h:59-61
    c->iter_main = c->iiter * 2000;                       // config.h:144
    c->spinup = 100000 * c->iiter;                        // config.h:139
    c->ic_kind = LBL_IC_REFERENCE;                        // data.cu:53-120
    c->ens_init = LBL_ENS_INDEPENDENT;                    // data.cu:31-35
    c->compat_stale_v = 1;                                // letkf.cu:340-355
    c->jacobi_max_sweeps = 100;                           // cu_matrix_eigensolver_wrapper.hpp:193
    c->letkf_covinf = 1.0;                                // config.h:48-50
    c->obs_error_rho = 0.01;                              // run/jserr:146-147
    c->obs_error_u = 0.1;
    c->cs = 0.2;                                          // lbm.cu:59
    c->nu = 1e-4;                                         // config.h:157
    c->cfl = 0.05;                                        // config.h:153
    c->rho_ref = 1;                                       // config.h:156
    c->u_ref = 1;                                         // config.h:182
    c->h_ref = 2 * M_PI;                                  // config.h:158
    c->kf = 4;                                            // config.h:161
    c->fkf = 5.6;                                         // config.h:171
    c->friction_rate = 5e-4;                              // config.h:180
    c->ic_amp = 0.01;                                     // data.cu:53
    c->ens_perturb = 0.1;
    c->jacobi_tol = 1e-6;                                 // cu_matrix_eigensolver_wrapper.hpp:192
    c->force_seed = 1991;                                 // data.cu:294
    c->obs_seed = 334;                                    // io.cu:321
    c->da_obs_ruv = 1;                                    // config.h:44
    c->da_nud_rate = 0.1;                                 // config.h:67-69
    return LBL_OK;
}

int orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

orc_ctx* orc_create(const lbl_config* cfg) {
    if (!cfg || cfg->nx <= 0 || cfg->ny <= 0 || cfg->n_ens <= 0) return nullptr;
    auto* o = new orc_ctx();
    o->cfg = *cfg;
    o->d = derive(*cfg);
    const size_t nxy = size_t(cfg->nx) * cfg->ny;
    o->f.assign(size_t(cfg->n_ens) * Q * nxy, 0.0);
    o->r.assign(size_t(cfg->n_ens) * nxy, 0.0);
    o->u.assign(size_t(cfg->n_ens) * nxy, 0.0);
    o->v.assign(size_t(cfg->n_ens) * nxy, 0.0);
    o->fx.assign(nxy, 0.0);
    o->fy.assign(nxy, 0.0);
    o->baseline_rng.seed(uint32_t(cfg->force_seed));
    return o;
}

void orc_destroy(orc_ctx* o) { delete o; }

// IC of one ensemble id (seed), FP32 like the reference: r = rho_ref, u, v, f = feq(r,u,v).
// data.cu:25-141.  seed already includes the +334 of DA mode.
int orc_ic_fields(const lbl_config* cfg, int seed, float* r, float* u, float* v, float* f) {
    std::vector<float> uu, vv;
    ic_member_uv(*cfg, seed, uu, vv);
    const size_t nxy = size_t(cfg->nx) * cfg->ny;
    const float cf = float(cfg->u_ref) / float(cfg->cfl);
    const float r0 = float(cfg->rho_ref);
    for (size_t ij = 0; ij < nxy; ij++) {
        if (r) r[ij] = r0;
        if (u) u[ij] = uu[ij];
        if (v) v[ij] = vv[ij];
        if (f)
            for (int q = 0; q < Q; q++) f[ij + nxy * q] = feq_f32(r0, uu[ij], vv[ij], q, cf);
    }
    return 0;
}

// IC of the whole ensemble (mirrors lbl_init): member k uses ensemble id k + ofs (+334 in DA).
int orc_init(orc_ctx* o, int ens_offset) {
    const auto& cfg = o->cfg;
    const size_t nxy = size_t(cfg.nx) * cfg.ny;
    const int add = (cfg.mode == LBL_MODE_DA_LETKF) ? 334 : 0;
    std::vector<float> un, vn;
    if (cfg.ens_init == LBL_ENS_PERTURBED) ic_member_uv(cfg, ens_offset, un, vn);  // nature IC (seed ofs)
    const float cf = float(cfg.u_ref) / float(cfg.cfl);
    const float r0 = float(cfg.rho_ref);
    for (int m = 0; m < cfg.n_ens; m++) {
        std::vector<float> uu, vv;
        ic_member_uv(cfg, m + ens_offset + add, uu, vv);
        if (cfg.ens_init == LBL_ENS_PERTURBED) {
            const float a = float(cfg.ens_perturb);
            for (size_t ij = 0; ij < nxy; ij++) { uu[ij] = un[ij] + a * uu[ij]; vv[ij] = vn[ij] + a * vv[ij]; }
        }
        for (size_t ij = 0; ij < nxy; ij++) {
            o->r[m * nxy + ij] = r0;
            o->u[m * nxy + ij] = uu[ij];
            o->v[m * nxy + ij] = vv[ij];
            for (int q = 0; q < Q; q++) o->f[(size_t(m) * Q + q) * nxy + ij] = feq_f32(r0, uu[ij], vv[ij], q, cf);
        }
    }
    return 0;
}

// Forcing mode table: data.cu:161-237 (amplitudes normalised in long double like the reference).
int orc_force_modes(const lbl_config* cfg, float* kx, float* ky, float* amp, int cap) {
    const float kf = float(cfg->kf), sigma = 1, dk = 2;
    const int kmax = int(kf + dk);
    std::vector<float> vkx, vky, vam;
    long double asum = 0;
    for (int y = 0; y < kmax; y++)
        for (int x = 0; x < kmax; x++) {
            if (x == 0 && y == 0) continue;
            const double k = std::sqrt(double(y * y + x * x));
            if (kf - dk <= k && k <= kf + dk) {
                const float a = float(std::exp(-(k - kf) * (k - kf) / sigma));
                asum += a;
                vkx.push_back(float(x));
                vky.push_back(float(y));
                vam.push_back(a);
            }
        }
    const float total = float(cfg->fkf * cfg->u_ref / 1.0);
    for (auto& a : vam) a = float(a * (total / asum));
    const int n = int(vam.size());
    if (cap < n) return -n;
    for (int i = 0; i < n; i++) { kx[i] = vkx[i]; ky[i] = vky[i]; amp[i] = vam[i]; }
    return n;
}

// Force field from one slice of 4*n normals: data.cu:317-348 (R = 0: white in time).
int orc_force(orc_ctx* o, const float* randoms, double* fx_out, double* fy_out) {
    const auto& cfg = o->cfg;
    if (o->kx.empty()) {
        float kx[128], ky[128], am[128];
        const int n = orc_force_modes(&cfg, kx, ky, am, 128);
        if (n <= 0) return -1;
        o->kx.assign(kx, kx + n); o->ky.assign(ky, ky + n); o->amp.assign(am, am + n);
    }
    const int nx = cfg.nx, ny = cfg.ny, n = int(o->amp.size());
#pragma omp parallel for schedule(static)
    for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
            const double x = double(i - nx / 2) / nx, y = double(j - ny / 2) / ny;
            double fx = 0, fy = 0;
            for (int k = 0; k < n; k++) {
                const double kx = o->kx[k], ky = o->ky[k];
                const double th = 2 * M_PI * (kx * x + ky * y);
                const double s = std::sin(th), c = std::cos(th);
                const double r0 = randoms[k], r1 = randoms[k + n], r2 = randoms[k + 2 * n], r3 = randoms[k + 3 * n];
                const double fek = (r0 * kx + r1 * ky) * s + (r2 * kx + r3 * ky) * c;
                fx += o->amp[k] * 2 * M_PI * ky * fek;
                fy += o->amp[k] * 2 * M_PI * (-kx) * fek;
            }
            o->fx[i + size_t(nx) * j] = fx;
            o->fy[i + size_t(nx) * j] = fy;
        }
    const size_t nxy = size_t(nx) * ny;
    if (fx_out) std::copy(o->fx.begin(), o->fx.begin() + nxy, fx_out);
    if (fy_out) std::copy(o->fy.begin(), o->fy.begin() + nxy, fy_out);
    return n;
}

int orc_set_force(orc_ctx* o, const float* fx, const float* fy) {
    const size_t nxy = size_t(o->cfg.nx) * o->cfg.ny;
    for (size_t i = 0; i < nxy; i++) { o->fx[i] = fx[i]; o->fy[i] = fy[i]; }
    return 0;
}

int orc_set_f(orc_ctx* o, int m, const float* f) {
    const size_t n = size_t(Q) * o->cfg.nx * o->cfg.ny;
    if (m < 0 || m >= o->cfg.n_ens) return -1;
    for (size_t i = 0; i < n; i++) o->f[m * n + i] = f[i];
    return 0;
}

int orc_get_f(orc_ctx* o, int m, double* f) {
    const size_t n = size_t(Q) * o->cfg.nx * o->cfg.ny;
    if (m < 0 || m >= o->cfg.n_ens) return -1;
    std::copy(o->f.begin() + m * n, o->f.begin() + (m + 1) * n, f);
    return 0;
}

int orc_set_macros(orc_ctx* o, int m, const float* r, const float* u, const float* v) {
    const size_t n = size_t(o->cfg.nx) * o->cfg.ny;
    if (m < 0 || m >= o->cfg.n_ens) return -1;
    for (size_t i = 0; i < n; i++) {
        if (r) o->r[m * n + i] = r[i];
        if (u) o->u[m * n + i] = u[i];
        if (v) o->v[m * n + i] = v[i];
    }
    return 0;
}

int orc_get_macros(orc_ctx* o, int m, double* r, double* u, double* v) {
    const size_t n = size_t(o->cfg.nx) * o->cfg.ny;
    if (m < 0 || m >= o->cfg.n_ens) return -1;
    if (r) std::copy(o->r.begin() + m * n, o->r.begin() + (m + 1) * n, r);
    if (u) std::copy(o->u.begin() + m * n, o->u.begin() + (m + 1) * n, u);
    if (v) std::copy(o->v.begin() + m * n, o->v.begin() + (m + 1) * n, v);
    return 0;
}

// One LBM step of every member with the current force field: lbm.h:16-29 minus the
// forcing refresh.  Stream (lbm.cu:67-103) -> Smagorinsky on post-stream u,v
// (lbm.cu:24-65) -> BGK toward feq + force term with friction (lbm.cu:105-160).
int orc_step_noforce(orc_ctx* o) {
    const Derived& d = o->d;
    const int nx = d.nx, ny = d.ny, M = d.M;
    const size_t nxy = size_t(nx) * ny;
    std::vector<double> fn(o->f.size());
#pragma omp parallel for collapse(2) schedule(static)
    for (int m = 0; m < M; m++)
        for (int j = 0; j < ny; j++) {
            const double* fm = &o->f[size_t(m) * Q * nxy];
            double* fnm = &fn[size_t(m) * Q * nxy];
            for (int i = 0; i < nx; i++) {
                double fc[Q], rho = 0, mu = 0, mv = 0;
                for (int q = 0; q < Q; q++) {
                    const int iu = (i - ex(q) + nx) % nx, ju = (j - ey(q) + ny) % ny;
                    fc[q] = fm[size_t(q) * nxy + iu + size_t(nx) * ju];
                }
                for (int q = 0; q < Q; q++) rho += fc[q];
                for (int q = 0; q < Q; q++) { mu += fc[q] * d.c * ex(q); mv += fc[q] * d.c * ey(q); }
                const size_t ij = i + size_t(nx) * j;
                for (int q = 0; q < Q; q++) fnm[size_t(q) * nxy + ij] = fc[q];
                o->r[m * nxy + ij] = rho;
                o->u[m * nxy + ij] = mu / rho;
                o->v[m * nxy + ij] = mv / rho;
            }
        }
#pragma omp parallel for collapse(2) schedule(static)
    for (int m = 0; m < M; m++)
        for (int j = 0; j < ny; j++) {
            double* fnm = &fn[size_t(m) * Q * nxy];
            const double* um = &o->u[m * nxy];
            const double* vm = &o->v[m * nxy];
            for (int i = 0; i < nx; i++) {
                const size_t ij = i + size_t(nx) * j;
                const size_t ije = (i + 1) % nx + size_t(nx) * j, ijw = (i - 1 + nx) % nx + size_t(nx) * j;
                const size_t ijn = i + size_t(nx) * ((j + 1) % ny), ijs = i + size_t(nx) * ((j - 1 + ny) % ny);
                const double ux = (um[ije] - um[ijw]) / (2 * d.dx), uy = (um[ijn] - um[ijs]) / (2 * d.dx);
                const double vx = (vm[ije] - vm[ijw]) / (2 * d.dx), vy = (vm[ijn] - vm[ijs]) / (2 * d.dx);
                const double s01 = 0.5 * (uy + vx);
                const double ss = std::sqrt(2 * (ux * ux + 2 * s01 * s01 + vy * vy));
                double nus = d.cs * d.cs * d.dx * d.dx * ss;
                if (!o->cl_w.empty()) nus *= closure_multiplier(o, ux, uy, vx, vy, d.dx);
                const double nut = d.nu + nus;
                const double tau = 0.5 + 3. * nut / d.c / d.c / d.dt;
                const double omega = 1. / tau;
                const double rho = o->r[m * nxy + ij], u = um[ij], v = vm[ij];
                const double fr_dt = double(float(d.friction) / float(d.dt));   // constexpr real (lbm.h:52)
                const double Fx = (o->fx[ij] - fr_dt * u) * d.dt;
                const double Fy = (o->fy[ij] - fr_dt * v) * d.dt;
                for (int q = 0; q < Q; q++) {
                    double fq = fnm[size_t(q) * nxy + ij];
                    fq -= omega * (fq - feq(rho, u, v, q, d.c));
                    const double cx = d.u_ref * ex(q), cy = d.u_ref * ey(q);
                    fq += (cx * Fx + cy * Fy) / d.cs2 * wq(q) * rho;
                    fnm[size_t(q) * nxy + ij] = fq;
                }
            }
        }
    o->f.swap(fn);
    return 0;
}

// nsteps full steps with forcing drawn from `randoms` (nsteps*4*n floats) or, when
// randoms is NULL, from an internal normal generator (for baseline timing only).
int orc_step(orc_ctx* o, int nsteps, const float* randoms) {
    if (o->kx.empty()) {
        std::vector<float> z(4 * 128, 0.f);
        orc_force(o, z.data(), nullptr, nullptr);
    }
    const int n = int(o->amp.size());
    std::vector<float> buf(4 * n);
    std::normal_distribution<float> nd(0.f, 0.84089641525f);
    for (int s = 0; s < nsteps; s++) {
        const float* rs = randoms ? randoms + size_t(s) * 4 * n : nullptr;
        if (!rs) { for (auto& x : buf) x = nd(o->baseline_rng); rs = buf.data(); }
        orc_force(o, rs, nullptr, nullptr);
        orc_step_noforce(o);
    }
    return 0;
}

// Vorticity exactly as io.cu:61-86 (host FP32, central differences, periodic).
int orc_vorticity_f32(const lbl_config* cfg, const float* u, const float* v, float* vor) {
    const int nx = cfg->nx, ny = cfg->ny;
    const float dx = float(cfg->h_ref) / float(cfg->ny - 1);   // constexpr real dx (config.h:250)
    for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
            const int iw = (i - 1 + nx) % nx, ie = (i + 1) % nx, js = (j - 1 + ny) % ny, jn = (j + 1) % ny;
            const float us = u[i + nx * js], un = u[i + nx * jn];
            const float uy = (un - us) / (2 * dx);
            const float vw = v[iw + nx * j], ve = v[ie + nx * j];
            const float vx = (ve - vw) / (2 * dx);
            vor[i + nx * j] = vx - uy;
        }
    return 0;
}

// OBSERVE noise + NaN pruning + observed vorticity: io.cu:160-246.  The engine is
// std::mt19937(obs_seed + ensemble_id 0) created at the first call and kept (it is a
// function-static in the reference); the normal distribution is new on every call.
int orc_observe(orc_ctx* o, const float* r, const float* u, const float* v,
                float* ro, float* uo, float* vo, float* voro) {
    const auto& cfg = o->cfg;
    if (!o->obs_engine_started) { o->obs_engine.seed(uint32_t(cfg.obs_seed)); o->obs_engine_started = true; }
    std::normal_distribution<float> dist(0, 1);
    const size_t nxy = size_t(cfg.nx) * cfg.ny;
    const float er = float(cfg.obs_error_rho), eu = float(cfg.obs_error_u);
    for (size_t ij = 0; ij < nxy; ij++) {
        ro[ij] = r[ij] + er * dist(o->obs_engine);
        uo[ij] = u[ij] + eu * dist(o->obs_engine);
        vo[ij] = v[ij] + eu * dist(o->obs_engine);
    }
    orc_vorticity_f32(&cfg, uo, vo, voro);
    const int p = cfg.da_xyprune;
    for (int j = 0; j < cfg.ny; j++)
        for (int i = 0; i < cfg.nx; i++)
            if (i % p != 0 || j % p != 0) {
                const size_t ij = i + size_t(cfg.nx) * j;
                ro[ij] = NAN; uo[ij] = NAN; vo[ij] = NAN; voro[ij] = NAN;
            }
    return 0;
}

// ---------------------------------------------------------------------------
// LETKF analysis (letkf.cu:29-118 geometry and R-localisation, 120-360 stage order;
// letkf_solver.h:235-349 maths), FP64, eigen-decomposition by cyclic Jacobi.
// ---------------------------------------------------------------------------
struct Geo { int p, nl, off, nox, nobs; double dloc; };

static Geo geometry(const lbl_config& cfg) {
    Geo g;
    g.p = cfg.da_xyprune;
    if (cfg.letkf_rloc_len <= 0) {
        g.dloc = g.p - 1;
        g.nl = g.p == 1 ? 0 : 2;
        g.off = g.p == 1 ? 0 : 1;
        g.nox = g.p == 1 ? 1 : 4;
    } else {
        g.dloc = double(cfg.letkf_rloc_len) * g.p;
        g.off = 0;
        g.nl = cfg.letkf_rloc_len * 2;
        g.nox = g.nl * 2 + 1;
    }
    g.nobs = g.nox * g.nox * 3;
    return g;
}

// symmetric eigen-decomposition A = V diag(w) V^T, cyclic two-sided Jacobi in FP64.
static int jacobi_eig(int n, std::vector<double>& A, std::vector<double>& V, std::vector<double>& w) {
    V.assign(size_t(n) * n, 0.0);
    for (int i = 0; i < n; i++) V[i + n * i] = 1.0;
    int sweep = 0;
    for (; sweep < 100; sweep++) {
        double off = 0, tot = 0;
        for (int j = 0; j < n; j++)
            for (int i = 0; i < n; i++) {
                tot += A[i + n * j] * A[i + n * j];
                if (i != j) off += A[i + n * j] * A[i + n * j];
            }
        if (off <= 1e-30 * tot) break;
        for (int p = 0; p < n - 1; p++)
            for (int q = p + 1; q < n; q++) {
                const double apq = A[p + n * q];
                if (std::fabs(apq) < 1e-300) continue;
                const double app = A[p + n * p], aqq = A[q + n * q];
                const double theta = (aqq - app) / (2 * apq);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1));
                const double c = 1 / std::sqrt(t * t + 1), s = t * c;
                for (int k = 0; k < n; k++) {  // columns p,q
                    const double akp = A[k + n * p], akq = A[k + n * q];
                    A[k + n * p] = c * akp - s * akq;
                    A[k + n * q] = s * akp + c * akq;
                }
                for (int k = 0; k < n; k++) {  // rows p,q
                    const double apk = A[p + n * k], aqk = A[q + n * k];
                    A[p + n * k] = c * apk - s * aqk;
                    A[q + n * k] = s * apk + c * aqk;
                }
                for (int k = 0; k < n; k++) {
                    const double vkp = V[k + n * p], vkq = V[k + n * q];
                    V[k + n * p] = c * vkp - s * vkq;
                    V[k + n * q] = s * vkp + c * vkq;
                }
            }
    }
    w.resize(n);
    for (int i = 0; i < n; i++) w[i] = A[i + n * i];
    return sweep;
}

// Observation weight r_o of window slot (a,b), variable var (0 u, 1 v, 2 rho) at point (i,j):
// diag of (rho o R)^-1 built by set_rR (letkf.cu:75-114).
int orc_obs_weight(const lbl_config* cfg, int i, int j, int a, int b, int var, double* w, int* valid) {
    const Geo g = geometry(*cfg);
    const int io = (i / g.p + a - (g.nl - g.off)) * g.p;
    const int jo = (j / g.p + b - (g.nl - g.off)) * g.p;
    const double sig = var == 2 ? cfg->obs_error_rho : cfg->obs_error_u;
    double wt = 1.0 / (sig * sig);
    if (g.p > 1) {
        const double di = i - io, dj = j - jo;
        const double dd = std::sqrt(di * di + dj * dj) / (g.dloc + 1e-6);
        wt *= gaspari_cohn(dd);
    }
    *w = wt;
    *valid = !(std::abs(i - io) > g.nl * g.p || std::abs(j - jo) > g.nl * g.p);
    return g.nobs;
}

// Full analysis of the ensemble held by o.  ro/uo/vo are observation fields (nx*ny,
// NaN off the lattice is never read).  Writes analysis populations into o->f and
// the analysis rho, u into o->r, o->u (lbm2euler, letkf.cu:336-357; v untouched).
// out_lambda (optional, nx*ny*M): eigenvalues per point sorted ascending.
int orc_assimilate_rows(orc_ctx* o, const float* ro, const float* uo, const float* vo, double* out_lambda,
                        int j0, int j1);

int orc_assimilate(orc_ctx* o, const float* ro, const float* uo, const float* vo, double* out_lambda) {
    return orc_assimilate_rows(o, ro, uo, vo, out_lambda, 0, o->cfg.ny);
}

// Analysis of grid rows [j0, j1) only (rows outside keep the forecast); the bounded
// samples of the CPU baseline use it.
int orc_assimilate_rows(orc_ctx* o, const float* ro, const float* uo, const float* vo, double* out_lambda,
                        int j0, int j1) {
    const auto& cfg = o->cfg;
    const Derived& d = o->d;
    const Geo g = geometry(cfg);
    const int nx = cfg.nx, ny = cfg.ny, M = cfg.n_ens;
    const size_t nxy = size_t(nx) * ny;
    const double beta = cfg.letkf_covinf;
    // H(x) of every member at every grid point (u, v, rho moments of f, pack_yk letkf.cu:148-187)
    std::vector<double> Hu(M * nxy), Hv(M * nxy), Hr(M * nxy);
#pragma omp parallel for collapse(2) schedule(static)
    for (int m = 0; m < M; m++)
        for (int ij = 0; ij < int(nxy); ij++) {
            double rho = 0, mu = 0, mv = 0;
            for (int q = 0; q < Q; q++) {
                const double fq = o->f[(size_t(m) * Q + q) * nxy + ij];
                rho += fq; mu += fq * d.c * ex(q); mv += fq * d.c * ey(q);
            }
            Hr[m * nxy + ij] = rho; Hu[m * nxy + ij] = mu / rho; Hv[m * nxy + ij] = mv / rho;
        }
    std::vector<double> fa(o->f);
    int max_sweeps = 0;
    j0 = std::max(0, j0);
    j1 = std::min(ny, j1);
#pragma omp parallel for schedule(dynamic, 64) reduction(max : max_sweeps)
    for (int ij = j0 * nx; ij < j1 * nx; ij++) {
        const int i = ij % nx, j = ij / nx;
        const int no = g.nobs, nox2 = g.nox * g.nox;
        std::vector<double> Y(size_t(no) * M, 0.0), yo(no, 0.0), rw(no, 0.0);
        for (int b = 0; b < g.nox; b++)
            for (int a = 0; a < g.nox; a++) {
                const int slot = a + g.nox * b;
                const int io = (i / g.p + a - (g.nl - g.off)) * g.p;
                const int jo = (j / g.p + b - (g.nl - g.off)) * g.p;
                const bool valid = !(std::abs(i - io) > g.nl * g.p || std::abs(j - jo) > g.nl * g.p);
                const int iop = (io + nx) % nx, jop = (jo + ny) % ny;
                const size_t s = iop + size_t(nx) * jop;
                for (int var = 0; var < 3; var++) {
                    double w; int vld;
                    orc_obs_weight(&cfg, i, j, a, b, var, &w, &vld);
                    rw[slot + var * nox2] = w;
                }
                if (!valid) continue;
                for (int m = 0; m < M; m++) {
                    Y[slot + 0 * nox2 + size_t(no) * m] = Hu[m * nxy + s];
                    Y[slot + 1 * nox2 + size_t(no) * m] = Hv[m * nxy + s];
                    Y[slot + 2 * nox2 + size_t(no) * m] = Hr[m * nxy + s];
                }
                yo[slot + 0 * nox2] = uo[s];
                yo[slot + 1 * nox2] = vo[s];
                yo[slot + 2 * nox2] = ro[s];
            }
        // ybar, dY, dyo (letkf_solver.h:239-243)
        std::vector<double> dY(size_t(no) * M), dyo(no);
        for (int k = 0; k < no; k++) {
            double ybar = 0;
            for (int m = 0; m < M; m++) ybar += Y[k + size_t(no) * m];
            ybar /= M;
            for (int m = 0; m < M; m++) dY[k + size_t(no) * m] = Y[k + size_t(no) * m] - ybar;
            dyo[k] = yo[k] - ybar;
        }
        // Q = (M-1)/beta I + dY^T R^-1 dY (letkf_solver.h:252-254)
        std::vector<double> Qm(size_t(M) * M, 0.0);
        for (int l = 0; l < M; l++)
            for (int k = 0; k < M; k++) {
                double s = 0;
                for (int ob = 0; ob < no; ob++) s += dY[ob + size_t(no) * k] * rw[ob] * dY[ob + size_t(no) * l];
                Qm[k + size_t(M) * l] = s + (k == l ? (M - 1) / beta : 0.0);
            }
        std::vector<double> V, lam;
        const int sw = jacobi_eig(M, Qm, V, lam);
        max_sweeps = std::max(max_sweeps, sw);
        // w = V Lambda^-1 V^T dY^T R^-1 dyo ; W = sqrt(M-1) V Lambda^-1/2 V^T (letkf_solver.h:289-306)
        std::vector<double> c(M, 0.0), y(M), wv(M, 0.0), T(size_t(M) * M, 0.0);
        for (int k = 0; k < M; k++)
            for (int ob = 0; ob < no; ob++) c[k] += dY[ob + size_t(no) * k] * rw[ob] * dyo[ob];
        for (int jj = 0; jj < M; jj++) {
            double s = 0;
            for (int k = 0; k < M; k++) s += V[k + size_t(M) * jj] * c[k];
            y[jj] = s / lam[jj];
        }
        for (int k = 0; k < M; k++)
            for (int jj = 0; jj < M; jj++) wv[k] += V[k + size_t(M) * jj] * y[jj];
        const double sq = std::sqrt(double(M - 1));
        for (int l = 0; l < M; l++)
            for (int k = 0; k < M; k++) {
                double s = 0;
                for (int jj = 0; jj < M; jj++) s += V[k + size_t(M) * jj] * V[l + size_t(M) * jj] / std::sqrt(lam[jj]);
                T[k + size_t(M) * l] = sq * s + wv[k];   // W + w 1^T (letkf_solver.h:314)
            }
        // Xa = xbar 1^T + dX T (letkf_solver.h:315-316)
        for (int q = 0; q < Q; q++) {
            double xbar = 0;
            std::vector<double> dX(M);
            for (int m = 0; m < M; m++) xbar += o->f[(size_t(m) * Q + q) * nxy + ij];
            xbar /= M;
            for (int m = 0; m < M; m++) dX[m] = o->f[(size_t(m) * Q + q) * nxy + ij] - xbar;
            for (int l = 0; l < M; l++) {
                double s = 0;
                for (int k = 0; k < M; k++) s += dX[k] * T[k + size_t(M) * l];
                fa[(size_t(l) * Q + q) * nxy + ij] = xbar + s;
            }
        }
        if (out_lambda) {
            std::sort(lam.begin(), lam.end());
            for (int k = 0; k < M; k++) out_lambda[size_t(ij) * M + k] = lam[k];
        }
    }
    o->f.swap(fa);
    // lbm2euler: rho, u from the analysis f (v left stale, letkf.cu:340-355)
    for (int m = 0; m < M; m++)
        for (size_t ij = size_t(j0) * nx; ij < size_t(j1) * nx; ij++) {
            double rho = 0, mu = 0, mv = 0;
            for (int q = 0; q < Q; q++) {
                const double fq = o->f[(size_t(m) * Q + q) * nxy + ij];
                rho += fq; mu += fq * d.c * ex(q); mv += fq * d.c * ey(q);
            }
            o->r[m * nxy + ij] = rho;
            o->u[m * nxy + ij] = mu / rho;
            if (!cfg.compat_stale_v) o->v[m * nxy + ij] = mv / rho;
        }
    o->max_sweeps_seen = max_sweeps;
    return max_sweeps;
}

int orc_max_sweeps(orc_ctx* o) { return o->max_sweeps_seen; }

// the multiplier of n feature rows x [n][6] (FP64 under the BF16 operand contract)
int orc_closure_forward(const float* params, const double* x, int n, double* out) {
    std::vector<double> w(1313);
    contract_params(params, w.data());
    for (int i = 0; i < n; i++) out[i] = mlp_multiplier(w.data(), x + size_t(i) * 6);
    return 0;
}

// learned closure in the steps (params: 1313 floats, NULL = plain Smagorinsky);
// nu_ref, dx_ref <= 0 take this run's nu and h_ref/255 like lbl_set_closure
int orc_set_closure(orc_ctx* o, const float* params, double nu_ref, double dx_ref) {
    if (!params) { o->cl_w.clear(); return 0; }
    o->cl_w.resize(1313);
    contract_params(params, o->cl_w.data());
    o->cl_nu_ref = nu_ref > 0 ? nu_ref : double(float(o->d.nu));
    o->cl_dx_ref = dx_ref > 0 ? dx_ref : o->cfg.h_ref / 255.0;
    return 0;
}

// DA_NUDGING (nudging.cu:40-143): f <- alpha feq(rho_o, u_o, v_o) + (1 - alpha) f for every
// member, in FP64.  ro, uo, vo are full fields (NaN off the p-lattice, never read);
// with p > 1 the lattice values are interpolated bilinearly between (iw, js) and
// (iw + p, js + p), periodic (nudging.cu:98-127).  DA_QUADRA masks x >= nx/2 (odd)
// and y >= ny/2 (>= 2); DA_OBS_UV (da_obs_ruv = 0) takes rho from the model.
int orc_nudge(orc_ctx* o, const float* ro, const float* uo, const float* vo) {
    const lbl_config& cfg = o->cfg;
    const int nx = cfg.nx, ny = cfg.ny, p = cfg.da_xyprune;
    const size_t nxy = size_t(nx) * ny;
    const double alpha = float(cfg.da_nud_rate);
    const bool skip_east = cfg.da_quadra % 2 == 1, skip_north = cfg.da_quadra >= 2;
    auto at = [&](const float* a, int i, int j) { return double(a[size_t((i % nx + nx) % nx) + size_t(nx) * ((j % ny + ny) % ny)]); };
    for (int m = 0; m < cfg.n_ens; m++) {
#pragma omp parallel for schedule(static)
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) {
                if (skip_east && !(i < nx / 2)) continue;
                if (skip_north && !(j < ny / 2)) continue;
                const size_t ij = size_t(i) + size_t(nx) * j;
                double u, v, r;
                if (p == 1) {
                    u = uo[ij]; v = vo[ij]; r = ro[ij];
                } else {
                    const int iw = (i / p) * p, js = (j / p) * p;
                    const double ir = double(i - iw) / p, jr = double(j - js) / p;
                    auto itp = [&](const float* a) {
                        return (1 - ir) * (1 - jr) * at(a, iw, js) + ir * (1 - jr) * at(a, iw + p, js) +
                               (1 - ir) * jr * at(a, iw, js + p) + ir * jr * at(a, iw + p, js + p);
                    };
                    u = itp(uo); v = itp(vo); r = itp(ro);
                }
                if (!cfg.da_obs_ruv) r = o->r[m * nxy + ij];
                for (int q = 0; q < Q; q++) {
                    double& fq = o->f[(m * Q + q) * nxy + ij];
                    fq = alpha * feq(r, u, v, q, o->d.c) + (1 - alpha) * fq;
                }
            }
    }
    return 0;
}

}  // extern "C"
