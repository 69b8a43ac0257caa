// ref_osse_harness.cu -- ORACLE TOOLING (test infrastructure only).
//
// The reference's forecast-and-assimilate cycle (the DA_LETKF loop of main.cu:80-116)
// on one GPU, built from the reference's own pieces where they can be built here:
//
//   * the nature run and each of the M members are one reference `data` object
//     (data.h:45-64: initial condition, forcing, cuRAND stream; the members take the
//     ensemble ids 334 + k that data.cu:34 gives the DA ranks), advanced by the
//     reference's `update()` (lbm.h:16-29) from src/lbm.cu and src/data.cu compiled
//     unmodified where they lie (oracle/Makefile);
//   * every `steps` steps the members are analysed by the reference's LETKF call
//     sequence (ref_letkf_solver.cu: letkf.cu's glue, letkf_solver.h's cuBLAS /
//     cuSOLVER calls) from their current populations into their next buffer; rho and u
//     of the next buffer are refreshed from the analysis and the buffers swap, as
//     assimilate_letkf_uv does after update_xk (letkf.cu:316-355; v is left as it is,
//     the reference's own omission, which only output can see: update() recomputes
//     every macro from f).
//
// Observations: (rho, u, v) of the nature run's post-step macros at every p-th point in
// x and y (p = DA_XYPRUNE of the glue), NaN elsewhere like io/observed files, plus
// Gaussian noise of the glue's OBS_ERROR_RHO / OBS_ERROR_U drawn from std::mt19937(seed)
// with std::normal_distribution<float>, rho, u, v per site, sites in row-major order.
//
// Output, per cycle c = 1 .. cycles (the analysis at step c * steps):
//   int32 c; float32 ro, uo, vo [ny][nx] (the observations used); float32 u_true,
//   v_true [ny][nx] (the nature run's macros); float64 forecast_rmse, analysis_rmse
// where an RMSE is sqrt(mean over the grid of |mean_k (u, v)_k - (u, v)_true|^2): the
// forecast one from the members' post-step macros, the analysis one from the moments of
// the analysis populations (rf, uf, vf of lbm.h:72-109).
//
// usage: ref_osse <M> <cycles> <steps> <seed> <out.bin>
//        ref_osse time <M> <cycles> <steps> <warmup_cycles>
//
// The `time` form measures the cycle of the reference's code on this GPU, as one
// process: the M members each advanced `steps` steps by update() in turn, then the
// analysis (ranks in turn) with one fixed set of observations made from the nature run
// once beforehand, the refresh and the swap; no file output, no RMSE.  After
// `warmup_cycles` untimed cycles it prints
//   ref_osse_time <M> <cycles> <steps> <seconds>
// for `cycles` cycles, CLOCK_MONOTONIC around them with a device synchronisation at
// both ends.  The reference itself runs one MPI rank per member, the members'
// forecasts in separate processes sharing the GPU and the ranks' analyses side by
// side; this measures the same device work issued from one process.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <random>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "config.h"
#include "data.h"
#include "lbm.h"
#include "ref_letkf_glue.h"
#include "ref_letkf_solver.h"

#define CK(x)                                                                                  \
    do {                                                                                       \
        cudaError_t e_ = (x);                                                                  \
        if (e_ != cudaSuccess) {                                                               \
            std::fprintf(stderr, "%s:%d: %s\n", __FILE__, __LINE__, cudaGetErrorString(e_));    \
            std::exit(2);                                                                      \
        }                                                                                      \
    } while (0)

// lbm2euler after update_xk (letkf.cu:336-355): rho and u of the analysis populations
__global__ void k_refresh_ru(const real* fn, real* rn, real* un, int nxy) {
    const int i = threadIdx.x + blockDim.x * blockIdx.x;
    if (i >= nxy) return;
    real fc[config::Q];
    for (int q = 0; q < config::Q; q++) fc[q] = fn[i + size_t(nxy) * q];
    const real rnc = rf(fc);
    rn[i] = rnc;
    un[i] = uf(fc, rnc);
}

// one member's (u, v) moments of populations f, added into the ensemble sums
__global__ void k_add_uv(const real* f, double* su, double* sv, int nxy) {
    const int i = threadIdx.x + blockDim.x * blockIdx.x;
    if (i >= nxy) return;
    real fc[config::Q];
    for (int q = 0; q < config::Q; q++) fc[q] = f[i + size_t(nxy) * q];
    const real rc = rf(fc);
    su[i] += double(uf(fc, rc));
    sv[i] += double(vf(fc, rc));
}

static double rmse(const std::vector<double>& mu, const std::vector<double>& mv, const std::vector<real>& ut,
                   const std::vector<real>& vt) {
    double s = 0;
    for (size_t i = 0; i < ut.size(); i++) {
        const double du = mu[i] - double(ut[i]), dv = mv[i] - double(vt[i]);
        s += du * du + dv * dv;
    }
    return std::sqrt(s / double(ut.size()));
}

static int time_cycles(int argc, char** argv) {
    if (argc != 6) {
        std::fprintf(stderr, "usage: %s time <M> <cycles> <steps> <warmup_cycles>\n", argv[0]);
        return 1;
    }
    const int M = std::atoi(argv[2]), cycles = std::atoi(argv[3]), steps = std::atoi(argv[4]);
    const int warmup = std::atoi(argv[5]);
    const int nx = config::nx, ny = config::ny, nxy = nx * ny;
    const int p = glue::xyprune();
    if (M < 2 || M > 64 || ny % M || cycles < 1 || steps < 1 || warmup < 0) {
        std::fprintf(stderr, "bad arguments\n");
        return 1;
    }
    std::vector<std::unique_ptr<data>> mem;
    for (int k = 0; k < M; k++) mem.emplace_back(new data(334 + k));
    // one set of observations of the nature run after `steps` steps
    std::vector<real> hr(nxy), hu(nxy), hv(nxy), hro(nxy), huo(nxy), hvo(nxy);
    {
        auto nature = data(0);
        for (int t = 0; t < steps; t++) update(nature, t);
        CK(cudaDeviceSynchronize());
        CK(cudaMemcpy(hr.data(), nature.d().r.data(), sizeof(real) * nxy, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(hu.data(), nature.d().u.data(), sizeof(real) * nxy, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(hv.data(), nature.d().v.data(), sizeof(real) * nxy, cudaMemcpyDeviceToHost));
    }
    std::mt19937 gen(1);
    std::normal_distribution<float> nd(0.f, 1.f);
    for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
            const int ij = i + nx * j;
            const bool site = i % p == 0 && j % p == 0;
            hro[ij] = site ? hr[ij] + glue::obs_error_rho() * nd(gen) : NAN;
            huo[ij] = site ? hu[ij] + glue::obs_error_u() * nd(gen) : NAN;
            hvo[ij] = site ? hv[ij] + glue::obs_error_u() * nd(gen) : NAN;
        }
    real *ro, *uo, *vo;
    CK(cudaMalloc(&ro, sizeof(real) * nxy));
    CK(cudaMalloc(&uo, sizeof(real) * nxy));
    CK(cudaMalloc(&vo, sizeof(real) * nxy));
    CK(cudaMemcpy(ro, hro.data(), sizeof(real) * nxy, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(uo, huo.data(), sizeof(real) * nxy, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(vo, hvo.data(), sizeof(real) * nxy, cudaMemcpyHostToDevice));
    const int blocks = (nxy + 255) / 256;
    std::vector<const float*> fin(M);
    std::vector<float*> fout(M);
    int t = 0;
    auto cycle = [&]() {
        for (int s = 0; s < steps; s++, t++)
            for (auto& d : mem) update(*d, t);
        for (int k = 0; k < M; k++) {
            fin[k] = mem[k]->d().f.data();
            fout[k] = mem[k]->dn().f.data();
        }
        refletkf::analyse(fin, fout, ro, uo, vo, nx, ny, 0, ny, nullptr);
        for (auto& d : mem) {
            k_refresh_ru<<<blocks, 256>>>(d->dn().f.data(), d->dn().r.data(), d->dn().u.data(), nxy);
            d->swap();
        }
    };
    for (int c = 0; c < warmup; c++) cycle();
    CK(cudaDeviceSynchronize());
    const auto t0 = std::chrono::steady_clock::now();
    for (int c = 0; c < cycles; c++) cycle();
    CK(cudaDeviceSynchronize());
    const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::printf("ref_osse_time %d %d %d %.6f\n", M, cycles, steps, sec);
    return 0;
}

int main(int argc, char** argv) {
    if (argc >= 2 && std::string(argv[1]) == "time") return time_cycles(argc, argv);
    if (argc != 6) {
        std::fprintf(stderr, "usage: %s <M> <cycles> <steps> <seed> <out.bin>\n", argv[0]);
        return 1;
    }
    const int M = std::atoi(argv[1]), cycles = std::atoi(argv[2]), steps = std::atoi(argv[3]);
    const unsigned seed = unsigned(std::strtoul(argv[4], nullptr, 10));
    const int nx = config::nx, ny = config::ny;
    const int nxy = nx * ny;
    const int p = glue::xyprune();
    const real su = glue::obs_error_u(), sr = glue::obs_error_rho();
    if (M < 2 || M > 64 || ny % M || cycles < 1 || steps < 1) {
        std::fprintf(stderr, "bad arguments\n");
        return 1;
    }
    std::FILE* out = std::fopen(argv[5], "wb");
    if (!out) { std::fprintf(stderr, "cannot write %s\n", argv[5]); return 1; }

    auto nature = data(0);
    std::vector<std::unique_ptr<data>> mem;
    for (int k = 0; k < M; k++) mem.emplace_back(new data(334 + k));

    real *ro, *uo, *vo;
    double *su_d, *sv_d;
    CK(cudaMalloc(&ro, sizeof(real) * nxy));
    CK(cudaMalloc(&uo, sizeof(real) * nxy));
    CK(cudaMalloc(&vo, sizeof(real) * nxy));
    CK(cudaMalloc(&su_d, sizeof(double) * nxy));
    CK(cudaMalloc(&sv_d, sizeof(double) * nxy));
    std::vector<real> hr(nxy), hu(nxy), hv(nxy), hro(nxy), huo(nxy), hvo(nxy), tmp(nxy);
    std::vector<double> mu(nxy), mv(nxy);
    std::mt19937 gen(seed);
    std::normal_distribution<float> nd(0.f, 1.f);
    const int blocks = (nxy + 255) / 256;

    int t = 0;
    for (int c = 1; c <= cycles; c++) {
        for (int s = 0; s < steps; s++, t++) {
            update(nature, t);
            for (auto& d : mem) update(*d, t);
        }
        CK(cudaDeviceSynchronize());
        // the nature run's macros and the observations of them
        CK(cudaMemcpy(hr.data(), nature.d().r.data(), sizeof(real) * nxy, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(hu.data(), nature.d().u.data(), sizeof(real) * nxy, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(hv.data(), nature.d().v.data(), sizeof(real) * nxy, cudaMemcpyDeviceToHost));
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) {
                const int ij = i + nx * j;
                if (i % p == 0 && j % p == 0) {
                    hro[ij] = hr[ij] + sr * nd(gen);
                    huo[ij] = hu[ij] + su * nd(gen);
                    hvo[ij] = hv[ij] + su * nd(gen);
                } else {
                    hro[ij] = huo[ij] = hvo[ij] = NAN;
                }
            }
        CK(cudaMemcpy(ro, hro.data(), sizeof(real) * nxy, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(uo, huo.data(), sizeof(real) * nxy, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(vo, hvo.data(), sizeof(real) * nxy, cudaMemcpyHostToDevice));
        // forecast RMSE: the ensemble mean of the members' post-step macros
        std::fill(mu.begin(), mu.end(), 0.0);
        std::fill(mv.begin(), mv.end(), 0.0);
        for (auto& d : mem) {
            CK(cudaMemcpy(tmp.data(), d->d().u.data(), sizeof(real) * nxy, cudaMemcpyDeviceToHost));
            for (int i = 0; i < nxy; i++) mu[i] += double(tmp[i]);
            CK(cudaMemcpy(tmp.data(), d->d().v.data(), sizeof(real) * nxy, cudaMemcpyDeviceToHost));
            for (int i = 0; i < nxy; i++) mv[i] += double(tmp[i]);
        }
        for (int i = 0; i < nxy; i++) { mu[i] /= M; mv[i] /= M; }
        const double f_rmse = rmse(mu, mv, hu, hv);
        // the analysis: current populations in, next buffer out; rho and u refreshed; swap
        std::vector<const float*> fin(M);
        std::vector<float*> fout(M);
        for (int k = 0; k < M; k++) {
            fin[k] = mem[k]->d().f.data();
            fout[k] = mem[k]->dn().f.data();
        }
        refletkf::analyse(fin, fout, ro, uo, vo, nx, ny, 0, ny, nullptr);
        for (auto& d : mem) {
            k_refresh_ru<<<blocks, 256>>>(d->dn().f.data(), d->dn().r.data(), d->dn().u.data(), nxy);
            CK(cudaGetLastError());
            d->swap();
        }
        CK(cudaDeviceSynchronize());
        // analysis RMSE: the ensemble mean of the analysis populations' moments
        CK(cudaMemset(su_d, 0, sizeof(double) * nxy));
        CK(cudaMemset(sv_d, 0, sizeof(double) * nxy));
        for (auto& d : mem) k_add_uv<<<blocks, 256>>>(d->d().f.data(), su_d, sv_d, nxy);
        CK(cudaGetLastError());
        CK(cudaMemcpy(mu.data(), su_d, sizeof(double) * nxy, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(mv.data(), sv_d, sizeof(double) * nxy, cudaMemcpyDeviceToHost));
        for (int i = 0; i < nxy; i++) { mu[i] /= M; mv[i] /= M; }
        const double a_rmse = rmse(mu, mv, hu, hv);

        std::fwrite(&c, sizeof(int), 1, out);
        std::fwrite(hro.data(), sizeof(real), nxy, out);
        std::fwrite(huo.data(), sizeof(real), nxy, out);
        std::fwrite(hvo.data(), sizeof(real), nxy, out);
        std::fwrite(hu.data(), sizeof(real), nxy, out);
        std::fwrite(hv.data(), sizeof(real), nxy, out);
        std::fwrite(&f_rmse, sizeof(double), 1, out);
        std::fwrite(&a_rmse, sizeof(double), 1, out);
        std::printf("ref_osse cycle %d step %d forecast_rmse %.6e analysis_rmse %.6e\n", c, t, f_rmse, a_rmse);
        std::fflush(stdout);
    }
    std::fclose(out);
    return 0;
}
