// lbl_internal.h -- device-side data structures and kernel launchers shared by the
// liblbl translation units.  Not part of the public ABI (see include/lbl.h).
#pragma once

#include <cuda.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <curand.h>

#include <cstdint>
#include <map>
#include <string>
#include <thread>
#include <vector>

#include "../../include/lbl.h"
#include "closure.h"

namespace lbl {

constexpr int kQ = 9;
constexpr int kMaxModes = 128;     // forcing modes (29 at kf=4)
constexpr int kMaxNobs = 3 * 33 * 33;  // observation window slots (RLOC_LEN <= 8)
constexpr int kMaxMemberLanes = 32;    // warp-resident analysis kernel handles M <= 32
constexpr int kMaxAnalysisMembers = 64; // the 64-thread analysis kernel handles 32 < M <= 64

// Physical constants derived once per context, in the precision the reference
// evaluates them in (config.h:248-254 are constexpr `real` = float).
struct Phys {
    int nx, ny, M;
    int nxy;                 // nx*ny
    float c;                 // u_ref/cfl
    float dx, dt;            // h_ref/(ny-1), dx/c
    float nu;                // molecular viscosity (float, config::nu)
    float cs2;               // c*c/3 (lbm.h:50)
    float fr_dt;             // friction_rate/dt (lbm.h:52, constexpr real)
    float u_ref;
    float two_dx;            // 2*dx (lbm.cu:44-47)
    double les_k;            // cs*cs*dx*dx evaluated in double like lbm.cu:59-60
    double tau_k;            // 3/c/c/dt chain, applied as ((3*nu)/c)/c)/dt in double
    double c_d, dt_d;        // c, dt widened to double for the tau chain
    float inv_nx, inv_ny;    // 1/nx, 1/ny of the global grid for the forcing coordinates
    int y0g, nyg;            // global row of local row 0 and the global row count (a y-slab; else 0, ny)
    // reciprocals of the constant divisors, rounded to float on the host: under
    // -use_fast_math, x / constant rounds exactly like x * (1/constant)
    float inv_c, inv_c2, inv_cs2, inv_two_dx;
};

// LETKF geometry (letkf.cu:29-56)
struct Geo {
    int p;        // DA_XYPRUNE
    int nl;       // n_obs_local
    int off;      // obs_offset
    int nox;      // n_obs_x
    int nobs;     // 3*nox*nox
    double dloc;  // d_local (GC length)
    int nsx, nsy; // observation sites per row / column (nx/p, ny/p)
};

struct TimerMap {
    std::map<std::string, double> map;
    std::string cur = "_uninitialized";
    double t0 = 0;
};

}  // namespace lbl

struct lbl_ctx {
    lbl_config cfg{};
    lbl::Phys P{};
    lbl::Geo G{};
    int device = 0;
    int ens_offset = 0;
    bool initialised = false;
    int phases = 0;                      // phase events of the last graph: 0 none, 1 forecast, 2 analysis + forecast
    std::string err;
    cudaStream_t stream = nullptr;
    cudaStream_t side = nullptr;         // forcing branch of the cycle graph
    cudaStream_t hi = nullptr;           // analysis branch of the cycle graph, at the highest priority
    cudaEvent_t fork_ev = nullptr, join_ev = nullptr, hi_ev = nullptr;

    // ensemble state, double buffered like data::d()/dn() (data.h:45-64)
    float* f[2] = {nullptr, nullptr};    // [M][9][ny][nx] FP32 populations (LBL_STORAGE_F32)
    __half* h[2] = {nullptr, nullptr};   // [M][9][ny][nx] FP16 deviations f - w_q (LBL_STORAGE_F16)
    float* fs[2] = {nullptr, nullptr};   // FP32 forecast / analysis copies for the analysis (FP16 storage)
    bool f16 = false;                    // storage == LBL_STORAGE_F16
    float* mac[2] = {nullptr, nullptr};  // [M][3][ny][nx]  rho, u, v (post-stream macros)
    int cur = 0;                         // index of d()

    // forcing (data.cu:161-350)
    int n_modes = 0;
    float h_kx[lbl::kMaxModes], h_ky[lbl::kMaxModes], h_amp[lbl::kMaxModes];
    double h_amps[2 * lbl::kMaxModes];   // the FP64 per-mode factors held in d_amps
    float* d_modes = nullptr;            // [2][n_modes] kx, ky
    double* d_amps = nullptr;            // [2][n_modes] amp*2*pi*ky, amp*2*pi*(-kx) in FP64
    curandGenerator_t gen = nullptr;
    int n_rand_buf = 0;                  // 4096 * n_modes
    int i_rand_outdated = 0;             // cursor of data.cu:240-247
    long long rand_block = -1;           // index of the normal block currently in use
    int pool_slots = 4;
    float* d_pool = nullptr;             // [pool_slots][n_rand_buf]
    int force_cap = 0;                   // steps the force buffer holds
    float* d_force = nullptr;            // [force_cap][2][ny][nx]
    int* d_sched = nullptr;              // [force_cap] offsets into d_pool
    int* h_sched[2] = {nullptr, nullptr};  // pinned staging, alternating
    int sched_buf = 0;
    int last_sched = 0;                  // pool offset used by the last step's forcing
    int last_force_slot = 0;             // force-buffer slot of the last step

    // LETKF
    int* d_wtab = nullptr;               // int4 [p*p][nobs] window entries + int [p*p] counts
    float* d_wdense = nullptr;           // LBL_GRAM_TF32X3: [p*p][kpad] slot weights per pattern
    float* d_Q = nullptr;                // LBL_GRAM_TF32X3: Q - (M-1)/beta I per point, [nxy][mpq][mpq],
                                         // then c = dY^T R^-1 dyo per point, [nxy][mpq]
    float* d_yo = nullptr;               // [3][nsites] observations at sites (u, v, rho)
    bool have_obs = false;               // d_yo holds observations given by the caller
    float* h_yo[2] = {nullptr, nullptr}; // pinned staging of the above, alternating
    int yo_buf = 0;
    float* d_dY = nullptr;               // [3][nsites][M] H(x)-mean at sites
    float* d_dyo = nullptr;              // [3][nsites] yo - mean
    int* d_stats = nullptr;              // [0] max sweeps, [1] non-converged points, [2] NaN flag, [3] sweep total
    int h_stats[4] = {0, 0, 0, 0};

    // diagnostics scratch
    double* d_red = nullptr;             // reduction scratch (8 doubles)
    float* d_tmp = nullptr;              // nxy*2 floats (truth fields)
    float* d_dump = nullptr;             // LETKF matrix dump of one chunk (write_mat only)
    std::vector<float> h_dump;
    std::string io_prefix = "io";        // config::prefix (config.h:287) for the matrix dumps

    // OBSERVE noise engine state lives host side (io.cu:321 function-static engine)
    void* obs_engine = nullptr;          // std::mt19937*
    std::vector<float> h_obs[4];         // last generated observed rho, u, v, vor

    // TMA descriptors of the two population buffers (input side of a step)
    CUtensorMap tmap[2];
    bool use_tma = false;
    int vec = 0;                         // columns per thread of the vector-load stream-collide (0: one)
    bool vec_pf = false;                 // its march prefetches the row after next
    bool vec_auto = false;               // LBL_LBM_AUTO: lbl_autotune may change the columns per thread
    int ty_held = 0;                     // strip height of the closure's held-multiplier steps (0: ty's)
    int ty_tuned = 0;                    // stream-collide strip height chosen by lbl_autotune (0: heuristic)
    int ty_default = 0;                  // the heuristic's strip height for the kernel that runs
    int* d_err = nullptr;                // bounded-wait timeout flag of the TMA kernel
    int inject_tma_stall = 0;            // lbl_inject: > 0 = TMA producer issues nothing, waits poll this often

    // asynchronous output (lbl_output_async): vorticity and ensemble statistics on the
    // device, one pinned staging copy, and a writer thread for the files
    float* d_outf = nullptr;             // [M][nxy] vorticity, [4][nxy] statistics, 1 int NaN flag
    float* h_outf = nullptr;             // pinned: [M][3][nxy] macros, then the above
    cudaEvent_t out_ev = nullptr;        // the staging copy is complete
    std::thread out_thread;
    int out_rc = 0;                      // the writer's status and message
    std::string out_err;

    // learned closure (closure.h): fragment-ordered BF16 parameters, feature scales
    uint32_t* d_closure = nullptr;       // [kPackWords]
    int closure_every = 1;               // lbl_set_closure_refresh: the network runs every this many steps
    float* d_mclos = nullptr;            // [M][ny][nx] the cells' multipliers between evaluations (closure_every > 1)
    bool closure = false;
    lbl::ClosureScales closure_sc{};

    // y-slab split (lbl_slab_set): this context holds the global rows [slab_row0, slab_row0 + ny - 2 slab_halo)
    // of a grid of slab_ny rows, plus slab_halo rows on each side; slab_ny = 0 for a whole grid
    int slab_ny = 0, slab_row0 = 0, slab_halo = 0;
    int fc_total = 0, fc_off = 0;        // chunked forecast (lbl_slab_forecast_begin): steps begun, steps done
    bool fc_free_recorded = false;       // ev[15] follows the last reader of the forcing slots

    // CUDA graphs keyed by (kind, n, parity)
    std::map<long long, cudaGraphExec_t> graphs;

    // timers
    lbl::TimerMap timers[2];
    cudaEvent_t ev[17] = {};             // 0-3 stage timing, 4-5 sched staging, 6-7 obs staging, 8-9 profile,
                                         // 10-12 phase events recorded inside the graphs, 13-14 the
                                         // asynchronous RMSE's true fields (arrived / read), 15-16 a chunked
                                         // forecast's forcing slots (free after its last step / filled)
    cudaEvent_t user_ev[8] = {};         // lbl_event_record slots
    bool have_events = false;
};

namespace lbl {

// ---- kernels (lbm_kernels.cu, compiled with the reference's -use_fast_math) ----
void launch_ic_velocity(const double* modes /*[4][n]*/, int n_modes, int nx, int ny,
                        float* u, float* v, cudaStream_t s);
void launch_force_chunk(const lbl_ctx* c, int nsteps, int slot0, cudaStream_t s);
// y-slab halos (slab.cu): rows [a_prev, a_prev + rows) and [a_next, a_next + rows) of every (member, q)
// plane of the populations `f` (elem bytes each) to / from two packed buffers [plane][rows][nx]
void launch_slab_halo(void* f, size_t elem, int nx, int ny, int planes, int rows, int a_prev, int a_next,
                      void* buf_prev, void* buf_next, bool unpack, cudaStream_t s);
// one step from population buffer src to dst (FP32 or FP16 storage)
// pdl: the previous launch on s is the previous step; the launch may then overlap its
// tail (programmatic dependent launch; the kernel waits for that grid's completion)
// step: the step's index in its forecast chunk (it picks the closure's evaluate-or-hold variant)
void launch_lbm_step(const lbl_ctx* c, int src, int dst, const float* force, float* mac_out, cudaStream_t s,
                     bool pdl = false, int step = 0);
// strip height of the stream-collide for this grid, ensemble and kernel variant
// (occupancy heuristic); call outside stream capture
int lbm_strip_rows(const lbl_ctx* c);
int lbm_strip_rows_held(const lbl_ctx* c);  // for the closure's held-multiplier steps
// fill both population buffers with the rest state (rho = rho_ref, u = v = 0)
void launch_rest_state(const lbl_ctx* c, cudaStream_t s);
// FP16 deviation storage <-> FP32 populations, all members
void launch_expand(const lbl_ctx* c, const __half* h, float* f, cudaStream_t s);
void launch_compress(const lbl_ctx* c, const float* f, __half* h, cudaStream_t s);
// dynamic shared memory of the learned-closure stream-collide for rows of nx columns
size_t closure_step_smem(int nx);
// CTAs per row of the stream-collide: 1 up to 1024 columns, else a cluster of up to
// 8 CTAs of 1024, 512 or 256 columns; 0 = unsupported width
int cluster_chunks(int nx);
int lbm_tma_prepare(int nx);
bool lbm_tma_supported(int nx);
size_t lbm_tma_smem(int nx);
void launch_macros(const lbl_ctx* c, int buf, float* mac, cudaStream_t s);

// Batched persistent stream-collide (lbl_batch_*): one launch steps every experiment
// of a batch; work items are (experiment, member, strip, kBatchW-column chunk)
constexpr int kBatchW = 128;
constexpr int kMaxBatch = 16;
struct BatchExp {
    float* f[2];           // population buffers (FP32)
    float* mac[2];         // macro buffers
    const float* force;    // forcing chunk, [step][2][nxy]
    Phys P;
    int ty, strips, chunks, item0;  // strip height, strips per member, chunks per row, first item
    int cur;               // buffer read by step 0 of the launched sequence
};
// step `step` of every experiment (exps: device table sorted by item0, counter[step]
// zeroed before); mac: write the macros (the last two steps of a forecast)
void launch_batch_step(const BatchExp* exps, int n_exp, int total, int step, int* counter, int grid, bool mac,
                       bool pdl, cudaStream_t s);
int batch_step_slots();  // resident CTAs of the batched kernel on the current device

// ---- kernels (letkf_kernels.cu) ----
void launch_obs_ensemble(const lbl_ctx* c, const float* f, cudaStream_t s);
void launch_nudging(const lbl_ctx* c, int buf, const float* mac, cudaStream_t s);
void launch_analysis(const lbl_ctx* c, const float* fin, float* fout, float* mac_out, cudaStream_t s);
// LETKF matrix dumps (need_save_mat, letkf_solver.h:243-345): the 14 matrices of the
// rows [j0, j1), each [rows][cols][points] column-major with the point slowest, laid
// out one after the other in buf in the order of kDumpLabels
constexpr int kDumpCount = 14;
constexpr const char* kDumpLabels[kDumpCount] = {"_dYf", "_dyo", "_Q", "_V", "_Xf", "_dXf", "_Pa",
                                                 "_dWa", "_Xa", "_Wa", "_AI", "_Z", "_Lambda", "_Wma"};
void dump_sizes(int M, int nobs, size_t nb, size_t* sz);
void launch_analysis_dump(const lbl_ctx* c, const float* fin, float* buf, int j0, int j1, cudaStream_t s);
int write_h5_dataset(const std::string& path, const uint64_t dims[3], const void* data, bool is_double,
                     std::string& err);
int analysis_supported(int M);
size_t analysis_smem_bytes(int M, int nobs);
constexpr size_t kAnalysisSmemLimit = 200 * 1024;
int analysis_prepare();

// Explicit-pointer form of the analysis launch (no context), used by the entry
// point that allocates no device memory (noalloc.cu).
struct AnalysisArgs {
    const float* f_in;        // [M][9][ny][nx]
    float* f_out;             // [M][9][ny][nx]
    float* mac_out;           // [M][3][ny][nx]
    const float* yo;          // [3][nsites] u, v, rho at the sites
    float* dY;                // [3][nsites][M] scratch
    float* dyo;               // [3][nsites] scratch
    const int* wtab;          // int4 [p*p][nobs] + int [p*p] counts
    int* stats;               // int[4] scratch
    int nx, ny, M, p, nox, nl_off, nobs;
    float diag, sqrt_m1, tol, c;
    int max_sweeps, write_v;
};
void launch_obs_ensemble_args(const AnalysisArgs& a, cudaStream_t s);
// ---- the Gram on the tcgen05 tensor cores (gram_tc.cu) ----
struct GramTcParams {
    int nx, ny, M, p, nsx, nsy, nsites, nox, nl_off, nobs, kpad;
};
// M <= 64, p^2 a multiple of the points per 128-row tile, operands within shared memory
bool gram_tc_supported(int M, int p, int nobs);
size_t gram_tc_smem(int M, int p, int nobs);
int gram_tc_prepare();
// member padding of the Gram output Qout[point][mpq][mpq]: 16, 32 or 64
inline int gram_tc_mp(int M) { return M <= 16 ? 16 : (M <= 32 ? 32 : 64); }
// Qout = Q - (M-1)/beta I and Cout = dY^T R^-1 dyo for every grid point; wdense [p*p][kpad] =
// the slot weights of each pattern (i mod p, j mod p), zero for absent slots and the padding
void launch_gram_tc(const GramTcParams& G, const float* dY, const float* dyo, const float* wdense, float* Qout,
                    float* Cout, int* err, cudaStream_t s);

void launch_analysis_args(const AnalysisArgs& a, cudaStream_t s);

// ---- kernels (diag_kernels.cu) ----
void launch_diag(const lbl_ctx* c, const float* mac, int member, double* red, cudaStream_t s);
// per-member vorticity [M][nxy] and ensemble statistics [4][nxy] (mean u, mean v,
// mean vor, std vor) in the reference's FP32 order; *nan |= 1 on a NaN vorticity
void launch_output_fields(const lbl_ctx* c, const float* mac, float* vor, float* stats, int* nan, cudaStream_t s);
void launch_rmse(const lbl_ctx* c, const float* mac, const float* ut, const float* vt, double* red,
                 cudaStream_t s);
void launch_rmse_finish(const lbl_ctx* c, double* red, cudaStream_t s);
void rmse_cells(const lbl_ctx* c, int* ij0, int* n);  // the cells an RMSE covers

// ---- host helpers (host_io.cpp) ----
std::string to_string_aligned(int t, int digits);
int write_dat(const std::string& fname, const float* p, size_t n, std::string& err);
int read_dat(const std::string& fname, float* p, size_t n, std::string& err);
int mkdir_p(const std::string& path);
void vorticity_host(int nx, int ny, float dx, const float* u, const float* v, float* vor);
void* obs_engine_new(uint32_t seed);
void obs_engine_free(void* e);
void observe_host(void* engine, int nx, int ny, int p, float er, float eu, const float* r, const float* u,
                  const float* v, float* ro, float* uo, float* vo, float* voro, float dx);
double wall_time();
void timer_transit(TimerMap& t, const std::string& tag);
void timer_add(TimerMap& t, const std::string& tag, double sec);
std::string timer_csv(const TimerMap& t);

}  // namespace lbl
