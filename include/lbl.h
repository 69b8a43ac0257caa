/*
 * lbl.h -- C ABI of liblbl, the B200-native forecast-and-assimilate engine
 * (D2Q9 BGK + Smagorinsky lattice Boltzmann ensemble + LETKF analysis).
 *
 * One context (lbl_ctx) holds a whole ensemble of M members resident on one GPU
 * as a batch dimension.  It replaces the reference's one-MPI-rank-per-member
 * design: the reference's entry points for this path are the C++ functions
 *
 *   void update(data&, int t)                                  src/lbm.h:16-29
 *   void DataAssimilator::assimilate(data&, const mpi&, int t)  src/assimilate.h:54-68
 *   void output(const data&, util::mpi, int t)                  src/io.h:7, src/io.cu:22
 *   data::data(int ensemble_id)                                 src/data.h:55, src/data.cu:25-303
 *
 * and the run-time knobs are the compile-time macros of src/config.h and
 * config/makefile.macro.in, which lbl_config mirrors field by field.
 *
 * Conventions
 *   - every function returns int: 0 = LBL_OK, negative = error;
 *     lbl_last_error(ctx) gives the message of the last failure on that ctx;
 *   - no C++ exception crosses this boundary;
 *   - caller buffers are plain host pointers borrowed for the duration of the call;
 *   - a ctx owns all device memory, its stream and its CUDA graphs; one ctx per
 *     host thread; calls are synchronous on return unless named *_async.
 *   - field arrays are float32, nx*ny values, i (x) fastest, like the
 *     reference's ij(i,j) = i + nx*j (src/config.h:210).  Populations f are
 *     [q][y][x] per member (src/config.h:212, ijq = ij + nx*ny*q).
 */
#ifndef LBL_H_
#define LBL_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LBL_ABI_VERSION 2

/* status codes */
#define LBL_OK              0
#define LBL_ERR_ARG        -1   /* bad argument / configuration value          */
#define LBL_ERR_CUDA       -2   /* CUDA runtime error                          */
#define LBL_ERR_CURAND     -3   /* cuRAND error                                */
#define LBL_ERR_IO         -4   /* file could not be read / written            */
#define LBL_ERR_NAN        -5   /* NaN detected (reference: io.cu:79-83,       */
                                /*  letkf_solver.h:352-364)                    */
#define LBL_ERR_STATE      -6   /* call out of order (e.g. update before init) */
#define LBL_ERR_NOMEM      -7   /* device allocation failed                    */
#define LBL_ERR_UNSUPPORTED -8  /* configuration not supported by this build   */
#define LBL_ERR_NOCONV     -9   /* Jacobi eigensolver hit its sweep limit      */
#define LBL_ERR_TIMEOUT   -10   /* a bounded wait inside a kernel gave up      */

/* stream-collide kernel variants (lbl_config.lbm_variant) */
#define LBL_LBM_AUTO   0    /* direct loads, 1 or 2 columns per thread by storage and
                               width (the fastest measured on B200); lbl_autotune
                               may pick 1, 2 or 4                                */
#define LBL_LBM_DIRECT 1    /* per-thread global loads, 1 column per thread       */
#define LBL_LBM_TMA    2    /* rows streamed into shared memory by the TMA unit  */
#define LBL_LBM_VEC    3    /* 4 columns per thread: 128-bit loads and stores of
                               FP32 rows (64-bit for FP16 deviations), nx <= 1024 */
#define LBL_LBM_VEC2   4    /* 2 columns per thread: 64-bit (FP16: 32-bit)        */

/* population storage (lbl_config.storage) */
#define LBL_GRAM_F32  0  /* Gram dY^T R^-1 dY in FP32 (the reference's arithmetic)                       */
#define LBL_GRAM_BF16 1  /* precision form: BF16 operands on the tensor cores, FP32 sums; 32 < M <= 64   */
#define LBL_GRAM_TF32X3 2 /* the Gram of every p x p block on the tcgen05 tensor cores, FP32-accurate:      */
                          /* operands split into two TF32 terms, three MMAs, FP32 sums; M <= 64 and p*p a   */
                          /* multiple of 128/MP (MP = 16, 32, 64 members padded), e.g. p = 4             */
#define LBL_STORAGE_F32 0    /* FP32 populations (the reference's `real`)                   */
#define LBL_STORAGE_F16 1    /* FP16 deviations f - w_q from the lattice weights, FP32 collide */

/* run modes: the reference's -DTEST=<mode> (src/config.h:28-108) */
#define LBL_MODE_NATURE   0
#define LBL_MODE_OBSERVE  1
#define LBL_MODE_DA_LETKF 2
#define LBL_MODE_DA_NUDGING 3  /* DA_NUDGING: relax f toward feq of the observations (src/nudging.cu:40-143) */

/* initial condition kinds */
#define LBL_IC_REFERENCE  0  /* src/data.cu:53-120: band exp(-(k-kf)^2/5), |k-kf|<=10, max|u| = ic_amp */
#define LBL_IC_K4EXP      1  /* E(k) ~ k^4 exp(-2 (k/4)^2), rms |u| = ic_amp (physical units)          */

/* initial ensemble kinds */
#define LBL_ENS_INDEPENDENT 0 /* member k: own random phases, seed = k + ofs + 334 (src/data.cu:31-35) */
#define LBL_ENS_PERTURBED   1 /* member k: nature IC + independent random-phase field at ens_perturb amplitude */

/* timer selectors for lbl_timer_csv */
#define LBL_TIMER_MAIN  0    /* io/elapsed_time_rank%d.csv       (src/main.cu:143)  */
#define LBL_TIMER_LETKF 1    /* io/letkf_elapsed_time_rank%d.csv (src/main.cu:145)  */

typedef struct lbl_config {
    int32_t abi_version;     /* must be LBL_ABI_VERSION                                   */
    int32_t mode;            /* LBL_MODE_*                                                */
    int32_t nx, ny;          /* grid; reference NX = 64*SCALER, square (config.h:88-89)   */
    int32_t n_ens;           /* M, ensemble members (reference: MPI ranks)                */
    int32_t iiter;           /* steps per output slot; reference 5*SCALER (config.h:136)  */
    int32_t ioprune;         /* IOPRUNE (config.h:90-92)                                  */
    int32_t daprune;         /* DAPRUNE (config.h:55-57)                                  */
    int32_t da_xyprune;      /* DA_XYPRUNE, observation spacing p (config.h:59-61)        */
    int32_t letkf_rloc_len;  /* LETKF_RLOC_LEN; 0 = macro undefined (letkf.cu:45-55)      */
    int32_t iter_main;       /* iiter*2000 in the reference (config.h:144)                */
    int32_t spinup;          /* spin-up steps; reference 100000*iiter (config.h:139)      */
    int32_t ic_kind;         /* LBL_IC_*                                                  */
    int32_t ens_init;        /* LBL_ENS_*                                                 */
    int32_t compat_stale_v;  /* 1: after an analysis v is not refreshed (letkf.cu:340-355) */
    int32_t jacobi_max_sweeps; /* reference syevj: 100 (cu_matrix_eigensolver_wrapper.hpp:193) */
    int32_t write_mat;       /* need_save_mat (letkf.cu:33): dump the LETKF matrices each analysis */
    int32_t lbm_variant;     /* LBL_LBM_* (stream-collide implementation)                 */
    double letkf_covinf;     /* LETKF_COVINF, multiplicative inflation beta (config.h:48-50) */
    double obs_error_rho;    /* OBS_ERROR_RHO (config.h:190-202)                          */
    double obs_error_u;      /* OBS_ERROR_U                                               */
    double cs;               /* Smagorinsky constant; reference hard-codes 0.2 (lbm.cu:59) */
    double nu;               /* molecular viscosity; reference 1e-4 (config.h:157)        */
    double tau;              /* if > 0 overrides nu: nu = (tau-0.5)*c*c*dt/3              */
    double cfl;              /* 0.05 (config.h:153)                                       */
    double rho_ref;          /* 1    (config.h:156)                                       */
    double u_ref;            /* 1    (config.h:182)                                       */
    double h_ref;            /* 2*pi (config.h:158)                                       */
    double kf;               /* forcing wavenumber 4 (config.h:161)                       */
    double fkf;              /* forcing amplitude 5.6 at nx=256 (config.h:171)            */
    double friction_rate;    /* 5e-4 (config.h:180)                                       */
    double ic_amp;           /* 0.01 = reference p_amp (data.cu:53)                       */
    double ens_perturb;      /* amplitude ratio for LBL_ENS_PERTURBED                     */
    double jacobi_tol;       /* reference syevj: 1e-6 (cu_matrix_eigensolver_wrapper.hpp:192) */
    uint64_t force_seed;     /* cuRAND MTGP32 seed, 1991 (data.cu:294)                    */
    uint64_t obs_seed;       /* OBSERVE noise engine seed 334 (io.cu:321)                 */
    /* appended in ABI version 2 */
    int32_t da_dummy;        /* DA_DUMMY (config.h:71-74): a DA run without analyses (main.cu:94) */
    int32_t da_quadra;       /* DA_QUADRA (config.h:63-65): nudge only x < nx/2 (odd), y < ny/2 (>= 2) */
    int32_t da_obs_ruv;      /* 1: DA_OBS_RUV, rho observed (config.h:44); 0: DA_OBS_UV, model rho */
    int32_t gram;            /* LBL_GRAM_*: the analysis Gram in FP32 or on BF16 tensor cores */
    double da_nud_rate;      /* DA_NUD_RATE, nudging weight alpha, 0.1 (config.h:67-69)   */
    int32_t storage;         /* LBL_STORAGE_* (the precision form stores FP16 deviations)  */
    int32_t reserved1;       /* must be 0                                                 */
} lbl_config;

typedef struct lbl_ctx lbl_ctx;

/* Fill *cfg with the reference's defaults for a run mode at grid nx (= 64*SCALER)
 * and ensemble size n_ens: config.h with SCALER = nx/64, LES on, FORCE_TURB on.
 * OBS_ERROR_* have no default in the reference (config.h:195 #error); they are
 * set to the values of run/jserr:146-147 (rho 0.01, u 0.1). */
int lbl_config_default(lbl_config* cfg, int mode, int nx, int n_ens);

/* Create a context on CUDA device `device`.  Replaces data(rank+ofs) allocation
 * plus DataAssimilator(mpi) (main.cu:58-61).  No initial condition yet. */
int lbl_create(const lbl_config* cfg, int device, lbl_ctx** out);
int lbl_destroy(lbl_ctx* ctx);
const char* lbl_last_error(const lbl_ctx* ctx);   /* never NULL */
const char* lbl_version(void);

/* Initial condition of every member and forcing initialisation.
 * ens_offset is main.cu's argv[1] (main.cu:42-45): member k uses ensemble id
 * k + ens_offset (seed +334 in DA_LETKF, data.cu:31-35).
 * Replaces stdata::init_lbm (data.cu:25-141) and init_force/init_forces
 * (data.cu:143-237), including the two update_forces calls made at init. */
int lbl_init(lbl_ctx* ctx, int ens_offset);

/* nsteps LBM steps of every member: update(dat, t0), ..., update(dat, t0+nsteps-1)
 * (lbm.h:16-29: forcing refresh, pull streaming + macros, Smagorinsky, BGK+force,
 * swap).  t is accepted for interface parity; the reference ignores it. */
int lbl_update(lbl_ctx* ctx, int t0, int nsteps);
int lbl_update_async(lbl_ctx* ctx, int t0, int nsteps);

/* One LETKF analysis at time t, observations given as host arrays (nx*ny each,
 * NaN off the observation lattice, like io/observed/ens0000/{rho,u,v}_step*.dat).
 * Replaces DataAssimilator::assimilate -> assimilate_letkf_uv (letkf.cu:120-360),
 * including its `(t/iiter) % daprune` gate: returns LBL_OK without work off-cycle. */
int lbl_assimilate(lbl_ctx* ctx, int t, const float* rho_o, const float* u_o, const float* v_o);
int lbl_assimilate_async(lbl_ctx* ctx, int t, const float* rho_o, const float* u_o, const float* v_o);
/* Same, reading io/observed/ens0000/{rho,u,v}_step%010d.dat under `io_prefix`
 * (letkf.cu:197-220). */
int lbl_assimilate_files(lbl_ctx* ctx, int t, const char* io_prefix);

/* One forecast-and-assimilate cycle: analysis at t (if due) followed by
 * n_fc forecast steps, launched as one CUDA graph.  Given observations become the
 * resident ones (also when the DA gate skips this call's analysis); NULL observation
 * pointers reuse them, and a due analysis with none given yet is LBL_ERR_STATE. */
int lbl_cycle_async(lbl_ctx* ctx, int t, const float* rho_o, const float* u_o, const float* v_o, int n_fc);
int lbl_sync(lbl_ctx* ctx);  /* also waits for a pending lbl_output_async writer */

/* output(dat, mpi, t) (io.cu:22-266): writes the reference's .dat files under
 * io_prefix for the mode (calc/, nature/, observed/, ensemble statistics).
 * Gate `t % (iiter*ioprune) == 0` as in the reference.  The vorticity and the
 * ensemble statistics are computed on the GPU in the reference's FP32 operation
 * order (the files match its host loops bit for bit). */
int lbl_output(lbl_ctx* ctx, int t, const char* io_prefix);
/* The same output without waiting for the files: the fields are computed and copied
 * to a pinned staging buffer in stream order, and a host thread writes the files
 * while later forecasts run.  The next lbl_output / lbl_output_async, lbl_sync,
 * lbl_get_observed, lbl_assimilate_files or lbl_destroy waits for that writer and
 * returns its status (LBL_ERR_NAN, LBL_ERR_IO).  (The reference writes synchronously,
 * io.cu:22-266.) */
int lbl_output_async(lbl_ctx* ctx, int t, const char* io_prefix);

/* Field access (parity injection and inspection). */
int lbl_get_f(lbl_ctx* ctx, int member, float* f /* 9*nx*ny */);
int lbl_set_f(lbl_ctx* ctx, int member, const float* f);
int lbl_get_fields(lbl_ctx* ctx, int member, float* rho, float* u, float* v, float* vor);
int lbl_get_ens_stats(lbl_ctx* ctx, float* u_mean, float* v_mean, float* vor_mean, float* vor_std);
int lbl_get_force(lbl_ctx* ctx, float* fx, float* fy);
/* The 4*n_modes normals the forcing of the last step used, the mode table and
 * the reference's buffer cursor (data.cu:239-350). */
int lbl_get_force_state(lbl_ctx* ctx, float* randoms /* 4*n_modes */, float* kx, float* ky,
                        float* amp, int* n_modes, int* i_rand_outdated);
/* Observations generated by OBSERVE mode at the last output (host copies). */
int lbl_get_observed(lbl_ctx* ctx, float* rho_o, float* u_o, float* v_o, float* vor_o);
/* Analysis diagnostics of the last assimilate: max Jacobi sweeps, number of
 * grid points that hit the sweep limit, NaN flag, sweeps summed over grid points. */
int lbl_get_letkf_stats(lbl_ctx* ctx, int* max_sweeps, int* n_noconv, int* nan_flag, int* total_sweeps);
/* FP64 domain reductions of member `member` (-1 = ensemble mean fields):
 * kinetic energy, enstrophy, mass (src/data.cu:458-542 inspect()). */
int lbl_get_diagnostics(lbl_ctx* ctx, int member, double* energy, double* enstrophy, double* mass);
/* RMSE of the ensemble-mean (u,v) against host truth fields (FP64). */
int lbl_rmse_uv(lbl_ctx* ctx, const float* u_true, const float* v_true, double* rmse);

/* lbl_rmse_uv without waiting: enqueues the upload of the true fields (on the context's
 * second stream, so that it overlaps the work already queued, such as a cycle's forecast),
 * the FP64 reduction and the copy of the RMSE into *rmse on the context's stream, and returns.
 * u_true, v_true and rmse must stay valid (and the fields unchanged) until the stream
 * has passed this point (lbl_sync, an lbl_event_elapsed on a later event, or the next
 * blocking call); in pinned host memory the copies are asynchronous. */
int lbl_rmse_uv_async(lbl_ctx* ctx, const float* u_true, const float* v_true, double* rmse);

/* The context's CUDA stream (a cudaStream_t), for ordering a caller's own device work
 * with the context's: work the caller enqueues on it runs between the context's calls
 * in submission order.  Valid until lbl_destroy. */
void* lbl_get_stream(lbl_ctx* ctx);

/* Profiling: n back-to-back launches of the fused stream-collide kernel on the
 * context's stream, timed with CUDA events; *ms_per_launch = average per launch.
 * The state advances by n steps with the last computed force field. */
int lbl_profile_step(lbl_ctx* ctx, int n, double* ms_per_launch);
/* Device time of the phases of the last graph that lbl_update / lbl_update_async /
 * lbl_cycle_async launched, from events recorded inside the graph: *analysis_ms =
 * observation operator + LETKF analysis (with the forcing chunk beside it; 0 for a
 * forecast-only graph), *forecast_ms = the n stream-collide launches (a forecast-only
 * graph runs its forcing chunk first and counts it here).  Waits for the
 * graph to finish.  No counterpart in the reference (its util/timer.hpp timers are
 * host clocks around synchronised calls; those are lbl_timer_*). */
int lbl_get_cycle_phases(lbl_ctx* ctx, double* analysis_ms, double* forecast_ms);

/* CUDA events on the context's stream, for device-side timing by callers:
 * slot in [0, 8).  lbl_event_elapsed waits for slot b and returns ms from a to b. */
int lbl_event_record(lbl_ctx* ctx, int slot);
int lbl_event_elapsed(lbl_ctx* ctx, int slot_a, int slot_b, double* ms);

/* LETKF analysis for callers that cannot allocate device memory.  No counterpart
 * in the reference: it serves code that owns every GPU buffer (a framework with
 * its own caching allocator or memory budget, where a hidden cudaMalloc would
 * overrun its pool and synchronise the device).  The caller passes device
 * pointers to the forecast populations f_in [M][9][ny][nx], the output
 * populations f_out and macros mac_out [M][3][ny][nx] (rho, u and, unless
 * compat_stale_v, v), and the observations at the sites yo_sites
 * [3][ny/p][nx/p] (u, v, rho; site (si, sj) is grid point (si*p, sj*p)).  The
 * analysis scratch lives in one static device array of 8 MiB; configurations
 * needing more are rejected with LBL_ERR_UNSUPPORTED.  CUDA loads that array
 * lazily: the first call on a device takes the 8 MiB (and the module holding it)
 * from the device, so make it during set-up, before a memory budget is fixed; the
 * device then holds it until exit.  The first call on a device also looks the
 * array up (cudaGetSymbolAddress) and must come before any stream capture.  All
 * calls share the array: calls that overlap on the GPU race and must be
 * serialised.  Every call only enqueues kernels and a memset on `stream` (a
 * cudaStream_t, NULL = legacy default stream): the window weight table is rebuilt
 * on the device and the counters cleared each time, with no host memory involved.
 * host_stats (int[4]: max sweeps, non-converged points, NaN flag, sweep total) is
 * optional; given, the call waits for the stream and returns LBL_ERR_NAN on a NaN
 * in the analysis.  Without it the call does not wait and cannot report a NaN.
 * err (optional) receives a message of at most err_cap bytes. */
int lbl_letkf_analysis_noalloc(const lbl_config* cfg, const float* f_in, float* f_out, float* mac_out,
                               const float* yo_sites, void* stream, int* host_stats, char* err, size_t err_cap);

/* Fault injection for tests of the failure paths.  No counterpart in the reference,
 * whose failures abort the MPI job (main.cu:152-155).  what = LBL_INJECT_TMA_STALL:
 * from the next stream-collide on, the TMA-fed kernel's producer issues no bulk copy and
 * every bounded wait polls at most `value` (1 .. 2^20) times, so the consumers' waits run
 * out with nothing in flight, no population is written and the call (or the next
 * lbl_sync) returns LBL_ERR_TIMEOUT; the context stays usable (re-run lbl_init).
 * what = LBL_INJECT_NONE clears it.  Waits for the context's work and drops its captured
 * graphs.  Nothing here faults or hangs a GPU. */
#define LBL_INJECT_NONE      0
#define LBL_INJECT_TMA_STALL 1
int lbl_inject(lbl_ctx* ctx, int what, int value);

/* Tile autotuning for this context's grid and ensemble size: times the fused
 * stream-collide on the rest state for candidate strip heights (rows per CTA), and for
 * the vector-load kernel both forms of its march, and keeps the fastest for every
 * later step.  Call between lbl_create and lbl_init (it
 * overwrites the populations).  *strip_rows / *ms_per_launch (optional) receive
 * the choice and its time.  No counterpart in the reference. */
int lbl_autotune(lbl_ctx* ctx, int* strip_rows, double* ms_per_launch);

/* The stream-collide launch shape the context runs: columns per thread (1, or 2 / 4 for
 * the vector-load kernel), whether its march prefetches the row after next (1 for the
 * one-column kernels), and the strip height (rows per CTA).  lbl_autotune may change
 * the last two.  No GPU work. */
int lbl_stream_collide_shape(const lbl_ctx* ctx, int* columns_per_thread, int* prefetch, int* strip_rows);

/* Set that shape, e.g. one an earlier lbl_autotune logged: prefetch 0 or 1 (0 only for
 * the vector-load kernel), strip_rows in [1, ny], or 0 for the heuristic's.  Waits for
 * the context's work and drops its captured graphs; results do not depend on the
 * shape (every shape computes each cell in the same arithmetic). */
int lbl_set_stream_collide_shape(lbl_ctx* ctx, int prefetch, int strip_rows);

/* ---- y-slab split of one experiment over ranks --------------------------------------
 * Replaces the reference's member-sharded MPI layout, whose analysis transposes the ensemble
 * all-to-all every cycle (util/letkf_solver.h:135-215, 374-394; letkf.cu:191, 273, 315).
 * Every rank holds all M members of the rows [row0, row0 + own) of a grid of ny_global
 * rows, plus `halo` rows on each side: create the context with cfg.ny = own + 2 * halo
 * (the rest of cfg as for the whole grid), then call lbl_slab_set before lbl_init.  The
 * constants (dx = h_ref / (ny_global - 1), the forcing's coordinates) and the initial
 * condition then are the whole grid's, and local row r is global row
 * (row0 - halo + r) mod ny_global.  Every kernel runs over the slab as if it were periodic;
 * after k steps the outer 2k rows on each side are stale and the neighbours' packed rows
 * replace them:
 *   - step at most halo / 2 steps (lbl_slab_forecast_chunk, or lbl_update_async), then
 *     exchange 2k rows;
 *   - after lbl_assimilate_async exchange all `halo` rows (the analysis of the halo rows
 *     reads past the slab).
 * The observation fields given to lbl_assimilate are the slab's own nx * cfg.ny rows,
 * halos included.  Own rows then equal the whole-grid run bit for bit.  Conditions:
 * halo >= 2 and own >= halo; DA_LETKF also needs halo >= the window reach
 * (2 * LETKF_RLOC_LEN * DA_XYPRUNE rows, 2 * DA_XYPRUNE without LETKF_RLOC_LEN), and
 * halo and row0 multiples of lcm(8, DA_XYPRUNE).  Modes NATURE and DA_LETKF; no learned
 * closure, matrix dumps, files (output, lbl_assimilate_files), cycle graph
 * (lbl_cycle_async), diagnostics or batch.  lbl_rmse_uv covers the own rows; its truth
 * fields are the slab's nx * cfg.ny values. */
int lbl_slab_set(lbl_ctx* ctx, int ny_global, int row0, int halo);

/* A band's forecast in chunks, with the halo exchange between them.  lbl_slab_forecast_begin
 * computes the forcing of the next nsteps steps in one launch (nsteps in
 * [1, lbl_slab_forecast_steps], the steps the forcing buffer holds: every band of an experiment
 * must begin the same nsteps, so take the smallest over the bands).  Each
 * lbl_slab_forecast_chunk then advances k of those steps (k in [1, halo / 2]), on the
 * context's stream; rho, u, v are written on the last two steps of the begun forecast only, as
 * one lbl_update call writes them.  After each chunk the caller exchanges 2k rows.  Until the
 * last chunk, lbl_update and lbl_assimilate return LBL_ERR_STATE.  Replaces a loop of
 * lbl_update_async calls of k steps, which computes the forcing and writes the macros per call. */
int lbl_slab_forecast_steps(const lbl_ctx* ctx, int* max_steps);
int lbl_slab_forecast_begin(lbl_ctx* ctx, int t0, int nsteps);
int lbl_slab_forecast_chunk(lbl_ctx* ctx, int k);

/* Bytes of one packed halo buffer of `rows` rows: M * 9 * rows * nx elements of the
 * storage type (4 bytes, or 2 with LBL_STORAGE_F16).  No GPU work. */
int lbl_slab_halo_bytes(const lbl_ctx* ctx, int rows, size_t* bytes);

/* Pack, on the context's stream (lbl_get_stream), the rows the neighbours need after the
 * last call: to_prev (for the slab above, rows [row0 - rows, ...)) gets local rows
 * [2 halo - rows, 2 halo), to_next (for the slab below) local rows
 * [cfg.ny - 2 halo, cfg.ny - 2 halo + rows); both [member][q][rows][nx].  rows in
 * [1, halo]; device buffers of lbl_slab_halo_bytes, 16-byte aligned.  The transfer is
 * the caller's (NCCL send / receive, or a copy between contexts on one GPU). */
int lbl_slab_pack(lbl_ctx* ctx, int rows, void* to_prev, void* to_next);

/* Unpack, on the context's stream, the neighbours' packed rows: from_prev (the slab
 * above's to_next) into local rows [0, rows), from_next (the slab below's to_prev) into
 * [cfg.ny - rows, cfg.ny).  A single slab (ny_global = own) is its own neighbour. */
int lbl_slab_unpack(lbl_ctx* ctx, int rows, const void* from_prev, const void* from_next);

/* Directory prefix (config::prefix, "io" by default, config.h:287) under which the
 * LETKF matrix dumps go when cfg.write_mat is set: <prefix>/letkf/mat/ens<r>/
 * <label>.float_<rows>_<cols>_<batch>.<t>.h5 (letkf.cu:276-306, cu_matrix.hpp:97-117),
 * r = the reference rank whose batch is rows [r*ny/M, (r+1)*ny/M), labels _dYf _dyo
 * _Q _V _Xf _dXf _Pa _dWa _Xa _Wa _AI _Z _Lambda _Wma.  lbl_assimilate_files sets
 * it to its io_prefix. */
int lbl_set_io_prefix(lbl_ctx* ctx, const char* io_prefix);

/* The HDF5 writer of the matrix dumps, without libhdf5: one file with one contiguous
 * dataset "data" of dims {d0, d1, d2} (C order over data), float32 or float64
 * (is_double), like H5Fcreate + H5LTmake_dataset (cu_matrix.hpp:108-117). */
int lbl_h5_write_dataset(const char* path, uint64_t d0, uint64_t d1, uint64_t d2, const void* data, int is_double);

/* Learned eddy-viscosity closure.  No counterpart in the reference, whose closure is
 * the fixed Smagorinsky constant (lbm.cu:42-60).  A 6 -> 32 -> 32 -> 1 MLP (GELU,
 * softplus output) maps six invariants of the resolved velocity gradient to a
 * multiplier m >= 0 of the Smagorinsky viscosity, nu_t = m (cs dx)^2 |S|; m = 1 is
 * plain Smagorinsky.  Parameters: LBL_CLOSURE_PARAMS floats, laid out W1[32][6],
 * b1[32], W2[32][32], b2[32], W3[32], b3; they are used as BF16 with FP32 sums.
 * Features (LBL_CLOSURE_FEATURES per cell), with k = dx^2 / nu_ref:
 * log1p(k|S|), log1p(k|W|), (W:W - S:S)/(W:W + S:S), (S11 + S22)/sqrt(S:S),
 * dx/dx_ref, asinh(k omega). */
#define LBL_CLOSURE_PARAMS 1313
#define LBL_CLOSURE_FEATURES 6

/* Switch the context's stream-collide to the closure (params != NULL) or back to
 * plain Smagorinsky (params == NULL).  nu_ref, dx_ref: the feature scales of the
 * training (<= 0: this context's nu and h_ref/255).  Needs the direct-load
 * stream-collide (lbm_variant AUTO or DIRECT).  Switching drops a strip height that
 * lbl_autotune chose and returns to the heuristic's for the kernel now in use. */
int lbl_set_closure(lbl_ctx* ctx, const float* params, double nu_ref, double dx_ref);

/* Evaluate the closure's network every `steps` stream-collide steps (1, the default:
 * every step).  The network runs on steps 0, steps, 2 steps, ... of every forecast
 * chunk and stores each cell's multiplier m; the steps between keep m and apply it to
 * the current |S| (nu_t = m (cs dx)^2 |S|), at the cost of the plain stream-collide.
 * Needs nx <= 1024 for steps > 1.  No counterpart in the reference. */
int lbl_set_closure_refresh(lbl_ctx* ctx, int steps);

/* Training data from the code's own runs: a run of the fine configuration (mode set
 * to NATURE; every member a seeded random-phase IC) is spun up for `spinup` steps,
 * then every `spacing` steps, n_snapshots times, each member's (u, v, uu, uv, vv) is
 * box-filtered over filter x filter cells onto the coarse grid nx/filter.  Each
 * coarse cell gives one sample: the features of the filtered velocity gradient
 * (central differences, dx = h_ref/(ny/filter - 1), nu_ref = the fine run's nu,
 * dx_ref = h_ref/255) and the target multiplier that makes the Smagorinsky stress
 * match the filtered subgrid stress tau_d in the mean-square sense on that cell,
 * m* = -(tau_d : S) / (2 S:S (cs dx)^2 |S|), clipped to [0, 8].  features
 * [n][6], targets [n]; capacity >= n_ens * n_snapshots * (nx/filter)(ny/filter). */
int lbl_closure_generate(const lbl_config* fine, int filter, int spinup, int n_snapshots, int spacing, int device,
                         float* features, float* targets, size_t capacity, size_t* n_samples, char* err,
                         size_t err_cap);

/* Mean-square loss of the closure over n samples and its gradient with respect to
 * the FP32 parameters (one fused forward/backward launch on the GPU). */
int lbl_closure_grad(const float* params, const float* features, const float* targets, size_t n, int device,
                     float* grad, float* loss);

/* Adam training on the GPU: iters steps of `batch` samples drawn with replacement
 * (seeded), learning rate lr, betas 0.9/0.999.  init (optional) starts from given
 * parameters, else a seeded Xavier start with m = 1 everywhere.  params receives the
 * FP32 result; loss_curve (optional, iters floats) the minibatch losses. */
int lbl_closure_train(const float* features, const float* targets, size_t n, int iters, int batch, float lr,
                      uint64_t seed, int device, const float* init, float* params, float* loss_curve);

/* The closure's multiplier for n feature rows: path 0 = the tensor-core form used
 * inside the stream-collide, path 1 = the per-thread FP32 form. */
int lbl_closure_infer(const float* params, const float* features, size_t n, int path, int device, float* out);

/* Batches: several contexts (independent experiments of any grid and ensemble size)
 * cycled together.  No counterpart in the reference, which runs one experiment per
 * MPI job.  Each batch cycle is one CUDA graph: every context's analysis (when its
 * DA gate is due) and forcing chunk on parallel branches, then n_fc steps of all
 * the experiments, each step one launch of a persistent kernel whose CTAs take
 * (experiment, member, strip, 128-column chunk) items from a counter, tallest
 * strips first.  The populations match the contexts' own lbl_cycle_async bit for
 * bit.  The contexts must be initialised, on one device, with FP32 storage, the
 * direct stream-collide, no closure and nx % 128 == 0; strip_rows <= 0 takes 16.
 * While a batch is in use, its contexts take no other cycle or update calls and
 * must outlive it (destroy the batch first); accessors (lbl_get_f, lbl_rmse_uv, ...)
 * wait for the batch's last graph.
 * Observation arrays are per context in the order given to lbl_batch_create (NULL
 * array or entry: reuse that context's resident observations).  n_fc is at most
 * the smallest forcing buffer of the batch. */
typedef struct lbl_batch lbl_batch;
int lbl_batch_create(lbl_ctx* const* ctxs, int n, int strip_rows, lbl_batch** out);
const char* lbl_batch_last_error(const lbl_batch* b);  /* never NULL */
int lbl_batch_cycle_async(lbl_batch* b, int t, const float* const* rho_o, const float* const* u_o,
                          const float* const* v_o, int n_fc);
int lbl_batch_sync(lbl_batch* b);
int lbl_batch_destroy(lbl_batch* b);

/* Evaluation measures over the files lbl_output writes (host only; no context, no
 * GPU).  err (optional) receives a message of at most err_cap bytes.
 *
 * lbl_bindiff: RMSE of u and v together between dir0/<var>_step%010d.dat and dir1's
 * (bindiff/main.cpp:27-69): sqrt(sum (a-b)^2 / count), differences in float, sums
 * in long double; *count = values compared. */
int lbl_bindiff(const char* dir0, const char* dir1, int step, double* rmse, long long* count, char* err,
                size_t err_cap);
/* lbl_ensemble_stat: ensemble_stat/main.cpp:33-170 with the grid size taken from the
 * files: per-cell member mean and standard deviation (long double, kept as float) of
 * ens_dir/ens%04d, then against nature_dir/ens0000: out[0] spread and out[1] RMSE of
 * (u, v) together, out[2] rho spread, out[3] rho RMSE, out[4] max of the mean (u, v). */
int lbl_ensemble_stat(const char* nature_dir, const char* ens_dir, int n_ens, int step, double* out, char* err,
                      size_t err_cap);
/* lbl_energy_spectrum: postprocess/fourier.ipynb cell 2 for one (u, v) [ny][nx]:
 * F = DFT/(nx*ny); over the non-negative wavenumbers i, j <= nx/2, shell
 * k = int(sqrt(i^2 + j^2) + 0.5) <= nx/2 accumulates |(Fu^2 + Fv^2)/2| (complex
 * squares, as the notebook).  ek receives nx/2 + 1 values (FP64). */
int lbl_energy_spectrum(const float* u, const float* v, int nx, int ny, double* ek);

/* Timers: writes the "#tag,sec" CSV (util/timer.hpp:66-72) into buf.
 * Returns the number of bytes needed (excluding NUL) or a negative status. */
int lbl_timer_csv(lbl_ctx* ctx, int which, char* buf, size_t cap);
int lbl_timer_clear(lbl_ctx* ctx, int which);
/* Host-side tag timer driven by the caller (main.cu's util::timer). */
int lbl_timer_transit(lbl_ctx* ctx, int which, const char* tag);

#ifdef __cplusplus
}
#endif
#endif /* LBL_H_ */
