// lbl_api.cu -- the C ABI of liblbl (include/lbl.h): context, initial condition,
// forcing scheduler, forecast graphs, LETKF analysis, output and accessors.
//
// Host arithmetic that the reference performs on the CPU in FP32 (initial
// condition rescale and feq, data.cu:113-141) is done here in FP32 on the host in
// the same order, so the initial populations are bit-identical to the reference's.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <random>
#include <string>
#include <vector>

#include <cudaTypedefs.h>

#include "lbl_internal.h"

using namespace lbl;

namespace {

int wait_output(lbl_ctx* ctx);

// a chunked forecast (lbl_slab_forecast_begin) owns the forcing buffer until its last chunk
constexpr const char* kSlabBegun = "a chunked forecast (lbl_slab_forecast_begin) has steps left";

// what a y-slab context (lbl_slab_set) does not do
constexpr const char* kSlabCycle =
    "a y-slab exchanges halos between its steps: lbl_update_async, lbl_assimilate_async and lbl_slab_pack / "
    "lbl_slab_unpack replace the cycle graph";
constexpr const char* kSlabWhole = "a y-slab reads and writes no files and has no whole-grid diagnostics";

// a failed allocation is LBL_ERR_NOMEM; it is not sticky, so the runtime's last-error
// slot is cleared for the calls that follow
#define LBL_CK(call)                                                                            \
    do {                                                                                        \
        cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess) {                                                                \
            ctx->err = std::string(#call) + ": " + cudaGetErrorString(e_);                      \
            if (e_ == cudaErrorMemoryAllocation) {                                              \
                cudaGetLastError();                                                             \
                return LBL_ERR_NOMEM;                                                           \
            }                                                                                   \
            return LBL_ERR_CUDA;                                                                \
        }                                                                                       \
    } while (0)

#define LBL_CKR(call)                                                                           \
    do {                                                                                        \
        curandStatus_t e_ = (call);                                                             \
        if (e_ != CURAND_STATUS_SUCCESS) {                                                      \
            ctx->err = std::string(#call) + ": curand status " + std::to_string(int(e_));        \
            return LBL_ERR_CURAND;                                                              \
        }                                                                                       \
    } while (0)

#define LBL_TRY(expr)                     \
    do {                                  \
        int rc_ = (expr);                 \
        if (rc_ != LBL_OK) return rc_;    \
    } while (0)

constexpr int ex_h(int q) { return (q % 3) - 1; }
constexpr int ey_h(int q) { return (q / 3) - 1; }
constexpr float wq_h(int q) {
    return (ex_h(q) * ex_h(q) + ey_h(q) * ey_h(q)) == 0   ? float(4. / 9.)
           : (ex_h(q) * ex_h(q) + ey_h(q) * ey_h(q)) == 1 ? float(1. / 9.)
                                                           : float(1. / 36.);
}

// feq evaluated on the host in FP32 (lbm.h:31-39), as init_lbm does (data.cu:131-139)
inline float feq_host(float rho, float u, float v, int q, float c) {
    const float uc0 = (u * ex_h(q) + v * ey_h(q)) / c;
    const float uu0 = (u * u + v * v) / (c * c);
    return rho * wq_h(q) * (float(1.) + float(3.) * uc0 + float(4.5) * uc0 * uc0 - float(1.5) * uu0);
}

double gaspari_cohn(double d) {  // letkf.cu:104-109
    if (d <= 0) return 1.0;
    if (d <= 1) return -d * d * d * d * d / 4. + d * d * d * d / 2. + d * d * d * 5. / 8. - d * d * 5. / 3. + 1;
    if (d <= 2) return d * d * d * d * d / 12. - d * d * d * d / 2. + d * d * d * 5. / 8. + d * d * 5. / 3. - d * 5 + 4 - 2. / 3. / d;
    return 0.0;
}

int fail(lbl_ctx* ctx, int code, const std::string& msg) {
    if (ctx) ctx->err = msg;
    return code;
}

int set_device(lbl_ctx* ctx) {
    LBL_CK(cudaSetDevice(ctx->device));
    return LBL_OK;
}

// ---------------------------------------------------------------------------
// configuration
// ---------------------------------------------------------------------------
// The physical constants come from the grid of ny_global rows (dx = h_ref / (ny_global - 1), the forcing's
// 1/ny); the array shape from cfg.ny.  The two differ only for a y-slab, whose cfg.ny is its own rows plus halos.
Phys derive_phys(const lbl_config& cfg, int ny_global = 0, int row0_local = 0) {
    const int nyg = ny_global > 0 ? ny_global : cfg.ny;
    Phys P{};
    P.nx = cfg.nx; P.ny = cfg.ny; P.M = cfg.n_ens; P.nxy = cfg.nx * cfg.ny;
    P.y0g = row0_local; P.nyg = nyg;
    // the reference's constexpr `real` arithmetic: h_ref is rounded to float first
    // (config.h:158), then divided in float (config.h:250-251)
    P.c = float(cfg.u_ref) / float(cfg.cfl);                       // config.h:248 (constexpr real)
    P.dx = float(cfg.h_ref) / float(nyg - 1);                      // config.h:250
    P.dt = P.dx / P.c;                                             // config.h:251
    double nu = cfg.nu;
    if (cfg.tau > 0) nu = (cfg.tau - 0.5) * double(P.c) * double(P.c) * double(P.dt) / 3.0;
    P.nu = float(nu);
    P.cs2 = P.c * P.c / 3;                                         // lbm.h:50
    P.fr_dt = float(cfg.friction_rate) / P.dt;                     // lbm.h:52 (constexpr real)
    P.u_ref = float(cfg.u_ref);
    P.two_dx = 2 * P.dx;
    P.les_k = cfg.cs * cfg.cs * double(P.dx) * double(P.dx);       // lbm.cu:59-60 (double cs)
    P.c_d = P.c; P.dt_d = P.dt;
    P.tau_k = 3.0 / P.c_d / P.c_d / P.dt_d;
    P.inv_nx = 1.0f / float(cfg.nx);
    P.inv_ny = 1.0f / float(nyg);
    P.inv_c = 1.0f / P.c;
    P.inv_c2 = 1.0f / (P.c * P.c);
    P.inv_cs2 = 1.0f / P.cs2;
    P.inv_two_dx = 1.0f / P.two_dx;
    return P;
}

Geo derive_geo(const lbl_config& cfg) {
    Geo G{};
    G.p = cfg.da_xyprune;
    if (cfg.letkf_rloc_len <= 0) {                                 // letkf.cu:45-49
        G.dloc = G.p - 1;
        G.nl = G.p == 1 ? 0 : 2;
        G.off = G.p == 1 ? 0 : 1;
        G.nox = G.p == 1 ? 1 : 4;
    } else {                                                       // letkf.cu:50-55
        G.dloc = double(cfg.letkf_rloc_len) * G.p;
        G.off = 0;
        G.nl = cfg.letkf_rloc_len * 2;
        G.nox = G.nl * 2 + 1;
    }
    G.nobs = G.nox * G.nox * 3;                                    // letkf.cu:56
    G.nsx = cfg.nx / G.p;
    G.nsy = cfg.ny / G.p;
    return G;
}

int validate(const lbl_config& c, std::string& err) {
    if (c.abi_version != LBL_ABI_VERSION) { err = "abi_version mismatch"; return LBL_ERR_ARG; }
    if (c.mode < LBL_MODE_NATURE || c.mode > LBL_MODE_DA_NUDGING) { err = "unknown mode"; return LBL_ERR_ARG; }
    if (c.da_dummy != 0 && c.mode != LBL_MODE_DA_LETKF && c.mode != LBL_MODE_DA_NUDGING) {
        err = "da_dummy needs DA_LETKF or DA_NUDGING (config.h:38-41)"; return LBL_ERR_ARG;
    }
    if (c.da_quadra < 0 || c.da_quadra > 3) { err = "DA_QUADRA out of range [0, 3]"; return LBL_ERR_ARG; }
    if (c.mode == LBL_MODE_DA_NUDGING && !(c.da_nud_rate >= 0 && c.da_nud_rate <= 1)) {
        err = "DA_NUD_RATE must lie in [0, 1]"; return LBL_ERR_ARG;
    }
    if (c.reserved1 != 0) { err = "reserved fields must be 0"; return LBL_ERR_ARG; }
    if (c.gram != LBL_GRAM_F32 && c.gram != LBL_GRAM_BF16 && c.gram != LBL_GRAM_TF32X3) {
        err = "unknown gram"; return LBL_ERR_ARG;
    }
    if (c.gram == LBL_GRAM_TF32X3) {
        const Geo g = derive_geo(c);
        if (c.mode != LBL_MODE_DA_LETKF || !gram_tc_supported(c.n_ens, g.p, g.nobs)) {
            err = "the tensor-core Gram (LBL_GRAM_TF32X3) needs DA_LETKF, n_ens <= 64 and DA_XYPRUNE^2 a multiple of "
                  "128/MP points (MP = n_ens padded to 16, 32 or 64), e.g. DA_XYPRUNE = 4";
            return LBL_ERR_UNSUPPORTED;
        }
    }
    if (c.gram == LBL_GRAM_BF16 && (c.mode != LBL_MODE_DA_LETKF || c.n_ens <= 32 || c.write_mat)) {
        err = "the BF16 tensor-core Gram serves the wide analysis (DA_LETKF, 32 < n_ens <= 64, no matrix dumps)";
        return LBL_ERR_UNSUPPORTED;
    }
    if (c.storage != LBL_STORAGE_F32 && c.storage != LBL_STORAGE_F16) { err = "unknown storage"; return LBL_ERR_ARG; }
    if (c.storage == LBL_STORAGE_F16 && c.lbm_variant == LBL_LBM_TMA) {
        err = "the TMA stream-collide reads FP32 populations only"; return LBL_ERR_UNSUPPORTED;
    }
    if (c.nx < 32 || c.ny < 8 || c.nx % 32 != 0 || cluster_chunks(c.nx) == 0) {
        err = "nx must be a multiple of 32 up to 1024, or a multiple of 256 up to 8192 with nx/256 <= 8, "
              "nx/512 <= 8 or nx/1024 <= 8 (rows split over a cluster), and ny >= 8";
        return LBL_ERR_ARG;
    }
    if (c.nx > 1024 && c.mode != LBL_MODE_NATURE && c.mode != LBL_MODE_OBSERVE) {
        err = "grids wider than 1024 run NATURE and OBSERVE in this build"; return LBL_ERR_UNSUPPORTED;
    }
    if (c.n_ens < 1) { err = "n_ens must be >= 1"; return LBL_ERR_ARG; }
    if (c.iiter < 1 || c.ioprune < 1 || c.daprune < 1) { err = "iiter/ioprune/daprune must be >= 1"; return LBL_ERR_ARG; }
    if (c.da_xyprune < 1 || c.nx % c.da_xyprune != 0 || c.ny % c.da_xyprune != 0) {
        err = "DA_XYPRUNE must divide nx and ny (letkf.cu:30 static_assert)"; return LBL_ERR_ARG;
    }
    if (c.letkf_rloc_len < 0 || c.letkf_rloc_len > 8) { err = "LETKF_RLOC_LEN out of range [0, 8]"; return LBL_ERR_ARG; }
    if (!(c.letkf_covinf > 0)) { err = "LETKF_COVINF must be > 0"; return LBL_ERR_ARG; }
    if (!(c.obs_error_rho > 0) || !(c.obs_error_u > 0)) { err = "OBS_ERROR_RHO/OBS_ERROR_U must be > 0"; return LBL_ERR_ARG; }
    if (!(c.cfl > 0) || !(c.u_ref > 0) || !(c.h_ref > 0)) { err = "cfl, u_ref, h_ref must be > 0"; return LBL_ERR_ARG; }
    if (c.tau != 0 && !(c.tau > 0.5)) { err = "tau must be > 0.5 (or 0 to use nu)"; return LBL_ERR_ARG; }
    if (c.jacobi_max_sweeps < 1 || c.jacobi_max_sweeps > 1000) { err = "jacobi_max_sweeps out of range"; return LBL_ERR_ARG; }
    if (c.write_mat != 0 && c.mode != LBL_MODE_DA_LETKF) { err = "write_mat needs DA_LETKF"; return LBL_ERR_ARG; }
    if (c.write_mat != 0 && c.n_ens > kMaxMemberLanes) {
        err = "write_mat supports n_ens <= 32 in this build"; return LBL_ERR_UNSUPPORTED;
    }
    if (c.write_mat != 0 && c.ny % c.n_ens != 0) {  // letkf.cu:34-35, 74: whole rows per rank
        err = "write_mat needs ny divisible by n_ens (the reference's batch per rank is whole rows)";
        return LBL_ERR_ARG;
    }
    if (c.lbm_variant < LBL_LBM_AUTO || c.lbm_variant > LBL_LBM_VEC2) { err = "unknown lbm_variant"; return LBL_ERR_ARG; }
    if ((c.lbm_variant == LBL_LBM_VEC || c.lbm_variant == LBL_LBM_VEC2) && c.nx > 1024) {
        err = "the vector-load stream-collide serves nx <= 1024"; return LBL_ERR_UNSUPPORTED;
    }
    if (c.mode == LBL_MODE_DA_LETKF && !analysis_supported(c.n_ens)) {
        err = "DA_LETKF supports 2 <= n_ens <= 64 in this build"; return LBL_ERR_UNSUPPORTED;
    }
    if (c.mode == LBL_MODE_DA_LETKF && analysis_smem_bytes(c.n_ens, derive_geo(c).nobs) > kAnalysisSmemLimit) {
        err = "observation window too large for the analysis kernel's shared memory (reduce LETKF_RLOC_LEN)";
        return LBL_ERR_UNSUPPORTED;
    }
    return LBL_OK;
}

// ---------------------------------------------------------------------------
// forcing: the reference's cursor over a buffer of 4096*n normals refilled by
// curandGenerateNormal (data.cu:240-247).  Returns the pool offset of the 4*n
// normals of this call.
// ---------------------------------------------------------------------------
int force_call(lbl_ctx* ctx, int* offset) {
    const int n4 = 4 * ctx->n_modes;
    ctx->i_rand_outdated += n4;
    if (ctx->i_rand_outdated + n4 >= ctx->n_rand_buf) {
        ctx->rand_block++;
        const int slot = int(ctx->rand_block % ctx->pool_slots);
        LBL_CKR(curandGenerateNormal(ctx->gen, ctx->d_pool + size_t(slot) * ctx->n_rand_buf, ctx->n_rand_buf,
                                     0.0f, 0.84089641525f));
        ctx->i_rand_outdated = 0;
    }
    *offset = int(ctx->rand_block % ctx->pool_slots) * ctx->n_rand_buf + ctx->i_rand_outdated;
    ctx->last_sched = *offset;
    return LBL_OK;
}

// compact the observations at the sites into [u, v, rho][site] (letkf.cu:230-269 gather)
void compact_obs(const lbl_ctx* ctx, const float* ro, const float* uo, const float* vo, float* dst) {
    const int ns = ctx->G.nsx * ctx->G.nsy, p = ctx->G.p, nx = ctx->P.nx;
    for (int sj = 0; sj < ctx->G.nsy; sj++)
        for (int si = 0; si < ctx->G.nsx; si++) {
            const int s = si + ctx->G.nsx * sj;
            const size_t ij = size_t(si) * p + size_t(nx) * sj * p;
            dst[s] = uo[ij];
            dst[ns + s] = vo[ij];
            dst[2 * ns + s] = ro[ij];
        }
}

// schedule the forcing of `n` consecutive calls and upload the offsets through
// one of two pinned staging buffers (an event guards each buffer's reuse), on `st`
// (the context's stream by default)
int schedule_force(lbl_ctx* ctx, int n, cudaStream_t st = nullptr) {
    if (!st) st = ctx->stream;
    const int b = ctx->sched_buf;
    ctx->sched_buf ^= 1;
    LBL_CK(cudaEventSynchronize(ctx->ev[4 + b]));
    int* h = ctx->h_sched[b];
    for (int s = 0; s < n; s++) LBL_TRY(force_call(ctx, &h[s]));
    LBL_CK(cudaMemcpyAsync(ctx->d_sched, h, sizeof(int) * n, cudaMemcpyHostToDevice, st));
    LBL_CK(cudaEventRecord(ctx->ev[4 + b], st));
    return LBL_OK;
}

// stage the site observations through one of two pinned buffers and upload them
int upload_obs(lbl_ctx* ctx, const float* ro, const float* uo, const float* vo) {
    const int b = ctx->yo_buf;
    ctx->yo_buf ^= 1;
    LBL_CK(cudaEventSynchronize(ctx->ev[6 + b]));
    compact_obs(ctx, ro, uo, vo, ctx->h_yo[b]);
    const size_t ns = size_t(ctx->G.nsx) * ctx->G.nsy;
    LBL_CK(cudaMemcpyAsync(ctx->d_yo, ctx->h_yo[b], sizeof(float) * 3 * ns, cudaMemcpyHostToDevice, ctx->stream));
    LBL_CK(cudaEventRecord(ctx->ev[6 + b], ctx->stream));
    ctx->have_obs = true;
    return LBL_OK;
}

// enqueue: forcing chunk + n LBM steps starting from buffer `cur`; macros are
// written on the last two steps (the only ones output/lbm2euler can observe).
void enqueue_steps(lbl_ctx* ctx, int n, int cur, cudaStream_t s, bool force_done = false) {
    if (!force_done) launch_force_chunk(ctx, n, 0, s);
    for (int k = 0; k < n; k++) {
        const int src = (cur + k) & 1, dst = src ^ 1;
        const bool mac = k >= n - 2;
        launch_lbm_step(ctx, src, dst, ctx->d_force + size_t(k) * 2 * ctx->P.nxy,
                        mac ? ctx->mac[dst] : nullptr, s, /*pdl=*/k > 0, k);
    }
}

// The FP32 populations the LETKF reads (forecast) and writes (analysis) for buffer cur:
// the buffers themselves, or, with FP16 storage, FP32 copies expanded before and
// compressed after the analysis.
const float* analysis_input(lbl_ctx* ctx, int cur, cudaStream_t s) {
    if (!ctx->f16) return ctx->f[cur];
    launch_expand(ctx, ctx->h[cur], ctx->fs[0], s);
    return ctx->fs[0];
}
float* analysis_output(lbl_ctx* ctx, int cur) { return ctx->f16 ? ctx->fs[1] : ctx->f[cur ^ 1]; }
void analysis_commit(lbl_ctx* ctx, int cur, cudaStream_t s) {
    if (ctx->f16) launch_compress(ctx, ctx->fs[1], ctx->h[cur ^ 1], s);
}

// enqueue the assimilation of the resident observations into buffer `cur`; returns the
// buffer that holds the result (the LETKF writes the other buffer, nudging works in place)
int enqueue_analysis(lbl_ctx* ctx, int cur, cudaStream_t s) {
    if (ctx->cfg.mode == LBL_MODE_DA_NUDGING) {
        launch_nudging(ctx, cur, ctx->mac[cur], s);
        return cur;
    }
    cudaMemsetAsync(ctx->d_stats, 0, sizeof(int) * 4, s);
    const float* fin = analysis_input(ctx, cur, s);
    launch_obs_ensemble(ctx, fin, s);
    launch_analysis(ctx, fin, analysis_output(ctx, cur), ctx->mac[cur ^ 1], s);
    analysis_commit(ctx, cur, s);
    return cur ^ 1;
}

// Build (once) and launch a graph.  kind: 0 = steps, 1 = cycle (analysis + steps).
int launch_graph(lbl_ctx* ctx, int kind, int n) {
    const long long key = ((long long)kind << 40) | ((long long)n << 1) | ctx->cur;
    auto it = ctx->graphs.find(key);
    if (it == ctx->graphs.end()) {
        cudaGraph_t g = nullptr;
        LBL_CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
        int cur = ctx->cur;
        // phase events become event-record nodes of the graph (device timestamps of each launch)
        cudaEventRecordWithFlags(ctx->ev[10], ctx->stream, cudaEventRecordExternal);
        if (kind == 1 && n > 0) {
            // the forcing of the coming steps does not depend on the flow: compute it
            // on a side branch while the analysis runs (different pipes: XU/FP64 vs FMA/SHFL)
            cudaEventRecord(ctx->fork_ev, ctx->stream);
            cudaStreamWaitEvent(ctx->side, ctx->fork_ev, 0);
            launch_force_chunk(ctx, n, 0, ctx->side);
            cudaEventRecord(ctx->join_ev, ctx->side);
            cudaStreamWaitEvent(ctx->hi, ctx->fork_ev, 0);
            cur = enqueue_analysis(ctx, cur, ctx->hi);
            cudaEventRecord(ctx->hi_ev, ctx->hi);
            cudaStreamWaitEvent(ctx->stream, ctx->hi_ev, 0);
            cudaStreamWaitEvent(ctx->stream, ctx->join_ev, 0);
            cudaEventRecordWithFlags(ctx->ev[11], ctx->stream, cudaEventRecordExternal);
            enqueue_steps(ctx, n, cur, ctx->stream, true);
        } else {
            if (kind == 1) cur = enqueue_analysis(ctx, cur, ctx->stream);
            cudaEventRecordWithFlags(ctx->ev[11], ctx->stream, cudaEventRecordExternal);
            if (n > 0) enqueue_steps(ctx, n, cur, ctx->stream);
        }
        cudaEventRecordWithFlags(ctx->ev[12], ctx->stream, cudaEventRecordExternal);
        const cudaError_t le = cudaGetLastError();
        const cudaError_t ee = cudaStreamEndCapture(ctx->stream, &g);
        if (le != cudaSuccess || ee != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            return fail(ctx, LBL_ERR_CUDA, std::string("graph capture failed: ") +
                                               cudaGetErrorString(le != cudaSuccess ? le : ee));
        }
        cudaGraphExec_t ge;
        const cudaError_t ie = cudaGraphInstantiate(&ge, g, cudaGraphInstantiateFlagUseNodePriority);
        cudaGraphDestroy(g);
        if (ie != cudaSuccess) return fail(ctx, LBL_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ie));
        it = ctx->graphs.emplace(key, ge).first;
    }
    LBL_CK(cudaGraphLaunch(it->second, ctx->stream));
    ctx->phases = kind == 1 ? 2 : 1;
    return LBL_OK;
}

int check_timeout(lbl_ctx* ctx) {
    int h = 0;
    LBL_CK(cudaMemcpy(&h, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (h) {
        cudaMemset(ctx->d_err, 0, sizeof(int));
        return fail(ctx, LBL_ERR_TIMEOUT, std::string(h == 4 ? "tensor-core Gram: the MMA completion wait"
                                                               : "stream-collide: a bounded shared-memory pipeline wait") +
                                              " gave up (code " + std::to_string(h) + ")");
    }
    return LBL_OK;
}

int read_stats(lbl_ctx* ctx) {
    LBL_CK(cudaMemcpy(ctx->h_stats, ctx->d_stats, sizeof(int) * 3, cudaMemcpyDeviceToHost));
    if (ctx->h_stats[2]) return fail(ctx, LBL_ERR_NAN, "NaN in the LETKF analysis (letkf_solver.h:352-364 sanity)");
    return LBL_OK;
}

bool da_due(const lbl_ctx* ctx, int t) { return ((t / ctx->cfg.iiter) % ctx->cfg.daprune) == 0; }

// the reference's DATA_ASSIMILATION run modes (config.h:32-53)
bool is_da_mode(int mode) { return mode == LBL_MODE_DA_LETKF || mode == LBL_MODE_DA_NUDGING; }

// initial velocity of one ensemble id on the device, rescaled on the host (FP32).  A y-slab
// computes and rescales the whole grid's field, then keeps its own rows and halos.
int ic_member(lbl_ctx* ctx, int seed, std::vector<float>& u, std::vector<float>& v) {
    const lbl_config& cfg = ctx->cfg;
    const int nx = cfg.nx, ny = ctx->slab_ny ? ctx->slab_ny : cfg.ny, nk = nx / 2;
    std::mt19937 eng(seed);                                      // data.cu:43-45
    std::uniform_real_distribution<float> dist(-1, 1);
    std::vector<double> kx, ky, pp, th;
    const float k0 = float(cfg.kf);
    for (int kj = 0; kj < nk; kj++)
        for (int ki = 0; ki < nk; ki++) {
            const float k = std::sqrt(float(ki * ki + kj * kj));
            float pk;
            if (cfg.ic_kind == LBL_IC_REFERENCE) {
                const float dk = 10, sigma = 5;
                pk = (k0 - dk <= k && k <= k0 + dk) ? std::exp(-(k - k0) * (k - k0) / sigma) : 0.f;
            } else {
                const float s = k / k0;
                pk = (k > 0 && s * s <= 23.0f) ? std::sqrt(k) * std::exp(-s * s) : 0.f;
            }
            const float theta = float(dist(eng) * M_PI);
            if (pk != 0.f) {
                kx.push_back(2 * M_PI * ki / nx);
                ky.push_back(2 * M_PI * kj / ny);
                pp.push_back(pk);
                th.push_back(theta);
            }
        }
    const int n = int(kx.size());
    std::vector<double> tab;
    tab.insert(tab.end(), kx.begin(), kx.end());
    tab.insert(tab.end(), ky.begin(), ky.end());
    tab.insert(tab.end(), pp.begin(), pp.end());
    tab.insert(tab.end(), th.begin(), th.end());
    double* d_tab = nullptr;
    float* d_uv = nullptr;
    const size_t nxy = size_t(nx) * ny;
    LBL_CK(cudaMalloc(&d_tab, sizeof(double) * std::max<size_t>(tab.size(), 1)));
    LBL_CK(cudaMalloc(&d_uv, sizeof(float) * 2 * nxy));
    LBL_CK(cudaMemcpy(d_tab, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice));
    launch_ic_velocity(d_tab, n, nx, ny, d_uv, d_uv + nxy, ctx->stream);
    LBL_CK(cudaGetLastError());
    u.resize(nxy); v.resize(nxy);
    LBL_CK(cudaMemcpyAsync(u.data(), d_uv, sizeof(float) * nxy, cudaMemcpyDeviceToHost, ctx->stream));
    LBL_CK(cudaMemcpyAsync(v.data(), d_uv + nxy, sizeof(float) * nxy, cudaMemcpyDeviceToHost, ctx->stream));
    LBL_CK(cudaStreamSynchronize(ctx->stream));
    cudaFree(d_tab);
    cudaFree(d_uv);
    if (cfg.ic_kind == LBL_IC_REFERENCE) {                       // data.cu:113-120
        float vmax = float(1e-30 * cfg.u_ref);
        for (size_t ij = 0; ij < nxy; ij++) vmax = std::max(vmax, std::sqrt(u[ij] * u[ij] + v[ij] * v[ij]));
        const float s = float(cfg.u_ref) / vmax * float(cfg.ic_amp);
        for (size_t ij = 0; ij < nxy; ij++) { u[ij] *= s; v[ij] *= s; }
    } else {
        double e = 0;
        for (size_t ij = 0; ij < nxy; ij++) e += double(u[ij]) * u[ij] + double(v[ij]) * v[ij];
        const float s = float(cfg.ic_amp / std::sqrt(e / double(nxy) + 1e-300));
        for (size_t ij = 0; ij < nxy; ij++) { u[ij] *= s; v[ij] *= s; }
    }
    if (ctx->slab_ny) {
        std::vector<float> us(size_t(ctx->P.nxy)), vs(size_t(ctx->P.nxy));
        for (int j = 0; j < ctx->P.ny; j++) {
            const size_t g = size_t((j + ctx->P.y0g) % ny) * nx, l = size_t(j) * nx;
            std::copy(u.begin() + g, u.begin() + g + nx, us.begin() + l);
            std::copy(v.begin() + g, v.begin() + g + nx, vs.begin() + l);
        }
        u.swap(us);
        v.swap(vs);
    }
    return LBL_OK;
}

int build_weight_table(lbl_ctx* ctx) {
    const Geo& G = ctx->G;
    const lbl_config& cfg = ctx->cfg;
    const int np = G.p * G.p;
    std::vector<int> tab(size_t(4) * np * G.nobs + np, 0);
    int* cnt = tab.data() + size_t(4) * np * G.nobs;
    for (int pj = 0; pj < G.p; pj++)
        for (int pi = 0; pi < G.p; pi++) {
            const int pat = pi + G.p * pj;
            int n = 0;
            for (int b = 0; b < G.nox; b++)
                for (int a = 0; a < G.nox; a++) {
                    const int da = a - (G.nl - G.off), db = b - (G.nl - G.off);
                    const int di = pi - da * G.p, dj = pj - db * G.p;   // i - io, j - jo
                    (void)da; (void)db;
                    const bool valid = !(std::abs(di) > G.nl * G.p || std::abs(dj) > G.nl * G.p);
                    if (!valid) continue;
                    double gc = 1.0;
                    if (G.p > 1) gc = gaspari_cohn(std::sqrt(double(di * di + dj * dj)) / (G.dloc + 1e-6));
                    for (int var = 0; var < 3; var++) {
                        const double sig = var == 2 ? cfg.obs_error_rho : cfg.obs_error_u;
                        const float w = float(gc / (sig * sig));
                        if (!(w > 0.f)) continue;
                        int* e = tab.data() + (size_t(pat) * G.nobs + n) * 4;
                        e[0] = a + G.nox * b + var * G.nox * G.nox;  // window slot (letkf.cu:155, 183-185)
                        e[1] = var;
                        const float sw = std::sqrt(w);  // correctly rounded, as the device's sqrtf
                        std::memcpy(&e[2], &sw, sizeof(float));
                        std::memcpy(&e[3], &w, sizeof(float));
                        n++;
                    }
                }
            cnt[pat] = n;
        }
    LBL_CK(cudaMalloc(&ctx->d_wtab, sizeof(int) * tab.size()));
    LBL_CK(cudaMemcpy(ctx->d_wtab, tab.data(), sizeof(int) * tab.size(), cudaMemcpyHostToDevice));
    if (cfg.gram == LBL_GRAM_TF32X3) {  // the same weights, dense per pattern, for the tensor-core Gram
        const int kpad = (G.nobs + 7) & ~7;
        std::vector<float> dense(size_t(np) * kpad, 0.f);
        for (int pat = 0; pat < np; pat++)
            for (int n = 0; n < cnt[pat]; n++) {
                const int* e = tab.data() + (size_t(pat) * G.nobs + n) * 4;
                std::memcpy(&dense[size_t(pat) * kpad + e[0]], &e[3], sizeof(float));
            }
        LBL_CK(cudaMalloc(&ctx->d_wdense, sizeof(float) * dense.size()));
        LBL_CK(cudaMemcpy(ctx->d_wdense, dense.data(), sizeof(float) * dense.size(), cudaMemcpyHostToDevice));
        const int mpq = gram_tc_mp(ctx->P.M);
        LBL_CK(cudaMalloc(&ctx->d_Q, sizeof(float) * size_t(ctx->P.nxy) * (size_t(mpq) * mpq + mpq)));
        if (gram_tc_prepare() != 0) return fail(ctx, LBL_ERR_CUDA, "cudaFuncSetAttribute(gram_tc_kernel) failed");
    }
    return LBL_OK;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no libcuda link)
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

// 3-D map over one population buffer: x (nx), y (ny), plane (member*9 + q); box = one
// row segment of up to 256 floats
bool make_population_map(const lbl_ctx* ctx, float* base, CUtensorMap* map) {
    auto enc = tensor_map_encoder();
    if (!enc) return false;
    const cuuint64_t dims[3] = {cuuint64_t(ctx->P.nx), cuuint64_t(ctx->P.ny), cuuint64_t(ctx->P.M) * kQ};
    const cuuint64_t strides[2] = {cuuint64_t(ctx->P.nx) * sizeof(float), cuuint64_t(ctx->P.nxy) * sizeof(float)};
    const cuuint32_t box[3] = {cuuint32_t(ctx->P.nx < 256 ? ctx->P.nx : 256), 1, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    return enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, base, dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

int create_impl(const lbl_config* cfg, int device, lbl_ctx* ctx) {
    ctx->cfg = *cfg;
    ctx->device = device;
    LBL_TRY(validate(*cfg, ctx->err));
    ctx->P = derive_phys(*cfg);
    ctx->G = derive_geo(*cfg);
    LBL_TRY(set_device(ctx));
    // The engine's and the side stream at the default priority; the cycle graph's analysis
    // branch is captured on a stream at the device's highest priority and keeps it (node
    // priorities), so the forcing beside it fills the SMs the analysis leaves idle instead of
    // competing with it.  Only the analysis is raised: steps and forcing of contexts that
    // share the GPU keep competing on equal terms.
    int prio_low = 0, prio_high = 0;
    LBL_CK(cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high));
    LBL_CK(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    LBL_CK(cudaStreamCreateWithFlags(&ctx->side, cudaStreamNonBlocking));
    LBL_CK(cudaStreamCreateWithPriority(&ctx->hi, cudaStreamNonBlocking, prio_high));
    LBL_CK(cudaEventCreateWithFlags(&ctx->fork_ev, cudaEventDisableTiming));
    LBL_CK(cudaEventCreateWithFlags(&ctx->join_ev, cudaEventDisableTiming));
    LBL_CK(cudaEventCreateWithFlags(&ctx->hi_ev, cudaEventDisableTiming));
    const size_t nxy = size_t(ctx->P.nxy), M = size_t(ctx->P.M);
    ctx->f16 = cfg->storage == LBL_STORAGE_F16;
    for (int b = 0; b < 2; b++) {
        if (ctx->f16) {
            LBL_CK(cudaMalloc(&ctx->h[b], sizeof(__half) * M * kQ * nxy));
            if (cfg->mode == LBL_MODE_DA_LETKF) LBL_CK(cudaMalloc(&ctx->fs[b], sizeof(float) * M * kQ * nxy));
        } else {
            LBL_CK(cudaMalloc(&ctx->f[b], sizeof(float) * M * kQ * nxy));
        }
        LBL_CK(cudaMalloc(&ctx->mac[b], sizeof(float) * M * 3 * nxy));
        LBL_CK(cudaMemset(ctx->mac[b], 0, sizeof(float) * M * 3 * nxy));
    }
    // forcing mode table (data.cu:161-237), amplitudes normalised in long double
    {
        const float kf = float(cfg->kf), sigma = 1, dk = 2;
        const int kmax = int(kf + dk);
        long double asum = 0;
        int n = 0;
        for (int y = 0; y < kmax; y++)
            for (int x = 0; x < kmax; x++) {
                if (x == 0 && y == 0) continue;
                const double k = std::sqrt(double(y * y + x * x));
                if (kf - dk <= k && k <= kf + dk) {
                    if (n >= kMaxModes) return fail(ctx, LBL_ERR_UNSUPPORTED, "too many forcing modes");
                    const float a = float(std::exp(-(k - kf) * (k - kf) / sigma));
                    asum += a;
                    ctx->h_kx[n] = float(x); ctx->h_ky[n] = float(y); ctx->h_amp[n] = a;
                    n++;
                }
            }
        if (n == 0) return fail(ctx, LBL_ERR_ARG, "forcing wavenumber band is empty");
        const float total = float(cfg->fkf * cfg->u_ref / 1.0);
        for (int i = 0; i < n; i++) ctx->h_amp[i] = float(ctx->h_amp[i] * (total / asum));
        ctx->n_modes = n;
        std::vector<float> tab(2 * n);
        std::vector<double> amps(2 * n);
        for (int i = 0; i < n; i++) {
            tab[i] = ctx->h_kx[i];
            tab[n + i] = ctx->h_ky[i];
            // amp*2*M_PI*ky, amp*2*M_PI*(-kx) of data.cu:342-343, evaluated left to right in FP64
            amps[i] = double(ctx->h_amp[i] * 2) * M_PI * double(ctx->h_ky[i]);
            amps[n + i] = double(ctx->h_amp[i] * 2) * M_PI * double(-ctx->h_kx[i]);
        }
        LBL_CK(cudaMalloc(&ctx->d_modes, sizeof(float) * 2 * n));
        LBL_CK(cudaMemcpy(ctx->d_modes, tab.data(), sizeof(float) * 2 * n, cudaMemcpyHostToDevice));
        LBL_CK(cudaMalloc(&ctx->d_amps, sizeof(double) * 2 * n));
        LBL_CK(cudaMemcpy(ctx->d_amps, amps.data(), sizeof(double) * 2 * n, cudaMemcpyHostToDevice));
        std::copy(amps.begin(), amps.end(), ctx->h_amps);
        ctx->n_rand_buf = n * 4096;                                        // data.cu:297
        LBL_CK(cudaMalloc(&ctx->d_pool, sizeof(float) * ctx->pool_slots * size_t(ctx->n_rand_buf)));
    }
    // steps of forcing one graph can hold: 256 MB of fields (512 steps at 256^2, 128 at 512^2)
    ctx->force_cap = int(std::max<long long>(8, std::min<long long>(1023, (256ll << 20) / (8ll * nxy))));
    LBL_CK(cudaMalloc(&ctx->d_force, sizeof(float) * 2 * nxy * ctx->force_cap));
    LBL_CK(cudaMemset(ctx->d_force, 0, sizeof(float) * 2 * nxy * ctx->force_cap));
    LBL_CK(cudaMalloc(&ctx->d_sched, sizeof(int) * ctx->force_cap));
    for (int b = 0; b < 2; b++) LBL_CK(cudaMallocHost(&ctx->h_sched[b], sizeof(int) * ctx->force_cap));
    LBL_CKR(curandCreateGenerator(&ctx->gen, CURAND_RNG_PSEUDO_MTGP32));   // data.cu:293-294
    LBL_CKR(curandSetPseudoRandomGeneratorSeed(ctx->gen, cfg->force_seed));
    LBL_CKR(curandSetStream(ctx->gen, ctx->stream));
    // observation sites (both DA modes) and LETKF buffers
    if (cfg->mode == LBL_MODE_DA_LETKF || cfg->mode == LBL_MODE_DA_NUDGING) {
        const size_t ns = size_t(ctx->G.nsx) * ctx->G.nsy;
        LBL_CK(cudaMalloc(&ctx->d_yo, sizeof(float) * 3 * ns));
        for (int b = 0; b < 2; b++) LBL_CK(cudaMallocHost(&ctx->h_yo[b], sizeof(float) * 3 * ns));
    }
    if (cfg->mode == LBL_MODE_DA_LETKF) {
        const size_t ns = size_t(ctx->G.nsx) * ctx->G.nsy;
        LBL_TRY(build_weight_table(ctx));
        LBL_CK(cudaMalloc(&ctx->d_dY, sizeof(float) * 3 * ns * M));
        LBL_CK(cudaMalloc(&ctx->d_dyo, sizeof(float) * 3 * ns));
    }
    LBL_CK(cudaMalloc(&ctx->d_stats, sizeof(int) * 4));
    LBL_CK(cudaMemset(ctx->d_stats, 0, sizeof(int) * 4));  // max sweeps, non-converged, NaN, sweep total
    LBL_CK(cudaMalloc(&ctx->d_red, sizeof(double) * 8));
    LBL_CK(cudaMalloc(&ctx->d_tmp, sizeof(float) * 2 * nxy));
    LBL_CK(cudaMalloc(&ctx->d_err, sizeof(int)));
    LBL_CK(cudaMemset(ctx->d_err, 0, sizeof(int)));
    if (cfg->lbm_variant == LBL_LBM_TMA && !ctx->f16 && lbm_tma_supported(cfg->nx)) {
        ctx->use_tma = make_population_map(ctx, ctx->f[0], &ctx->tmap[0]) &&
                       make_population_map(ctx, ctx->f[1], &ctx->tmap[1]) && lbm_tma_prepare(cfg->nx) == 0;
    }
    if (cfg->lbm_variant == LBL_LBM_TMA && !ctx->use_tma)
        return fail(ctx, LBL_ERR_UNSUPPORTED, "TMA stream-collide unavailable for this grid (nx <= 512) or driver");
    if (cfg->lbm_variant == LBL_LBM_VEC) ctx->vec = 4;
    if (cfg->lbm_variant == LBL_LBM_VEC2) ctx->vec = 2;
    // measured on B200 (back-to-back launches): the 2-column march gains from the
    // prefetched row up to 256 columns, the 4-column one (215 against 168 registers)
    // loses; FP16 deviations pay only with vector loads (512^2 x 64: 164 against
    // 218 us), FP32 at 512^2 x 64 stays fastest one column per thread (215 against
    // 228 us), and at 256^2 x 16 two columns gain (12.9 against 14.4 us).  On a grid that
    // is not square (a y-slab's band) the prefetching 2-column march holds 128 registers
    // against 94 without prefetch, and loses: 256 x 272 x 16, 16.4 against 14.5 us
    ctx->vec_auto = cfg->lbm_variant == LBL_LBM_AUTO && cfg->nx <= 1024;
    if (ctx->vec_auto) ctx->vec = (ctx->f16 || cfg->nx <= 256) ? 2 : 0;
    ctx->vec_pf = ctx->vec == 2 ? cfg->nx <= 256 && cfg->nx == cfg->ny
                                : ctx->vec == 0;  // (the one-column kernels always prefetch)
    ctx->ty_default = lbm_strip_rows(ctx);
    for (auto& e : ctx->ev) LBL_CK(cudaEventCreate(&e));
    for (auto& e : ctx->user_ev) LBL_CK(cudaEventCreate(&e));
    ctx->have_events = true;
    if (analysis_prepare() != 0) return fail(ctx, LBL_ERR_CUDA, "cudaFuncSetAttribute(analysis_kernel) failed");
    ctx->timers[LBL_TIMER_MAIN].t0 = wall_time();
    ctx->timers[LBL_TIMER_LETKF].t0 = wall_time();
    return LBL_OK;
}

void destroy_impl(lbl_ctx* ctx) {
    cudaSetDevice(ctx->device);
    if (ctx->out_thread.joinable()) ctx->out_thread.join();
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (auto& g : ctx->graphs) cudaGraphExecDestroy(g.second);
    ctx->graphs.clear();
    if (ctx->gen) curandDestroyGenerator(ctx->gen);
    for (int b = 0; b < 2; b++) {
        cudaFree(ctx->f[b]); cudaFree(ctx->h[b]); cudaFree(ctx->fs[b]); cudaFree(ctx->mac[b]);
    }
    cudaFree(ctx->d_modes); cudaFree(ctx->d_amps); cudaFree(ctx->d_pool); cudaFree(ctx->d_force); cudaFree(ctx->d_sched);
    cudaFree(ctx->d_wtab); cudaFree(ctx->d_yo); cudaFree(ctx->d_dY); cudaFree(ctx->d_dyo);
    cudaFree(ctx->d_wdense); cudaFree(ctx->d_Q);
    cudaFree(ctx->d_stats); cudaFree(ctx->d_red); cudaFree(ctx->d_tmp); cudaFree(ctx->d_err); cudaFree(ctx->d_dump);
    cudaFree(ctx->d_closure);
    cudaFree(ctx->d_mclos);
    for (int b = 0; b < 2; b++) {
        if (ctx->h_yo[b]) cudaFreeHost(ctx->h_yo[b]);
        if (ctx->h_sched[b]) cudaFreeHost(ctx->h_sched[b]);
    }
    if (ctx->have_events) {
        for (auto& e : ctx->ev) cudaEventDestroy(e);
        for (auto& e : ctx->user_ev) cudaEventDestroy(e);
    }
    if (ctx->obs_engine) obs_engine_free(ctx->obs_engine);
    cudaFree(ctx->d_outf);
    if (ctx->h_outf) cudaFreeHost(ctx->h_outf);
    if (ctx->out_ev) cudaEventDestroy(ctx->out_ev);
    if (ctx->fork_ev) cudaEventDestroy(ctx->fork_ev);
    if (ctx->join_ev) cudaEventDestroy(ctx->join_ev);
    if (ctx->hi_ev) cudaEventDestroy(ctx->hi_ev);
    if (ctx->hi) cudaStreamDestroy(ctx->hi);
    if (ctx->side) cudaStreamDestroy(ctx->side);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
}

// one member's FP32 populations [9][ny][nx] to/from buffer b, converting for FP16 storage
int upload_member(lbl_ctx* ctx, int b, int m, const float* f) {
    const size_t n = size_t(kQ) * ctx->P.nxy;
    if (!ctx->f16) {
        LBL_CK(cudaMemcpy(ctx->f[b] + size_t(m) * n, f, sizeof(float) * n, cudaMemcpyHostToDevice));
        return LBL_OK;
    }
    std::vector<__half> h(n);
    for (size_t e = 0; e < n; e++) h[e] = __float2half_rn(f[e] - wq_h(int(e / ctx->P.nxy)));
    LBL_CK(cudaMemcpy(ctx->h[b] + size_t(m) * n, h.data(), sizeof(__half) * n, cudaMemcpyHostToDevice));
    return LBL_OK;
}

int download_member(lbl_ctx* ctx, int b, int m, float* f) {
    const size_t n = size_t(kQ) * ctx->P.nxy;
    if (!ctx->f16) {
        LBL_CK(cudaMemcpy(f, ctx->f[b] + size_t(m) * n, sizeof(float) * n, cudaMemcpyDeviceToHost));
        return LBL_OK;
    }
    std::vector<__half> h(n);
    LBL_CK(cudaMemcpy(h.data(), ctx->h[b] + size_t(m) * n, sizeof(__half) * n, cudaMemcpyDeviceToHost));
    for (size_t e = 0; e < n; e++) f[e] = wq_h(int(e / ctx->P.nxy)) + __half2float(h[e]);
    return LBL_OK;
}

int init_impl(lbl_ctx* ctx, int ens_offset) {
    const lbl_config& cfg = ctx->cfg;
    const size_t nxy = size_t(ctx->P.nxy);
    const int M = ctx->P.M;
    ctx->ens_offset = ens_offset;
    ctx->cur = 0;
    const int add = is_da_mode(cfg.mode) ? 334 : 0;                // data.cu:31-35 (DATA_ASSIMILATION)
    std::vector<float> un, vn;
    if (cfg.ens_init == LBL_ENS_PERTURBED) LBL_TRY(ic_member(ctx, ens_offset, un, vn));
    std::vector<float> fh(kQ * nxy), mh(3 * nxy);
    const float r0 = float(cfg.rho_ref);
    for (int m = 0; m < M; m++) {
        std::vector<float> u, v;
        LBL_TRY(ic_member(ctx, m + ens_offset + add, u, v));
        if (cfg.ens_init == LBL_ENS_PERTURBED) {
            const float a = float(cfg.ens_perturb);
            for (size_t ij = 0; ij < nxy; ij++) { u[ij] = un[ij] + a * u[ij]; v[ij] = vn[ij] + a * v[ij]; }
        }
        for (size_t ij = 0; ij < nxy; ij++) {
            for (int q = 0; q < kQ; q++) fh[q * nxy + ij] = feq_host(r0, u[ij], v[ij], q, ctx->P.c);
            mh[ij] = r0; mh[nxy + ij] = u[ij]; mh[2 * nxy + ij] = v[ij];
        }
        for (int b = 0; b < 2; b++) {  // data_0_ and data_1_ both start from the IC (data.h:55)
            LBL_TRY(upload_member(ctx, b, m, fh.data()));
            LBL_CK(cudaMemcpy(ctx->mac[b] + size_t(m) * 3 * nxy, mh.data(), sizeof(float) * 3 * nxy,
                              cudaMemcpyHostToDevice));
        }
    }
    // forcing: cursor starts "outdated", two update_forces calls at init (data.cu:236, :158)
    ctx->fc_free_recorded = false;
    ctx->i_rand_outdated = ctx->n_rand_buf;
    ctx->rand_block = -1;
    LBL_TRY(schedule_force(ctx, 2));
    launch_force_chunk(ctx, 2, 0, ctx->stream);
    LBL_CK(cudaGetLastError());
    ctx->last_force_slot = 1;
    LBL_CK(cudaStreamSynchronize(ctx->stream));
    ctx->initialised = true;
    return LBL_OK;
}

int update_impl(lbl_ctx* ctx, int nsteps, bool sync) {
    if (!ctx->initialised) return fail(ctx, LBL_ERR_STATE, "lbl_update before lbl_init");
    if (ctx->fc_off < ctx->fc_total) return fail(ctx, LBL_ERR_STATE, kSlabBegun);
    if (nsteps < 0) return fail(ctx, LBL_ERR_ARG, "nsteps < 0");
    ctx->fc_free_recorded = false;  // these steps read the forcing slots on the context's stream
    int left = nsteps;
    while (left > 0) {
        // each chunk writes macros on its last two steps, so whatever the chunking,
        // the last two steps of the call leave rho,u,v in both buffers
        const int n = std::min(left, ctx->force_cap);
        LBL_TRY(schedule_force(ctx, n));
        LBL_TRY(launch_graph(ctx, 0, n));
        ctx->cur ^= (n & 1);
        ctx->last_force_slot = n - 1;
        left -= n;
    }
    if (sync) {
        LBL_CK(cudaStreamSynchronize(ctx->stream));
        LBL_TRY(check_timeout(ctx));
    }
    return LBL_OK;
}

// need_save_mat (letkf.cu:33, 276-306; letkf_solver.h:243-345): the matrices of every
// point, written per reference rank r (the rows [r*ny/M, (r+1)*ny/M)) to
// <prefix>/letkf/mat/ens<r>/<label>.float_<rows>_<cols>_<batch>.<t>.h5 (cu_matrix.hpp:97-117).
// fin is the forecast the analysis started from.
int dump_matrices(lbl_ctx* ctx, int t, const float* fin) {
    const int M = ctx->P.M, ny = ctx->P.ny, rows = ny / M, nobs = ctx->G.nobs;
    const size_t nb = size_t(rows) * ctx->P.nx;
    size_t sz[kDumpCount], total = 0;
    dump_sizes(M, nobs, nb, sz);
    for (size_t z : sz) total += z;
    if (!ctx->d_dump) LBL_CK(cudaMalloc(&ctx->d_dump, sizeof(float) * total));
    ctx->h_dump.resize(total);
    const uint64_t shape[kDumpCount][2] = {{uint64_t(nobs), uint64_t(M)}, {uint64_t(nobs), 1}, {uint64_t(M), uint64_t(M)},
                                           {uint64_t(M), uint64_t(M)}, {kQ, uint64_t(M)}, {kQ, uint64_t(M)},
                                           {uint64_t(M), uint64_t(M)}, {uint64_t(M), uint64_t(M)}, {kQ, uint64_t(M)},
                                           {uint64_t(M), uint64_t(M)}, {kQ, uint64_t(M)}, {uint64_t(M), uint64_t(M)},
                                           {uint64_t(M), uint64_t(M)}, {uint64_t(M), uint64_t(M)}};
    for (int r = 0; r < M; r++) {
        launch_analysis_dump(ctx, fin, ctx->d_dump, r * rows, (r + 1) * rows, ctx->stream);
        LBL_CK(cudaGetLastError());
        LBL_CK(cudaMemcpyAsync(ctx->h_dump.data(), ctx->d_dump, sizeof(float) * total, cudaMemcpyDeviceToHost,
                               ctx->stream));
        LBL_CK(cudaStreamSynchronize(ctx->stream));
        const std::string dir = ctx->io_prefix + "/letkf/mat/ens" + std::to_string(r);
        if (mkdir_p(dir) != 0) return fail(ctx, LBL_ERR_IO, "could not create " + dir);
        const float* p = ctx->h_dump.data();
        for (int i = 0; i < kDumpCount; i++) {
            const uint64_t dims[3] = {shape[i][0], shape[i][1], uint64_t(nb)};
            const std::string name = dir + "/" + kDumpLabels[i] + ".float_" + std::to_string(dims[0]) + "_" +
                                     std::to_string(dims[1]) + "_" + std::to_string(nb) + "." + std::to_string(t) +
                                     ".h5";
            std::string e;
            if (write_h5_dataset(name, dims, p, false, e) != LBL_OK) return fail(ctx, LBL_ERR_IO, e);
            p += sz[i];
        }
    }
    return LBL_OK;
}

// DA_NUDGING (nudging.cu:40-143): every member's f relaxes toward feq of the observed
// (bilinearly interpolated) rho, u, v, in place; the macros are not refreshed.
int nudging_impl(lbl_ctx* ctx, int t, const float* ro, const float* uo, const float* vo, bool sync) {
    if (!da_due(ctx, t)) return LBL_OK;                             // nudging.cu:43-44
    if (!ro || !uo || !vo) return fail(ctx, LBL_ERR_ARG, "null observation pointer");
    LBL_TRY(upload_obs(ctx, ro, uo, vo));
    launch_nudging(ctx, ctx->cur, ctx->mac[ctx->cur], ctx->stream);
    LBL_CK(cudaGetLastError());
    if (sync) LBL_CK(cudaStreamSynchronize(ctx->stream));
    return LBL_OK;
}

int assimilate_impl(lbl_ctx* ctx, int t, const float* ro, const float* uo, const float* vo, bool sync) {
    if (!ctx->initialised) return fail(ctx, LBL_ERR_STATE, "lbl_assimilate before lbl_init");
    if (!is_da_mode(ctx->cfg.mode)) return fail(ctx, LBL_ERR_STATE, "lbl_assimilate needs mode DA_LETKF or DA_NUDGING");
    if (ctx->fc_off < ctx->fc_total) return fail(ctx, LBL_ERR_STATE, kSlabBegun);
    if (ctx->cfg.da_dummy) return LBL_OK;                           // DA_DUMMY: no assimilation (main.cu:94)
    if (ctx->cfg.mode == LBL_MODE_DA_NUDGING) return nudging_impl(ctx, t, ro, uo, vo, sync);
    TimerMap& tm = ctx->timers[LBL_TIMER_LETKF];
    timer_transit(tm, "_ignored");                                  // letkf.cu:121
    if (!da_due(ctx, t)) return LBL_OK;                             // letkf.cu:122-123
    if (!ro || !uo || !vo) return fail(ctx, LBL_ERR_ARG, "null observation pointer");
    LBL_CK(cudaMemsetAsync(ctx->d_stats, 0, sizeof(int) * 4, ctx->stream));
    const double h0 = wall_time();
    LBL_CK(cudaEventRecord(ctx->ev[0], ctx->stream));
    LBL_TRY(upload_obs(ctx, ro, uo, vo));
    const double h1 = wall_time();
    LBL_CK(cudaEventRecord(ctx->ev[1], ctx->stream));
    const float* fin = analysis_input(ctx, ctx->cur, ctx->stream);
    launch_obs_ensemble(ctx, fin, ctx->stream);
    LBL_CK(cudaEventRecord(ctx->ev[2], ctx->stream));
    launch_analysis(ctx, fin, analysis_output(ctx, ctx->cur), ctx->mac[ctx->cur ^ 1], ctx->stream);
    analysis_commit(ctx, ctx->cur, ctx->stream);
    LBL_CK(cudaGetLastError());
    LBL_CK(cudaEventRecord(ctx->ev[3], ctx->stream));
    if (ctx->cfg.write_mat) {
        const double d0 = wall_time();
        LBL_TRY(dump_matrices(ctx, t, fin));
        timer_add(tm, "solve", wall_time() - d0);                   // the dumps sit in solve_evd/solve_xa
    }
    ctx->cur ^= 1;                                                   // dat.swap(), letkf.cu:357
    if (sync) {
        LBL_CK(cudaEventSynchronize(ctx->ev[3]));
        // stage tags of letkf.cu:133-336.  The member transposes and MPI exchanges of
        // the reference are index maps inside the kernels here, and update_xk /
        // lbm2euler are fused into the analysis kernel, so those tags stay at 0.
        float ms_h2d = 0, ms_obs = 0, ms_ana = 0;
        cudaEventElapsedTime(&ms_h2d, ctx->ev[0], ctx->ev[1]);
        cudaEventElapsedTime(&ms_obs, ctx->ev[1], ctx->ev[2]);
        cudaEventElapsedTime(&ms_ana, ctx->ev[2], ctx->ev[3]);
        timer_add(tm, "load_obs", (h1 - h0) + 1e-3 * ms_h2d);
        timer_add(tm, "pack_yk", 1e-3 * ms_obs);
        timer_add(tm, "solve", 1e-3 * ms_ana);
        for (const char* tag : {"pack_xk", "mpi_yk", "set_yo", "mpi_xk", "solve_comm_ovlp", "mpi_barrier",
                                "mpi_xsol", "update_xk", "lbm2euler"})
            timer_add(tm, tag, 0.0);
        timer_transit(tm, "_ignored");
        LBL_TRY(read_stats(ctx));
    }
    return LBL_OK;
}

// The files of one output (io.cu:22-266) from the staged copy: macros mh [M][3][nxy],
// vorticity vor [M][nxy], statistics st [4][nxy], NaN flag.  Runs on the writer thread;
// touches only the staging, the OBSERVE engine and h_obs, which no other call uses
// while an output is pending.
int write_output_files(lbl_ctx* ctx, int t, const std::string& pre, std::string& err) {
    const lbl_config& cfg = ctx->cfg;
    const int nx = cfg.nx, ny = cfg.ny, M = cfg.n_ens;
    const size_t nxy = size_t(nx) * ny;
    const float* mh = ctx->h_outf;
    const float* vor = mh + size_t(M) * 3 * nxy;
    const float* st = vor + size_t(M) * nxy;
    int nan_flag = 0;
    std::memcpy(&nan_flag, st + 4 * nxy, sizeof(int));
    if (nan_flag) { err = "nan value detected"; return LBL_ERR_NAN; }  // io.cu:79-83
    const std::string step = "_step" + to_string_aligned(t / cfg.iiter, 10) + ".dat";
    auto dname = [&](const std::string& kind, int id) { return pre + "/" + kind + "/ens" + to_string_aligned(id, 4); };
    auto mkdir = [&](const std::string& d) {
        if (mkdir_p(d) == 0) return LBL_OK;
        err = "could not create " + d;
        return LBL_ERR_IO;
    };
    if (cfg.mode == LBL_MODE_DA_LETKF) {                            // ENSEMBLE_STAT (io.cu:88-139)
        LBL_TRY(mkdir(pre + "/calc"));
        LBL_TRY(write_dat(pre + "/calc/ens_mean_u" + step, st, nxy, err));
        LBL_TRY(write_dat(pre + "/calc/ens_mean_v" + step, st + nxy, nxy, err));
        LBL_TRY(write_dat(pre + "/calc/ens_vor_mean" + step, st + 2 * nxy, nxy, err));
        LBL_TRY(write_dat(pre + "/calc/ens_vor_std" + step, st + 3 * nxy, nxy, err));
    }
    for (int m = 0; m < M; m++) {
        const int id = m + ctx->ens_offset;
        const float* r = mh + (size_t(m) * 3 + 0) * nxy;
        const float* u = mh + (size_t(m) * 3 + 1) * nxy;
        const float* v = mh + (size_t(m) * 3 + 2) * nxy;
        const float* w = vor + size_t(m) * nxy;
        if (cfg.mode != LBL_MODE_OBSERVE) {                          // io.cu:151-157
            const std::string d = dname("calc", id);
            LBL_TRY(mkdir(d));
            LBL_TRY(write_dat(d + "/vor" + step, w, nxy, err));
            LBL_TRY(write_dat(d + "/rho" + step, r, nxy, err));
            LBL_TRY(write_dat(d + "/u" + step, u, nxy, err));
            LBL_TRY(write_dat(d + "/v" + step, v, nxy, err));
        }
        if (cfg.mode == LBL_MODE_OBSERVE && id == 0) {               // io.cu:160-246
            if (!ctx->obs_engine) ctx->obs_engine = obs_engine_new(uint32_t(cfg.obs_seed + id));
            for (auto& a : ctx->h_obs) a.resize(nxy);
            observe_host(ctx->obs_engine, nx, ny, cfg.da_xyprune, float(cfg.obs_error_rho), float(cfg.obs_error_u),
                         r, u, v, ctx->h_obs[0].data(), ctx->h_obs[1].data(), ctx->h_obs[2].data(),
                         ctx->h_obs[3].data(), ctx->P.dx);
            const std::string d = dname("observed", id);
            LBL_TRY(mkdir(d));
            LBL_TRY(write_dat(d + "/rho" + step, ctx->h_obs[0].data(), nxy, err));
            LBL_TRY(write_dat(d + "/u" + step, ctx->h_obs[1].data(), nxy, err));
            LBL_TRY(write_dat(d + "/v" + step, ctx->h_obs[2].data(), nxy, err));
            LBL_TRY(write_dat(d + "/vor" + step, ctx->h_obs[3].data(), nxy, err));
        }
        if ((cfg.mode == LBL_MODE_NATURE || cfg.mode == LBL_MODE_OBSERVE) && id == 0) {  // io.cu:248-258
            const std::string d = dname("nature", id);
            LBL_TRY(mkdir(d));
            LBL_TRY(write_dat(d + "/rho" + step, r, nxy, err));
            LBL_TRY(write_dat(d + "/u" + step, u, nxy, err));
            LBL_TRY(write_dat(d + "/v" + step, v, nxy, err));
            LBL_TRY(write_dat(d + "/vor" + step, w, nxy, err));
        }
    }
    return LBL_OK;
}

// Waits for the writer of the previous output and returns its status.
int wait_output(lbl_ctx* ctx) {
    if (ctx->out_thread.joinable()) ctx->out_thread.join();
    const int rc = ctx->out_rc;
    if (rc != LBL_OK) {
        ctx->err = ctx->out_err;
        ctx->out_rc = LBL_OK;
        ctx->out_err.clear();
    }
    return rc;
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

const char* lbl_version(void) { return "liblbl 0.1 (sm_100a)"; }

const char* lbl_last_error(const lbl_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int lbl_config_default(lbl_config* c, int mode, int nx, int n_ens) {
    if (!c) return LBL_ERR_ARG;
    std::memset(c, 0, sizeof(*c));
    const int scaler = nx / 64;
    c->abi_version = LBL_ABI_VERSION;
    c->mode = mode;
    c->nx = nx; c->ny = nx;                  // config.h:133-134
    c->n_ens = n_ens;
    c->iiter = 5 * (scaler > 0 ? scaler : 1); // config.h:136
    c->ioprune = 10;                         // config.h:91
    c->daprune = 10;                         // config.h:56
    c->da_xyprune = 1;                       // config.h:60
    c->letkf_rloc_len = 0;
    c->iter_main = c->iiter * 2000;          // config.h:144
    c->spinup = 100000 * c->iiter;           // config.h:139
    c->ic_kind = LBL_IC_REFERENCE;
    c->ens_init = LBL_ENS_INDEPENDENT;
    c->compat_stale_v = 1;
    c->jacobi_max_sweeps = 100;
    c->letkf_covinf = 1.0;                   // config.h:49
    c->obs_error_rho = 0.01;                 // run/jserr:146-147
    c->obs_error_u = 0.1;
    c->cs = 0.2;                             // lbm.cu:59
    c->nu = 1e-4;                            // config.h:157
    c->tau = 0;
    c->cfl = 0.05;                           // config.h:153
    c->rho_ref = 1;
    c->u_ref = 1;
    c->h_ref = 2 * M_PI;
    c->kf = 4;                               // config.h:161
    c->fkf = 5.6;                            // config.h:171
    c->friction_rate = 5e-4;                 // config.h:180
    c->ic_amp = 0.01;                        // data.cu:53
    c->ens_perturb = 0.1;
    c->jacobi_tol = 1e-6;                    // cu_matrix_eigensolver_wrapper.hpp:192
    c->force_seed = 1991;                    // data.cu:294
    c->obs_seed = 334;                       // io.cu:321
    c->da_dummy = 0;                         // config.h:71 (commented out)
    c->da_quadra = 0;                        // config.h:63-65
    c->da_obs_ruv = 1;                       // config.h:44 (DA_OBS_RUV)
    c->da_nud_rate = 0.1;                    // config.h:67-69
    return LBL_OK;
}

int lbl_create(const lbl_config* cfg, int device, lbl_ctx** out) {
    if (!cfg || !out) return LBL_ERR_ARG;
    *out = nullptr;
    lbl_ctx* ctx = new (std::nothrow) lbl_ctx();
    if (!ctx) return LBL_ERR_NOMEM;
    const int rc = create_impl(cfg, device, ctx);
    *out = ctx;  // returned even on failure so lbl_last_error can explain; caller destroys
    return rc;
}

int lbl_destroy(lbl_ctx* ctx) {
    if (!ctx) return LBL_OK;
    destroy_impl(ctx);
    delete ctx;
    return LBL_OK;
}

int lbl_init(lbl_ctx* ctx, int ens_offset) {
    if (!ctx) return LBL_ERR_ARG;
    LBL_TRY(set_device(ctx));
    return init_impl(ctx, ens_offset);
}

int lbl_update(lbl_ctx* ctx, int t0, int nsteps) {
    (void)t0;
    if (!ctx) return LBL_ERR_ARG;
    LBL_TRY(set_device(ctx));
    return update_impl(ctx, nsteps, true);
}

int lbl_update_async(lbl_ctx* ctx, int t0, int nsteps) {
    (void)t0;
    if (!ctx) return LBL_ERR_ARG;
    LBL_TRY(set_device(ctx));
    return update_impl(ctx, nsteps, false);
}

int lbl_sync(lbl_ctx* ctx) {
    if (!ctx) return LBL_ERR_ARG;
    LBL_TRY(set_device(ctx));
    LBL_CK(cudaStreamSynchronize(ctx->stream));
    LBL_TRY(wait_output(ctx));
    LBL_TRY(check_timeout(ctx));
    if (ctx->cfg.mode == LBL_MODE_DA_LETKF) LBL_TRY(read_stats(ctx));
    return LBL_OK;
}

int lbl_inject(lbl_ctx* ctx, int what, int value) {
    if (!ctx) return LBL_ERR_ARG;
    if (what != LBL_INJECT_NONE && what != LBL_INJECT_TMA_STALL) return fail(ctx, LBL_ERR_ARG, "unknown injection");
    if (what == LBL_INJECT_TMA_STALL && (value < 1 || value > (1 << 20)))
        return fail(ctx, LBL_ERR_ARG, "LBL_INJECT_TMA_STALL takes a poll limit in [1, 2^20]");
    LBL_TRY(set_device(ctx));
    LBL_CK(cudaStreamSynchronize(ctx->stream));
    LBL_CK(cudaStreamSynchronize(ctx->side));
    // the stream-collide's parameters are baked into the captured graphs
    for (auto& g : ctx->graphs) cudaGraphExecDestroy(g.second);
    ctx->graphs.clear();
    ctx->inject_tma_stall = what == LBL_INJECT_TMA_STALL ? value : 0;
    return LBL_OK;
}

int lbl_assimilate(lbl_ctx* ctx, int t, const float* ro, const float* uo, const float* vo) {
    if (!ctx) return LBL_ERR_ARG;
    LBL_TRY(set_device(ctx));
    return assimilate_impl(ctx, t, ro, uo, vo, true);
}

int lbl_assimilate_async(lbl_ctx* ctx, int t, const float* ro, const float* uo, const float* vo) {
    if (!ctx) return LBL_ERR_ARG;
    LBL_TRY(set_device(ctx));
    return assimilate_impl(ctx, t, ro, uo, vo, false);
}

int lbl_assimilate_files(lbl_ctx* ctx, int t, const char* io_prefix) {
    if (!ctx || !io_prefix) return LBL_ERR_ARG;
    if (ctx->slab_ny) return fail(ctx, LBL_ERR_UNSUPPORTED, kSlabWhole);
    LBL_TRY(wait_output(ctx));  // an OBSERVE output of this context may still be writing the files
    if (!is_da_mode(ctx->cfg.mode)) return fail(ctx, LBL_ERR_STATE, "lbl_assimilate needs mode DA_LETKF or DA_NUDGING");
    if (ctx->cfg.da_dummy) return LBL_OK;                           // DA_DUMMY (main.cu:94)
    if (!da_due(ctx, t)) {
        if (ctx->cfg.mode == LBL_MODE_DA_LETKF) timer_transit(ctx->timers[LBL_TIMER_LETKF], "_ignored");
        return LBL_OK;
    }
    const size_t nxy = size_t(ctx->P.nxy);
    std::vector<float> ro(nxy, 0.f), uo(nxy), vo(nxy);
    const std::string step = to_string_aligned(t / ctx->cfg.iiter, 10);
    const std::string dir = std::string(io_prefix) + "/observed/ens0000/";
    // nudging reads the rho file only under DA_OBS_RUV (nudging.cu:72-80)
    if (ctx->cfg.mode == LBL_MODE_DA_LETKF || ctx->cfg.da_obs_ruv)
        LBL_TRY(read_dat(dir + "rho_step" + step + ".dat", ro.data(), nxy, ctx->err));
    LBL_TRY(read_dat(dir + "u_step" + step + ".dat", uo.data(), nxy, ctx->err));
    LBL_TRY(read_dat(dir + "v_step" + step + ".dat", vo.data(), nxy, ctx->err));
    ctx->io_prefix = io_prefix;                                     // config::prefix for the matrix dumps
    return lbl_assimilate(ctx, t, ro.data(), uo.data(), vo.data());
}

int lbl_cycle_async(lbl_ctx* ctx, int t, const float* ro, const float* uo, const float* vo, int n_fc) {
    if (!ctx) return LBL_ERR_ARG;
    LBL_TRY(set_device(ctx));
    if (!ctx->initialised) return fail(ctx, LBL_ERR_STATE, "lbl_cycle_async before lbl_init");
    if (ctx->slab_ny) return fail(ctx, LBL_ERR_UNSUPPORTED, kSlabCycle);
    if (n_fc < 0) return fail(ctx, LBL_ERR_ARG, "n_fc < 0");
    if (n_fc > ctx->force_cap) {
        // more steps than one graph's forcing buffer: the cycle graph takes the first
        // force_cap steps, forecast graphs the rest
        LBL_TRY(lbl_cycle_async(ctx, t, ro, uo, vo, ctx->force_cap));
        return update_impl(ctx, n_fc - ctx->force_cap, false);
    }
    const bool due = is_da_mode(ctx->cfg.mode) && !ctx->cfg.da_dummy && t > 0 && da_due(ctx, t);
    if (due && ctx->cfg.write_mat) {
        // matrix dumps write files: the analysis runs outside the graph, the forecast in one
        if (!(ro && uo && vo)) return fail(ctx, LBL_ERR_ARG, "write_mat needs the observations in each call");
        LBL_TRY(assimilate_impl(ctx, t, ro, uo, vo, true));
        return lbl_cycle_async(ctx, -1, nullptr, nullptr, nullptr, n_fc);
    }
    // given observations become the resident ones even when this call assimilates
    // nothing; NULL reuses them and needs some to have been given before
    if (ro && uo && vo && is_da_mode(ctx->cfg.mode)) LBL_TRY(upload_obs(ctx, ro, uo, vo));
    if (due && !ctx->have_obs)
        return fail(ctx, LBL_ERR_STATE, "lbl_cycle_async: an analysis is due and no observations were given yet");
    if (n_fc > 0) LBL_TRY(schedule_force(ctx, n_fc));
    LBL_TRY(launch_graph(ctx, due ? 1 : 0, n_fc));
    if (due && ctx->cfg.mode == LBL_MODE_DA_LETKF) ctx->cur ^= 1;
    ctx->cur ^= (n_fc & 1);
    if (n_fc > 0) ctx->last_force_slot = n_fc - 1;
    return LBL_OK;
}

int lbl_output_async(lbl_ctx* ctx, int t, const char* io_prefix) {
    if (!ctx || !io_prefix) return LBL_ERR_ARG;
    LBL_TRY(set_device(ctx));
    if (ctx->slab_ny) return fail(ctx, LBL_ERR_UNSUPPORTED, kSlabWhole);
    const lbl_config& cfg = ctx->cfg;
    if (t % (cfg.iiter * cfg.ioprune) != 0) return LBL_OK;          // io.cu:23
    LBL_TRY(wait_output(ctx));                                       // the staging is free again
    const size_t nxy = size_t(ctx->P.nxy), M = size_t(ctx->P.M);
    const size_t n_dev = (M + 4) * nxy + 4, n_host = 3 * M * nxy + n_dev;
    if (!ctx->d_outf) {
        LBL_CK(cudaMalloc(&ctx->d_outf, sizeof(float) * n_dev));
        LBL_CK(cudaMallocHost(&ctx->h_outf, sizeof(float) * n_host));
        LBL_CK(cudaEventCreateWithFlags(&ctx->out_ev, cudaEventDisableTiming));
    }
    int* d_nan = reinterpret_cast<int*>(ctx->d_outf + (M + 4) * nxy);
    LBL_CK(cudaMemsetAsync(d_nan, 0, sizeof(int), ctx->stream));
    launch_output_fields(ctx, ctx->mac[ctx->cur], ctx->d_outf, ctx->d_outf + M * nxy, d_nan, ctx->stream);
    LBL_CK(cudaGetLastError());
    LBL_CK(cudaMemcpyAsync(ctx->h_outf, ctx->mac[ctx->cur], sizeof(float) * 3 * M * nxy, cudaMemcpyDeviceToHost,
                           ctx->stream));
    LBL_CK(cudaMemcpyAsync(ctx->h_outf + 3 * M * nxy, ctx->d_outf, sizeof(float) * n_dev, cudaMemcpyDeviceToHost,
                           ctx->stream));
    LBL_CK(cudaEventRecord(ctx->out_ev, ctx->stream));
    const std::string pre(io_prefix);
    try {
        ctx->out_thread = std::thread([ctx, t, pre]() {
            std::string err;
            int rc = LBL_OK;
            cudaSetDevice(ctx->device);
            const cudaError_t e = cudaEventSynchronize(ctx->out_ev);
            if (e != cudaSuccess) {
                rc = LBL_ERR_CUDA;
                err = std::string("output staging copy: ") + cudaGetErrorString(e);
            } else {
                rc = write_output_files(ctx, t, pre, err);
            }
            ctx->out_err = err;
            ctx->out_rc = rc;
        });
    } catch (const std::exception& ex) {
        return fail(ctx, LBL_ERR_NOMEM, std::string("could not start the output writer: ") + ex.what());
    }
    return LBL_OK;
}

int lbl_output(lbl_ctx* ctx, int t, const char* io_prefix) {
    LBL_TRY(lbl_output_async(ctx, t, io_prefix));
    return wait_output(ctx);
}

int lbl_get_f(lbl_ctx* ctx, int member, float* f) {
    if (!ctx || !f || member < 0 || member >= ctx->P.M) return LBL_ERR_ARG;
    LBL_TRY(set_device(ctx));
    LBL_CK(cudaStreamSynchronize(ctx->stream));
    return download_member(ctx, ctx->cur, member, f);
}

int lbl_set_f(lbl_ctx* ctx, int member, const float* f) {
    if (!ctx || !f || member < 0 || member >= ctx->P.M) return LBL_ERR_ARG;
    LBL_TRY(set_device(ctx));
    LBL_CK(cudaStreamSynchronize(ctx->stream));
    LBL_TRY(upload_member(ctx, ctx->cur, member, f));
    launch_macros(ctx, ctx->cur, ctx->mac[ctx->cur], ctx->stream);
    LBL_CK(cudaGetLastError());
    LBL_CK(cudaStreamSynchronize(ctx->stream));
    return LBL_OK;
}

int lbl_get_fields(lbl_ctx* ctx, int member, float* rho, float* u, float* v, float* vor) {
    if (!ctx || member < 0 || member >= ctx->P.M) return LBL_ERR_ARG;
    LBL_TRY(set_device(ctx));
    const size_t nxy = size_t(ctx->P.nxy);
    std::vector<float> h(3 * nxy);
    LBL_CK(cudaStreamSynchronize(ctx->stream));
    LBL_CK(cudaMemcpy(h.data(), ctx->mac[ctx->cur] + size_t(member) * 3 * nxy, sizeof(float) * 3 * nxy,
                      cudaMemcpyDeviceToHost));
    if (rho) std::memcpy(rho, h.data(), sizeof(float) * nxy);
    if (u) std::memcpy(u, h.data() + nxy, sizeof(float) * nxy);
    if (v) std::memcpy(v, h.data() + 2 * nxy, sizeof(float) * nxy);
    if (vor) vorticity_host(ctx->P.nx, ctx->P.ny, ctx->P.dx, h.data() + nxy, h.data() + 2 * nxy, vor);
    return LBL_OK;
}

int lbl_get_ens_stats(lbl_ctx* ctx, float* u_mean, float* v_mean, float* vor_mean, float* vor_std) {
    if (!ctx) return LBL_ERR_ARG;
    LBL_TRY(set_device(ctx));
    const int M = ctx->P.M;
    const size_t nxy = size_t(ctx->P.nxy);
    std::vector<float> mh(size_t(M) * 3 * nxy), w(nxy);
    LBL_CK(cudaStreamSynchronize(ctx->stream));
    LBL_CK(cudaMemcpy(mh.data(), ctx->mac[ctx->cur], sizeof(float) * mh.size(), cudaMemcpyDeviceToHost));
    std::vector<float> um(nxy, 0.f), vm(nxy, 0.f), wm(nxy, 0.f), w2(nxy, 0.f);
    const float iv = float(1) / M;
    for (int m = 0; m < M; m++) {
        const float* u = mh.data() + (size_t(m) * 3 + 1) * nxy;
        const float* v = mh.data() + (size_t(m) * 3 + 2) * nxy;
        vorticity_host(ctx->P.nx, ctx->P.ny, ctx->P.dx, u, v, w.data());
        for (size_t ij = 0; ij < nxy; ij++) {
            um[ij] += u[ij]; vm[ij] += v[ij]; wm[ij] += w[ij]; w2[ij] += iv * (w[ij] * w[ij]);
        }
    }
    for (size_t ij = 0; ij < nxy; ij++) {
        um[ij] *= iv; vm[ij] *= iv; wm[ij] *= iv;
        if (u_mean) u_mean[ij] = um[ij];
        if (v_mean) v_mean[ij] = vm[ij];
        if (vor_mean) vor_mean[ij] = wm[ij];
        if (vor_std) vor_std[ij] = std::sqrt(w2[ij] - wm[ij] * wm[ij]);
    }
    return LBL_OK;
}

int lbl_get_force(lbl_ctx* ctx, float* fx, float* fy) {
    if (!ctx) return LBL_ERR_ARG;
    LBL_TRY(set_device(ctx));
    const size_t nxy = size_t(ctx->P.nxy);
    const float* F = ctx->d_force + size_t(ctx->last_force_slot) * 2 * nxy;
    LBL_CK(cudaStreamSynchronize(ctx->stream));
    if (fx) LBL_CK(cudaMemcpy(fx, F, sizeof(float) * nxy, cudaMemcpyDeviceToHost));
    if (fy) LBL_CK(cudaMemcpy(fy, F + nxy, sizeof(float) * nxy, cudaMemcpyDeviceToHost));
    return LBL_OK;
}

int lbl_get_force_state(lbl_ctx* ctx, float* randoms, float* kx, float* ky, float* amp, int* n_modes,
                        int* i_rand_outdated) {
    if (!ctx) return LBL_ERR_ARG;
    LBL_TRY(set_device(ctx));
    const int n = ctx->n_modes;
    LBL_CK(cudaStreamSynchronize(ctx->stream));
    if (randoms)
        LBL_CK(cudaMemcpy(randoms, ctx->d_pool + ctx->last_sched, sizeof(float) * 4 * n, cudaMemcpyDeviceToHost));
    for (int i = 0; i < n; i++) {
        if (kx) kx[i] = ctx->h_kx[i];
        if (ky) ky[i] = ctx->h_ky[i];
        if (amp) amp[i] = ctx->h_amp[i];
    }
    if (n_modes) *n_modes = n;
    if (i_rand_outdated) *i_rand_outdated = ctx->i_rand_outdated;
    return LBL_OK;
}

int lbl_get_observed(lbl_ctx* ctx, float* rho_o, float* u_o, float* v_o, float* vor_o) {
    if (!ctx) return LBL_ERR_ARG;
    LBL_TRY(wait_output(ctx));
    if (ctx->h_obs[0].empty()) return fail(ctx, LBL_ERR_STATE, "no observation generated yet (OBSERVE output)");
    const size_t n = sizeof(float) * ctx->P.nxy;
    if (rho_o) std::memcpy(rho_o, ctx->h_obs[0].data(), n);
    if (u_o) std::memcpy(u_o, ctx->h_obs[1].data(), n);
    if (v_o) std::memcpy(v_o, ctx->h_obs[2].data(), n);
    if (vor_o) std::memcpy(vor_o, ctx->h_obs[3].data(), n);
    return LBL_OK;
}

int lbl_get_letkf_stats(lbl_ctx* ctx, int* max_sweeps, int* n_noconv, int* nan_flag, int* total_sweeps) {
    if (!ctx) return LBL_ERR_ARG;
    LBL_TRY(set_device(ctx));
    LBL_CK(cudaStreamSynchronize(ctx->stream));
    LBL_CK(cudaMemcpy(ctx->h_stats, ctx->d_stats, sizeof(int) * 4, cudaMemcpyDeviceToHost));
    if (max_sweeps) *max_sweeps = ctx->h_stats[0];
    if (n_noconv) *n_noconv = ctx->h_stats[1];
    if (nan_flag) *nan_flag = ctx->h_stats[2];
    if (total_sweeps) *total_sweeps = ctx->h_stats[3];
    return LBL_OK;
}

int lbl_get_diagnostics(lbl_ctx* ctx, int member, double* energy, double* enstrophy, double* mass) {
    if (!ctx || member < -1 || member >= ctx->P.M) return LBL_ERR_ARG;
    LBL_TRY(set_device(ctx));
    if (ctx->slab_ny) return fail(ctx, LBL_ERR_UNSUPPORTED, kSlabWhole);
    launch_diag(ctx, ctx->mac[ctx->cur], member, ctx->d_red, ctx->stream);
    LBL_CK(cudaGetLastError());
    double h[3];
    LBL_CK(cudaMemcpyAsync(h, ctx->d_red, sizeof(double) * 3, cudaMemcpyDeviceToHost, ctx->stream));
    LBL_CK(cudaStreamSynchronize(ctx->stream));
    const double n = double(ctx->P.nxy);
    if (energy) *energy = h[0] / n;
    if (enstrophy) *enstrophy = h[1] / n;
    if (mass) *mass = h[2] / n;
    return LBL_OK;
}

int lbl_rmse_uv(lbl_ctx* ctx, const float* u_true, const float* v_true, double* rmse) {
    if (!ctx || !u_true || !v_true || !rmse) return LBL_ERR_ARG;
    LBL_TRY(set_device(ctx));
    const size_t nxy = size_t(ctx->P.nxy);
    LBL_CK(cudaMemcpyAsync(ctx->d_tmp, u_true, sizeof(float) * nxy, cudaMemcpyHostToDevice, ctx->stream));
    LBL_CK(cudaMemcpyAsync(ctx->d_tmp + nxy, v_true, sizeof(float) * nxy, cudaMemcpyHostToDevice, ctx->stream));
    launch_rmse(ctx, ctx->mac[ctx->cur], ctx->d_tmp, ctx->d_tmp + nxy, ctx->d_red, ctx->stream);
    LBL_CK(cudaGetLastError());
    double h = 0;
    LBL_CK(cudaMemcpyAsync(&h, ctx->d_red, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    LBL_CK(cudaStreamSynchronize(ctx->stream));
    int ij0, n;
    rmse_cells(ctx, &ij0, &n);
    *rmse = std::sqrt(h / double(n));
    return LBL_OK;
}

// The true fields go up on the side stream, beside the work the engine stream still has
// queued (a cycle's forecast): ev[14] marks that the previous RMSE has read d_tmp, ev[13]
// that this one's fields have arrived.
int lbl_rmse_uv_async(lbl_ctx* ctx, const float* u_true, const float* v_true, double* rmse) {
    if (!ctx || !u_true || !v_true || !rmse) return LBL_ERR_ARG;
    LBL_TRY(set_device(ctx));
    const size_t nxy = size_t(ctx->P.nxy);
    LBL_CK(cudaStreamWaitEvent(ctx->side, ctx->ev[14], 0));
    LBL_CK(cudaMemcpyAsync(ctx->d_tmp, u_true, sizeof(float) * nxy, cudaMemcpyHostToDevice, ctx->side));
    LBL_CK(cudaMemcpyAsync(ctx->d_tmp + nxy, v_true, sizeof(float) * nxy, cudaMemcpyHostToDevice, ctx->side));
    LBL_CK(cudaEventRecord(ctx->ev[13], ctx->side));
    LBL_CK(cudaStreamWaitEvent(ctx->stream, ctx->ev[13], 0));
    launch_rmse(ctx, ctx->mac[ctx->cur], ctx->d_tmp, ctx->d_tmp + nxy, ctx->d_red, ctx->stream);
    launch_rmse_finish(ctx, ctx->d_red, ctx->stream);
    LBL_CK(cudaGetLastError());
    LBL_CK(cudaEventRecord(ctx->ev[14], ctx->stream));
    LBL_CK(cudaMemcpyAsync(rmse, ctx->d_red + 1, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    return LBL_OK;
}

void* lbl_get_stream(lbl_ctx* ctx) { return ctx ? static_cast<void*>(ctx->stream) : nullptr; }

int lbl_profile_step(lbl_ctx* ctx, int n, double* ms_per_launch) {
    if (!ctx || n < 1 || !ms_per_launch) return LBL_ERR_ARG;
    LBL_TRY(set_device(ctx));
    if (!ctx->initialised) return fail(ctx, LBL_ERR_STATE, "lbl_profile_step before lbl_init");
    const float* force = ctx->d_force + size_t(ctx->last_force_slot) * 2 * ctx->P.nxy;
    LBL_CK(cudaEventRecord(ctx->ev[8], ctx->stream));
    for (int k = 0; k < n; k++) {
        launch_lbm_step(ctx, ctx->cur, ctx->cur ^ 1, force, nullptr, ctx->stream);
        ctx->cur ^= 1;
    }
    LBL_CK(cudaGetLastError());
    LBL_CK(cudaEventRecord(ctx->ev[9], ctx->stream));
    LBL_CK(cudaEventSynchronize(ctx->ev[9]));
    float ms = 0;
    LBL_CK(cudaEventElapsedTime(&ms, ctx->ev[8], ctx->ev[9]));
    *ms_per_launch = double(ms) / n;
    return LBL_OK;
}

int lbl_autotune(lbl_ctx* ctx, int* strip_rows_out, double* ms_per_launch) {
    if (!ctx) return LBL_ERR_ARG;
    LBL_TRY(set_device(ctx));
    if (ctx->initialised) return fail(ctx, LBL_ERR_STATE, "lbl_autotune runs between lbl_create and lbl_init");
    // time the stream-collide on the rest state for candidate strip heights
    launch_rest_state(ctx, ctx->stream);
    LBL_CK(cudaGetLastError());
    const float* force = ctx->d_force;
    int best = 0;
    double best_ms = 1e30;
    // each candidate: the best of three samples of at least ~2 ms of back-to-back launches
    auto sample = [&](int reps, double* ms_out) -> int {
        LBL_CK(cudaEventRecord(ctx->ev[8], ctx->stream));
        for (int k = 0; k < reps; k++) launch_lbm_step(ctx, k & 1, (k & 1) ^ 1, force, nullptr, ctx->stream);
        LBL_CK(cudaEventRecord(ctx->ev[9], ctx->stream));
        LBL_CK(cudaEventSynchronize(ctx->ev[9]));
        LBL_CK(cudaGetLastError());
        float ms = 0;
        LBL_CK(cudaEventElapsedTime(&ms, ctx->ev[8], ctx->ev[9]));
        *ms_out = double(ms) / reps;
        return LBL_OK;
    };
    // the vector-load kernel also has two march forms (with and without the prefetched
    // row), and an LBL_LBM_AUTO context may take 1, 2 or 4 columns per thread; the
    // heuristic's own choice comes first, so a tie keeps it
    struct Form { int vec; bool pf; };
    std::vector<Form> forms{{ctx->vec, ctx->vec_pf}};
    Form best_form = forms[0];
    if (!ctx->closure && (ctx->vec || ctx->vec_auto)) {
        const std::vector<int> widths = ctx->vec_auto ? std::vector<int>{0, 2, 4} : std::vector<int>{ctx->vec};
        for (int w : widths)
            for (bool pf : {true, false})
                if ((w || pf) && !(w == ctx->vec && pf == ctx->vec_pf)) forms.push_back({w, pf});
    }
    for (const Form& fm : forms) {
        ctx->vec = fm.vec;
        ctx->vec_pf = fm.pf;
        ctx->ty_tuned = 0;
        const int heuristic = lbm_strip_rows(ctx);
        if (best == 0) best = heuristic;
        for (int ty : {heuristic, 2, 3, 4, 5, 6, 7, 8, 10, 12, 14, 16, 20, 24, 32, 40, 48, 64}) {
            if (ty > ctx->P.ny) continue;
            ctx->ty_tuned = ty;
            double one = 0;
            LBL_TRY(sample(2, &one));  // warm-up and a first estimate
            const int reps = int(std::min(200.0, std::max(4.0, 2.0 / std::max(one, 1e-4))));
            double t = 1e30;
            for (int k = 0; k < 3; k++) {
                double m = 0;
                LBL_TRY(sample(reps, &m));
                t = std::min(t, m);
            }
            if (t < best_ms * 0.99) { best_ms = t; best = ty; best_form = fm; }
        }
    }
    ctx->vec = best_form.vec;
    ctx->vec_pf = best_form.pf;
    ctx->ty_default = lbm_strip_rows(ctx);  // the heuristic's height for the kept form
    ctx->ty_tuned = best;
    LBL_TRY(check_timeout(ctx));
    if (strip_rows_out) *strip_rows_out = best;
    if (ms_per_launch) *ms_per_launch = best_ms;
    return LBL_OK;
}

int lbl_stream_collide_shape(const lbl_ctx* ctx, int* columns_per_thread, int* prefetch, int* strip_rows) {
    if (!ctx) return LBL_ERR_ARG;
    const bool vec = ctx->vec && !ctx->closure && !ctx->use_tma;
    if (columns_per_thread) *columns_per_thread = vec ? ctx->vec : 1;
    if (prefetch) *prefetch = vec ? int(ctx->vec_pf) : 1;
    if (strip_rows) *strip_rows = ctx->ty_tuned > 0 ? ctx->ty_tuned : ctx->ty_default;
    return LBL_OK;
}

int lbl_set_stream_collide_shape(lbl_ctx* ctx, int prefetch, int strip_rows) {
    if (!ctx) return LBL_ERR_ARG;
    LBL_TRY(set_device(ctx));
    const bool vec = ctx->vec && !ctx->closure && !ctx->use_tma;
    if (prefetch != 0 && prefetch != 1) return fail(ctx, LBL_ERR_ARG, "prefetch must be 0 or 1");
    if (!vec && prefetch == 0)
        return fail(ctx, LBL_ERR_UNSUPPORTED, "only the vector-load stream-collide has a march without prefetch");
    if (strip_rows < 0 || strip_rows > ctx->P.ny) return fail(ctx, LBL_ERR_ARG, "strip_rows must lie in [0, ny]");
    // graphs captured with the old shape are rebuilt on demand
    LBL_CK(cudaStreamSynchronize(ctx->stream));
    LBL_CK(cudaStreamSynchronize(ctx->side));
    for (auto& g : ctx->graphs) cudaGraphExecDestroy(g.second);
    ctx->graphs.clear();
    if (vec) ctx->vec_pf = prefetch == 1;
    ctx->ty_tuned = strip_rows;
    ctx->ty_default = lbm_strip_rows(ctx);
    if (ctx->closure && ctx->closure_every > 1) ctx->ty_held = lbm_strip_rows_held(ctx);
    return LBL_OK;
}

// ---------------------------------------------------------------------------
// y-slab split of one experiment (slab.cu has the halo kernel).  The context was created with
// cfg.ny = own rows + 2 halo; the constants come from the global grid; the forcing and the
// initial condition use global rows.  Every kernel then runs unchanged over the slab as if it
// were periodic: the rows the wrap corrupts are the outer ones, which the neighbours refresh.
// ---------------------------------------------------------------------------
int lbl_slab_set(lbl_ctx* ctx, int ny_global, int row0, int halo) {
    if (!ctx) return LBL_ERR_ARG;
    LBL_TRY(set_device(ctx));
    if (ctx->initialised) return fail(ctx, LBL_ERR_STATE, "lbl_slab_set after lbl_init");
    const lbl_config& cfg = ctx->cfg;
    if (cfg.mode != LBL_MODE_NATURE && cfg.mode != LBL_MODE_DA_LETKF)
        return fail(ctx, LBL_ERR_UNSUPPORTED, "a y-slab runs NATURE or DA_LETKF (OBSERVE draws its noise over the "
                                              "whole grid, nudging is not split)");
    if (cfg.write_mat) return fail(ctx, LBL_ERR_UNSUPPORTED, "a y-slab writes no LETKF matrices");
    if (ctx->closure) return fail(ctx, LBL_ERR_UNSUPPORTED, "a y-slab runs the Smagorinsky closure only");
    const int own = cfg.ny - 2 * halo;
    if (halo < 2) return fail(ctx, LBL_ERR_ARG, "the halo must hold at least 2 rows (the stream-collide reaches j +- 2)");
    if (own < halo) return fail(ctx, LBL_ERR_ARG, "a y-slab must own at least `halo` rows (cfg.ny >= 3 halo)");
    if (ny_global < own || 2 * halo > ny_global || row0 < 0 || row0 >= ny_global)
        return fail(ctx, LBL_ERR_ARG, "need own rows <= ny_global, 2 halo <= ny_global and 0 <= row0 < ny_global");
    if (cfg.mode == LBL_MODE_DA_LETKF) {
        // the analysis of an own row reads observation sites up to nl * p rows away; sites and the
        // analysis tiles (2 or 8 rows) must fall on the whole grid's
        const int reach = ctx->G.nl * ctx->G.p, p = ctx->G.p;
        int align = 8;
        while (align % p) align += 8;
        if (halo < reach) return fail(ctx, LBL_ERR_ARG, "the halo must cover the analysis window (nl * p rows)");
        if (halo % align || row0 % align || ny_global % p)
            return fail(ctx, LBL_ERR_ARG, "halo and row0 must be multiples of lcm(8, DA_XYPRUNE) and DA_XYPRUNE "
                                          "must divide ny_global");
    }
    ctx->slab_ny = ny_global;
    ctx->slab_row0 = row0;
    ctx->slab_halo = halo;
    ctx->P = derive_phys(cfg, ny_global, ((row0 - halo) % ny_global + ny_global) % ny_global);
    for (auto& g : ctx->graphs) cudaGraphExecDestroy(g.second);
    ctx->graphs.clear();
    return LBL_OK;
}

int lbl_slab_halo_bytes(const lbl_ctx* ctx, int rows, size_t* bytes) {
    if (!ctx || !bytes || rows < 0) return LBL_ERR_ARG;
    *bytes = size_t(ctx->P.M) * kQ * size_t(rows) * ctx->P.nx * (ctx->f16 ? sizeof(__half) : sizeof(float));
    return LBL_OK;
}

namespace {
int slab_halo(lbl_ctx* ctx, int rows, void* prev, void* next, bool unpack) {
    if (!ctx) return LBL_ERR_ARG;
    LBL_TRY(set_device(ctx));
    if (!ctx->slab_ny) return fail(ctx, LBL_ERR_STATE, "not a y-slab context (lbl_slab_set)");
    if (!ctx->initialised) return fail(ctx, LBL_ERR_STATE, "halo exchange before lbl_init");
    if (rows < 1 || rows > ctx->slab_halo) return fail(ctx, LBL_ERR_ARG, "rows must lie in [1, halo]");
    if (!prev || !next || (reinterpret_cast<uintptr_t>(prev) | reinterpret_cast<uintptr_t>(next)) % 16)
        return fail(ctx, LBL_ERR_ARG, "the halo buffers must be 16-byte aligned device memory");
    const int h = ctx->slab_halo, ny = ctx->P.ny;
    // sent: rows [2h - rows, 2h) go to the previous slab, [ny - 2h, ny - 2h + rows) to the next;
    // received: the previous slab's into [0, rows), the next's into [ny - rows, ny)
    const int a_prev = unpack ? 0 : 2 * h - rows, a_next = unpack ? ny - rows : ny - 2 * h;
    void* f = ctx->f16 ? static_cast<void*>(ctx->h[ctx->cur]) : static_cast<void*>(ctx->f[ctx->cur]);
    launch_slab_halo(f, ctx->f16 ? sizeof(__half) : sizeof(float), ctx->P.nx, ny, ctx->P.M * kQ, rows, a_prev,
                     a_next, prev, next, unpack, ctx->stream);
    LBL_CK(cudaGetLastError());
    return LBL_OK;
}
}  // namespace

int lbl_slab_forecast_steps(const lbl_ctx* ctx, int* max_steps) {
    if (!ctx || !max_steps) return LBL_ERR_ARG;
    *max_steps = ctx->force_cap;
    return LBL_OK;
}

int lbl_slab_forecast_begin(lbl_ctx* ctx, int t0, int nsteps) {
    if (!ctx) return LBL_ERR_ARG;
    LBL_TRY(set_device(ctx));
    (void)t0;
    if (!ctx->slab_ny) return fail(ctx, LBL_ERR_STATE, "not a y-slab context (lbl_slab_set)");
    if (!ctx->initialised) return fail(ctx, LBL_ERR_STATE, "lbl_slab_forecast_begin before lbl_init");
    if (ctx->fc_off < ctx->fc_total) return fail(ctx, LBL_ERR_STATE, kSlabBegun);
    if (nsteps < 1 || nsteps > ctx->force_cap)
        return fail(ctx, LBL_ERR_ARG, "nsteps must lie in [1, lbl_slab_forecast_steps]");
    // The forcing of every step at once, as the whole-grid cycle graph computes it.  After a
    // chunked forecast it runs on the side stream, beside whatever the context's stream still
    // runs (the analysis), once the last step that read the slots is done (ev[15]); the first
    // chunk waits for it (ev[16]).
    const bool side = ctx->fc_free_recorded;
    cudaStream_t fs = side ? ctx->side : ctx->stream;
    if (side) LBL_CK(cudaStreamWaitEvent(ctx->side, ctx->ev[15], 0));
    LBL_TRY(schedule_force(ctx, nsteps, fs));
    launch_force_chunk(ctx, nsteps, 0, fs);
    LBL_CK(cudaGetLastError());
    if (side) {
        LBL_CK(cudaEventRecord(ctx->ev[16], ctx->side));
        LBL_CK(cudaStreamWaitEvent(ctx->stream, ctx->ev[16], 0));
    }
    ctx->fc_total = nsteps;
    ctx->fc_off = 0;
    return LBL_OK;
}

int lbl_slab_forecast_chunk(lbl_ctx* ctx, int k) {
    if (!ctx) return LBL_ERR_ARG;
    LBL_TRY(set_device(ctx));
    if (ctx->fc_off >= ctx->fc_total)
        return fail(ctx, LBL_ERR_STATE, "no chunked forecast has steps left (lbl_slab_forecast_begin)");
    if (k < 1 || k > ctx->slab_halo / 2 || k > ctx->fc_total - ctx->fc_off)
        return fail(ctx, LBL_ERR_ARG, "k must lie in [1, min(halo / 2, steps left)]");
    const size_t plane2 = size_t(2) * ctx->P.nxy;
    for (int s = 0; s < k; s++) {
        const int g = ctx->fc_off + s, src = ctx->cur, dst = src ^ 1;
        // rho, u, v are written on the forecast's last two steps only, as by one lbl_update call
        float* mac = g >= ctx->fc_total - 2 ? ctx->mac[dst] : nullptr;
        launch_lbm_step(ctx, src, dst, ctx->d_force + size_t(g) * plane2, mac, ctx->stream, /*pdl=*/s > 0, g);
        ctx->cur = dst;
    }
    LBL_CK(cudaGetLastError());
    ctx->fc_off += k;
    ctx->last_force_slot = ctx->fc_off - 1;
    if (ctx->fc_off == ctx->fc_total) {  // the forcing slots are free once this step is done
        LBL_CK(cudaEventRecord(ctx->ev[15], ctx->stream));
        ctx->fc_free_recorded = true;
    }
    return LBL_OK;
}

int lbl_slab_pack(lbl_ctx* ctx, int rows, void* to_prev, void* to_next) {
    return slab_halo(ctx, rows, to_prev, to_next, false);
}

int lbl_slab_unpack(lbl_ctx* ctx, int rows, const void* from_prev, const void* from_next) {
    return slab_halo(ctx, rows, const_cast<void*>(from_prev), const_cast<void*>(from_next), true);
}

int lbl_set_io_prefix(lbl_ctx* ctx, const char* io_prefix) {
    if (!ctx || !io_prefix) return LBL_ERR_ARG;
    ctx->io_prefix = io_prefix;
    return LBL_OK;
}

int lbl_h5_write_dataset(const char* path, uint64_t d0, uint64_t d1, uint64_t d2, const void* data, int is_double) {
    if (!path || (!data && d0 * d1 * d2 > 0)) return LBL_ERR_ARG;
    const uint64_t dims[3] = {d0, d1, d2};
    std::string e;
    return write_h5_dataset(path, dims, data, is_double != 0, e);
}

int lbl_get_cycle_phases(lbl_ctx* ctx, double* analysis_ms, double* forecast_ms) {
    if (!ctx || !analysis_ms || !forecast_ms) return LBL_ERR_ARG;
    LBL_TRY(set_device(ctx));
    if (!ctx->phases) return fail(ctx, LBL_ERR_STATE, "lbl_get_cycle_phases before any forecast or cycle");
    LBL_CK(cudaEventSynchronize(ctx->ev[12]));
    float a = 0, f = 0;
    LBL_CK(cudaEventElapsedTime(&a, ctx->ev[10], ctx->ev[11]));
    LBL_CK(cudaEventElapsedTime(&f, ctx->ev[11], ctx->ev[12]));
    *analysis_ms = ctx->phases == 2 ? a : 0.0;
    *forecast_ms = f;
    return LBL_OK;
}

int lbl_event_record(lbl_ctx* ctx, int slot) {
    if (!ctx || slot < 0 || slot >= 8) return LBL_ERR_ARG;
    LBL_TRY(set_device(ctx));
    LBL_CK(cudaEventRecord(ctx->user_ev[slot], ctx->stream));
    return LBL_OK;
}

int lbl_event_elapsed(lbl_ctx* ctx, int a, int b, double* ms) {
    if (!ctx || a < 0 || a >= 8 || b < 0 || b >= 8 || !ms) return LBL_ERR_ARG;
    LBL_TRY(set_device(ctx));
    LBL_CK(cudaEventSynchronize(ctx->user_ev[b]));
    float v = 0;
    LBL_CK(cudaEventElapsedTime(&v, ctx->user_ev[a], ctx->user_ev[b]));
    *ms = v;
    return LBL_OK;
}

int lbl_timer_csv(lbl_ctx* ctx, int which, char* buf, size_t cap) {
    if (!ctx || which < 0 || which > 1) return LBL_ERR_ARG;
    const std::string s = timer_csv(ctx->timers[which]);
    if (buf && cap > 0) {
        const size_t n = std::min(cap - 1, s.size());
        std::memcpy(buf, s.data(), n);
        buf[n] = 0;
    }
    return int(s.size());
}

int lbl_timer_clear(lbl_ctx* ctx, int which) {
    if (!ctx || which < 0 || which > 1) return LBL_ERR_ARG;
    ctx->timers[which].map.clear();
    return LBL_OK;
}

int lbl_timer_transit(lbl_ctx* ctx, int which, const char* tag) {
    if (!ctx || !tag || which < 0 || which > 1) return LBL_ERR_ARG;
    timer_transit(ctx->timers[which], tag);
    return LBL_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Batches: several contexts cycled together, their forecasts stepped by one batched
// persistent launch per step (lbm_batch_step_kernel), their analyses and forcing
// on parallel branches of one CUDA graph per cycle.
// ---------------------------------------------------------------------------
struct lbl_batch {
    std::vector<lbl_ctx*> ctx;         // in item order (tallest strips first)
    std::vector<int> order;            // caller's index of each
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t fork_ev = nullptr, done_ev = nullptr;
    std::vector<cudaEvent_t> ready_ev, join_ev;
    bool launched = false;
    std::vector<BatchExp> exps;        // host copy of the table (cur set per graph)
    BatchExp* d_exps = nullptr;        // one device table per cur pattern, keyed in tables
    std::map<int, BatchExp*> tables;
    int* d_counter = nullptr;          // [kMaxBatchSteps] work counters, one per step
    int total = 0, grid = 0;
    int max_steps = 0;
    std::map<long long, cudaGraphExec_t> graphs;
    std::string err;
};

namespace {

int batch_fail(lbl_batch* b, int code, const std::string& msg) {
    b->err = msg;
    return code;
}

#define BATCH_CK(call)                                                                            \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess) return batch_fail(b, LBL_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

void batch_free(lbl_batch* b) {
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    for (auto& g : b->graphs) cudaGraphExecDestroy(g.second);
    for (auto& t : b->tables) cudaFree(t.second);
    cudaFree(b->d_counter);
    for (auto e : b->ready_ev) cudaEventDestroy(e);
    for (auto e : b->join_ev) cudaEventDestroy(e);
    if (b->fork_ev) cudaEventDestroy(b->fork_ev);
    if (b->done_ev) cudaEventDestroy(b->done_ev);
    if (b->stream) cudaStreamDestroy(b->stream);
}

// the device table of this cur pattern
int batch_table(lbl_batch* b, int cur_mask, BatchExp** out) {
    auto it = b->tables.find(cur_mask);
    if (it == b->tables.end()) {
        std::vector<BatchExp> t = b->exps;
        for (size_t e = 0; e < t.size(); e++) t[e].cur = (cur_mask >> e) & 1;
        BatchExp* d = nullptr;
        BATCH_CK(cudaMalloc(&d, sizeof(BatchExp) * t.size()));
        BATCH_CK(cudaMemcpy(d, t.data(), sizeof(BatchExp) * t.size(), cudaMemcpyHostToDevice));
        it = b->tables.emplace(cur_mask, d).first;
    }
    *out = it->second;
    return LBL_OK;
}

}  // namespace

extern "C" {

int lbl_batch_create(lbl_ctx* const* ctxs, int n, int strip_rows, lbl_batch** out) {
    if (!ctxs || !out || n < 1 || n > kMaxBatch || strip_rows < 0) return LBL_ERR_ARG;
    *out = nullptr;
    auto* b = new (std::nothrow) lbl_batch();
    if (!b) return LBL_ERR_NOMEM;
    std::vector<lbl_ctx*> v(ctxs, ctxs + n);
    int rc = LBL_OK;
    for (lbl_ctx* c : v) {
        if (!c || !c->initialised) { rc = LBL_ERR_STATE; b->err = "every context must exist and be initialised"; break; }
        if (c->device != v[0]->device) { rc = LBL_ERR_ARG; b->err = "the contexts of a batch share one device"; break; }
        if (c->f16 || c->use_tma || c->closure || c->slab_ny || c->P.nx % kBatchW != 0) {
            rc = LBL_ERR_UNSUPPORTED;
            b->err = "batched steps need FP32 storage, the direct stream-collide, no closure, whole grids and nx a "
                     "multiple of 128";
            break;
        }
    }
    for (size_t i = 0; rc == LBL_OK && i < v.size(); i++)
        for (size_t j = i + 1; j < v.size(); j++)
            if (v[i] == v[j]) { rc = LBL_ERR_ARG; b->err = "a context appears twice"; }
    if (rc != LBL_OK) {
        *out = b;  // for lbl_batch_last_error; the caller destroys it
        return rc;
    }
    b->device = v[0]->device;
    cudaSetDevice(b->device);
    auto ty_of = [&](const lbl_ctx* c) { return std::max(2, std::min(strip_rows > 0 ? strip_rows : 16, c->P.ny)); };
    std::vector<int> order(v.size());
    for (size_t i = 0; i < order.size(); i++) order[i] = int(i);
    std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return ty_of(v[a]) > ty_of(v[c]); });
    for (int i : order) b->ctx.push_back(v[i]);
    b->order = order;
    v = b->ctx;
    int item = 0;
    b->max_steps = 1 << 30;
    for (lbl_ctx* c : v) {
        BatchExp e{};
        e.f[0] = c->f[0];
        e.f[1] = c->f[1];
        e.mac[0] = c->mac[0];
        e.mac[1] = c->mac[1];
        e.force = c->d_force;
        e.P = c->P;
        e.ty = ty_of(c);
        e.strips = (c->P.ny + e.ty - 1) / e.ty;
        e.chunks = c->P.nx / kBatchW;
        e.item0 = item;
        item += c->P.M * e.strips * e.chunks;
        b->exps.push_back(e);
        b->max_steps = std::min(b->max_steps, c->force_cap);
    }
    b->total = item;
    auto done = [&](int code, const std::string& msg) {
        b->err = msg;
        *out = b;
        return code;
    };
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->fork_ev, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->done_ev, cudaEventDisableTiming) != cudaSuccess ||
        cudaMalloc(&b->d_counter, sizeof(int) * b->max_steps) != cudaSuccess)
        return done(LBL_ERR_CUDA, "batch resources");
    b->ready_ev.resize(v.size());
    b->join_ev.resize(v.size());
    for (size_t e = 0; e < v.size(); e++)
        if (cudaEventCreateWithFlags(&b->ready_ev[e], cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&b->join_ev[e], cudaEventDisableTiming) != cudaSuccess)
            return done(LBL_ERR_CUDA, "batch events");
    b->grid = std::min(b->total, batch_step_slots());
    *out = b;
    return LBL_OK;
}

const char* lbl_batch_last_error(const lbl_batch* b) { return b ? b->err.c_str() : "null batch"; }

int lbl_batch_destroy(lbl_batch* b) {
    if (!b) return LBL_OK;
    batch_free(b);
    delete b;
    return LBL_OK;
}

}  // extern "C"

namespace {

// One batch graph: the due analyses and every forcing chunk beside each other, then
// n_fc batched steps.  t < 0: a forecast-only continuation (no analysis, no uploads).
int batch_launch(lbl_batch* b, int t, const float* const* rho_o, const float* const* u_o, const float* const* v_o,
                 int n_fc) {
    const int n = int(b->ctx.size());
    int due_mask = 0, cur_mask = 0, after_mask = 0;
    for (int e = 0; e < n; e++) {
        lbl_ctx* ctx = b->ctx[e];
        // the previous batch graph read this context's schedule and observations
        if (b->launched) BATCH_CK(cudaStreamWaitEvent(ctx->stream, b->done_ev, 0));
        const bool due = t > 0 && is_da_mode(ctx->cfg.mode) && !ctx->cfg.da_dummy && da_due(ctx, t);
        const int ui = b->order[e];  // the caller's index
        const float* ro = rho_o ? rho_o[ui] : nullptr;
        const float* uo = u_o ? u_o[ui] : nullptr;
        const float* vo = v_o ? v_o[ui] : nullptr;
        if (t >= 0 && ro && uo && vo && is_da_mode(ctx->cfg.mode)) {
            const int rc = upload_obs(ctx, ro, uo, vo);
            if (rc != LBL_OK) return batch_fail(b, rc, ctx->err);
        }
        if (due && !ctx->have_obs) return batch_fail(b, LBL_ERR_STATE, "an analysis is due and no observations were given yet");
        const int rc = schedule_force(ctx, n_fc);
        if (rc != LBL_OK) return batch_fail(b, rc, ctx->err);
        BATCH_CK(cudaEventRecord(b->ready_ev[e], ctx->stream));
        const int cur = ctx->cur & 1;
        if (due) due_mask |= 1 << e;
        cur_mask |= cur << e;
        after_mask |= ((due && ctx->cfg.mode == LBL_MODE_DA_LETKF) ? cur ^ 1 : cur) << e;
    }
    for (int e = 0; e < n; e++) BATCH_CK(cudaStreamWaitEvent(b->stream, b->ready_ev[e], 0));
    const long long key = ((long long)due_mask << 40) | ((long long)n_fc << 20) | cur_mask;
    auto it = b->graphs.find(key);
    if (it == b->graphs.end()) {
        BatchExp* table = nullptr;
        LBL_TRY(batch_table(b, after_mask, &table));  // allocates: before the capture
        for (lbl_ctx* ctx : b->ctx) BATCH_CK(cudaStreamSynchronize(ctx->stream));
        BATCH_CK(cudaStreamSynchronize(b->stream));
        cudaGraph_t g = nullptr;
        BATCH_CK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        cudaEventRecord(b->fork_ev, b->stream);
        for (int e = 0; e < n; e++) {
            lbl_ctx* ctx = b->ctx[e];
            cudaStreamWaitEvent(ctx->stream, b->fork_ev, 0);
            cudaStreamWaitEvent(ctx->side, b->fork_ev, 0);
            launch_force_chunk(ctx, n_fc, 0, ctx->side);  // beside the analysis
            cudaEventRecord(ctx->join_ev, ctx->side);
            if ((due_mask >> e) & 1) enqueue_analysis(ctx, (cur_mask >> e) & 1, ctx->stream);
            cudaStreamWaitEvent(ctx->stream, ctx->join_ev, 0);
            cudaEventRecord(b->join_ev[e], ctx->stream);
            cudaStreamWaitEvent(b->stream, b->join_ev[e], 0);
        }
        cudaMemsetAsync(b->d_counter, 0, sizeof(int) * n_fc, b->stream);
        for (int k = 0; k < n_fc; k++)
            launch_batch_step(table, n, b->total, k, b->d_counter, b->grid, k >= n_fc - 2, k > 0, b->stream);
        const cudaError_t le = cudaGetLastError();
        const cudaError_t ee = cudaStreamEndCapture(b->stream, &g);
        if (le != cudaSuccess || ee != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            return batch_fail(b, LBL_ERR_CUDA, std::string("batch graph capture failed: ") +
                                                   cudaGetErrorString(le != cudaSuccess ? le : ee));
        }
        cudaGraphExec_t ge;
        const cudaError_t ie = cudaGraphInstantiate(&ge, g, cudaGraphInstantiateFlagUseNodePriority);
        cudaGraphDestroy(g);
        if (ie != cudaSuccess) return batch_fail(b, LBL_ERR_CUDA, std::string("batch graph instantiate: ") + cudaGetErrorString(ie));
        it = b->graphs.emplace(key, ge).first;
    }
    BATCH_CK(cudaGraphLaunch(it->second, b->stream));
    BATCH_CK(cudaEventRecord(b->done_ev, b->stream));
    b->launched = true;
    for (int e = 0; e < n; e++) {
        lbl_ctx* ctx = b->ctx[e];
        ctx->cur = ((after_mask >> e) & 1) ^ (n_fc & 1);
        ctx->last_force_slot = n_fc - 1;
        ctx->phases = 0;
        // later calls on the context run after the batch's graph
        BATCH_CK(cudaStreamWaitEvent(ctx->stream, b->done_ev, 0));
    }
    return LBL_OK;
}

}  // namespace

extern "C" {

int lbl_batch_cycle_async(lbl_batch* b, int t, const float* const* rho_o, const float* const* u_o,
                          const float* const* v_o, int n_fc) {
    if (!b) return LBL_ERR_ARG;
    if (n_fc < 1) return batch_fail(b, LBL_ERR_ARG, "n_fc must be >= 1");
    BATCH_CK(cudaSetDevice(b->device));
    // more steps than the smallest forcing buffer: the cycle graph takes the first
    // max_steps, forecast-only graphs the rest
    const int first = std::min(n_fc, b->max_steps);
    LBL_TRY(batch_launch(b, t < 0 ? 0 : t, rho_o, u_o, v_o, first));
    for (int done = first; done < n_fc; done += b->max_steps)
        LBL_TRY(batch_launch(b, -1, nullptr, nullptr, nullptr, std::min(b->max_steps, n_fc - done)));
    return LBL_OK;
}

int lbl_batch_sync(lbl_batch* b) {
    if (!b) return LBL_ERR_ARG;
    BATCH_CK(cudaSetDevice(b->device));
    BATCH_CK(cudaStreamSynchronize(b->stream));
    for (lbl_ctx* ctx : b->ctx) {
        const int rc = lbl_sync(ctx);
        if (rc != LBL_OK) return batch_fail(b, rc, ctx->err);
    }
    return LBL_OK;
}

}  // extern "C"
