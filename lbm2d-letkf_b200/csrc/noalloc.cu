// noalloc.cu -- an LETKF analysis entry point that allocates no device memory.
//
// Who needs it: callers that own every device buffer themselves and must not let
// a library call cudaMalloc.  Examples are a host framework with its own caching
// allocator or memory budget, where a hidden cudaMalloc would fragment or overrun
// its pool and would synchronise the device, and code that launches from a
// context where allocation is not allowed.  Such a caller passes its forecast
// populations, its observations at the sites and its output buffers.
//
// The analysis needs scratch memory beyond its inputs and outputs: the
// observation-space ensemble at the sites (dY, dyo), the window weight table and
// four counters.  Here that scratch is one file-scope __device__ array of fixed
// size, kNoAllocScratchBytes (8 MiB).  CUDA loads the module that holds it lazily,
// so the first call on a device is the one that takes those 8 MiB (plus the
// module) from the device: make it during the caller's set-up, before a memory
// budget is fixed.  From then on the device holds the array until the process
// exits.  All calls share the array and it keeps the last call's contents; every
// call rebuilds the weight table on the device and clears the counters, so a call
// reads nothing an earlier call left.  Two calls that overlap on the GPU (different
// streams, or different host threads) race on it: serialise them.
//
// Set-up: the first call on a device, with that device current, looks up the
// device address of the array (cudaGetSymbolAddress) and opts the analysis kernel
// in to its shared-memory size.  Make that first call before any stream capture.
// Every call enqueues only kernels and a memset on the caller's stream; it waits
// for the stream only when host_stats is given, and only then can it report a NaN
// in the analysis (LBL_ERR_NAN).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "lbl_internal.h"

constexpr size_t kNoAllocScratchBytes = size_t(8) << 20;
constexpr size_t kNoAllocScratchFloats = kNoAllocScratchBytes / sizeof(float);

// The scratch.  In host code this name is only a stand-in: its device address
// comes from cudaGetSymbolAddress (scratch_for_current_device below).
static __device__ __align__(256) float g_noalloc_scratch[kNoAllocScratchFloats];

namespace {

constexpr int kMaxDevices = 64;
float* g_scratch_addr[kMaxDevices] = {};
std::mutex g_setup_mutex;
thread_local std::string g_noalloc_error;

int noalloc_fail(int code, const std::string& msg) {
    g_noalloc_error = msg;
    return code;
}

// once per device, with that device current
int scratch_for_current_device(float** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return noalloc_fail(LBL_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return noalloc_fail(LBL_ERR_UNSUPPORTED, "device index out of range");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[dev]) {
        float* ptr = nullptr;
        e = cudaGetSymbolAddress(reinterpret_cast<void**>(&ptr), g_noalloc_scratch);
        if (e != cudaSuccess || !ptr)
            return noalloc_fail(LBL_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        if (lbl::analysis_prepare() != 0) return noalloc_fail(LBL_ERR_CUDA, "cudaFuncSetAttribute(analysis_kernel) failed");
        g_scratch_addr[dev] = ptr;
    }
    *out = g_scratch_addr[dev];
    return LBL_OK;
}

// Gaspari-Cohn weight (letkf.cu:104-109) as IEEE double operations in the source
// order of the host table builder (lbl_api.cu), so the device-built table below is
// bit-identical to the one lbl_create uploads: no contraction into FMAs.
__device__ double gc_weight_rn(double d) {
    if (d <= 0) return 1.0;
    const double d2 = __dmul_rn(d, d), d3 = __dmul_rn(d2, d), d4 = __dmul_rn(d3, d), d5 = __dmul_rn(d4, d);
    const double t3 = __ddiv_rn(__dmul_rn(d3, 5.), 8.), t4 = __ddiv_rn(__dmul_rn(d2, 5.), 3.);
    if (d <= 1) {
        const double nd5 = __dmul_rn(__dmul_rn(__dmul_rn(__dmul_rn(-d, d), d), d), d);
        double s = __dadd_rn(__ddiv_rn(nd5, 4.), __ddiv_rn(d4, 2.));
        s = __dadd_rn(s, t3);
        s = __dsub_rn(s, t4);
        return __dadd_rn(s, 1.);
    }
    if (d <= 2) {
        double s = __dsub_rn(__ddiv_rn(d5, 12.), __ddiv_rn(d4, 2.));
        s = __dadd_rn(s, t3);
        s = __dadd_rn(s, t4);
        s = __dsub_rn(s, __dmul_rn(d, 5.));
        s = __dadd_rn(s, 4.);
        return __dsub_rn(s, __ddiv_rn(2. / 3., d));
    }
    return 0.0;
}

// The window weight table (set_rR, letkf.cu:75-114), built on the device on every
// call so that no host memory is involved: one thread per pattern (i mod p, j mod p)
// lists the window slots with weight > 0, {slot, var, sqrt(w) bits, w bits}, then
// the pattern's count at tab[4 p^2 nobs + pattern].
__global__ void noalloc_weight_table_kernel(int p, int nox, int nl, int off, double dloc, double sig_u,
                                            double sig_rho, int nobs, int* tab) {
    const int pat = blockIdx.x * blockDim.x + threadIdx.x;
    if (pat >= p * p) return;
    const int pi = pat % p, pj = pat / p;
    int n = 0;
    for (int b = 0; b < nox; b++)
        for (int a = 0; a < nox; a++) {
            const int di = pi - (a - (nl - off)) * p, dj = pj - (b - (nl - off)) * p;
            if (abs(di) > nl * p || abs(dj) > nl * p) continue;
            const double g =
                p > 1 ? gc_weight_rn(__ddiv_rn(__dsqrt_rn(double(di * di + dj * dj)), __dadd_rn(dloc, 1e-6))) : 1.0;
            for (int var = 0; var < 3; var++) {
                const double sig = var == 2 ? sig_rho : sig_u;
                const float w = __double2float_rn(__ddiv_rn(g, __dmul_rn(sig, sig)));
                if (!(w > 0.f)) continue;
                int* e = tab + (size_t(pat) * nobs + n) * 4;
                e[0] = a + nox * b + var * nox * nox;
                e[1] = var;
                e[2] = __float_as_int(__fsqrt_rn(w));
                e[3] = __float_as_int(w);
                n++;
            }
        }
    tab[size_t(4) * p * p * nobs + pat] = n;
}

}  // namespace

namespace {
int analysis_noalloc_impl(const lbl_config* cfg, const float* f_in, float* f_out, float* mac_out,
                          const float* yo_sites, void* stream, int* host_stats);
}

extern "C" int lbl_letkf_analysis_noalloc(const lbl_config* cfg, const float* f_in, float* f_out, float* mac_out,
                                          const float* yo_sites, void* stream, int* host_stats, char* err,
                                          size_t err_cap) {
    g_noalloc_error.clear();
    const int rc = analysis_noalloc_impl(cfg, f_in, f_out, mac_out, yo_sites, stream, host_stats);
    if (err && err_cap > 0) {
        const size_t n = std::min(err_cap - 1, g_noalloc_error.size());
        std::memcpy(err, g_noalloc_error.data(), n);
        err[n] = 0;
    }
    return rc;
}

namespace {
int analysis_noalloc_impl(const lbl_config* cfg, const float* f_in, float* f_out, float* mac_out,
                          const float* yo_sites, void* stream, int* host_stats) {
    if (!cfg || !f_in || !f_out || !mac_out || !yo_sites) return noalloc_fail(LBL_ERR_ARG, "null argument");
    const lbl_config& c = *cfg;
    if (c.abi_version != LBL_ABI_VERSION) return noalloc_fail(LBL_ERR_ARG, "abi_version mismatch");
    if (c.nx < 32 || c.nx > 1024 || c.nx % 32 != 0 || c.ny < 8)
        return noalloc_fail(LBL_ERR_ARG, "nx must be a multiple of 32 in [32, 1024] and ny >= 8");
    if (c.n_ens < 2 || c.n_ens > lbl::kMaxMemberLanes)
        return noalloc_fail(LBL_ERR_UNSUPPORTED, "n_ens must be in [2, 32]");
    if (c.da_xyprune < 1 || c.nx % c.da_xyprune || c.ny % c.da_xyprune)
        return noalloc_fail(LBL_ERR_ARG, "DA_XYPRUNE must divide nx and ny");
    if (c.letkf_rloc_len < 0 || c.letkf_rloc_len > 8) return noalloc_fail(LBL_ERR_ARG, "LETKF_RLOC_LEN out of range");
    if (!(c.letkf_covinf > 0) || !(c.obs_error_u > 0) || !(c.obs_error_rho > 0) || !(c.cfl > 0) || !(c.u_ref > 0))
        return noalloc_fail(LBL_ERR_ARG, "LETKF_COVINF, OBS_ERROR_*, cfl and u_ref must be > 0");
    if (c.jacobi_max_sweeps < 1 || c.jacobi_max_sweeps > 1000) return noalloc_fail(LBL_ERR_ARG, "jacobi_max_sweeps out of range");

    // window geometry (letkf.cu:45-56)
    const int p = c.da_xyprune;
    int nl, off, nox;
    double dloc;
    if (c.letkf_rloc_len <= 0) {
        dloc = p - 1; nl = p == 1 ? 0 : 2; off = p == 1 ? 0 : 1; nox = p == 1 ? 1 : 4;
    } else {
        dloc = double(c.letkf_rloc_len) * p; off = 0; nl = c.letkf_rloc_len * 2; nox = nl * 2 + 1;
    }
    const int nobs = 3 * nox * nox;
    const int M = c.n_ens;
    const size_t nsites = size_t(c.nx / p) * (c.ny / p);
    if (lbl::analysis_smem_bytes(M, nobs) > lbl::kAnalysisSmemLimit)
        return noalloc_fail(LBL_ERR_UNSUPPORTED, "observation window too large for the analysis kernel");

    // scratch layout (floats, each part 256-B aligned): dY, dyo, weight table, counters
    auto round64 = [](size_t n) { return (n + 63) & ~size_t(63); };
    const size_t n_dY = round64(3 * nsites * M), n_dyo = round64(3 * nsites);
    const size_t n_tab = round64(size_t(4) * p * p * nobs + size_t(p) * p), n_stats = 64;
    const size_t need = n_dY + n_dyo + n_tab + n_stats;
    if (need > kNoAllocScratchFloats)
        return noalloc_fail(LBL_ERR_UNSUPPORTED,
                            "configuration needs " + std::to_string(need * sizeof(float)) +
                                " bytes of analysis scratch; the allocation-free entry point holds " +
                                std::to_string(kNoAllocScratchBytes) + " (reduce n_ens, grid or raise DA_XYPRUNE)");

    float* scratch = nullptr;
    int rc = scratch_for_current_device(&scratch);
    if (rc != LBL_OK) return rc;
    float* dY = scratch;
    float* dyo = dY + n_dY;
    int* tab = reinterpret_cast<int*>(dyo + n_dyo);
    int* stats = reinterpret_cast<int*>(dyo + n_dyo + n_tab);

    // every call: the weight table for this configuration, then cleared counters;
    // kernels and a memset only, all on `stream`, no host memory involved
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    noalloc_weight_table_kernel<<<(p * p + 127) / 128, 128, 0, s>>>(p, nox, nl, off, dloc, c.obs_error_u,
                                                                     c.obs_error_rho, nobs, tab);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemsetAsync(stats, 0, sizeof(int) * 4, s);
    if (e != cudaSuccess) return noalloc_fail(LBL_ERR_CUDA, std::string("scratch set-up: ") + cudaGetErrorString(e));

    lbl::AnalysisArgs a{};
    a.f_in = f_in; a.f_out = f_out; a.mac_out = mac_out; a.yo = yo_sites;
    a.dY = dY; a.dyo = dyo; a.wtab = tab; a.stats = stats;
    a.nx = c.nx; a.ny = c.ny; a.M = M; a.p = p; a.nox = nox; a.nl_off = nl - off; a.nobs = nobs;
    a.diag = float((M - 1) / c.letkf_covinf);
    a.sqrt_m1 = float(std::sqrt(double(M - 1)));
    a.tol = float(c.jacobi_tol);
    a.c = float(c.u_ref) / float(c.cfl);
    a.max_sweeps = c.jacobi_max_sweeps;
    a.write_v = c.compat_stale_v ? 0 : 1;
    lbl::launch_obs_ensemble_args(a, s);
    lbl::launch_analysis_args(a, s);
    e = cudaGetLastError();
    if (e != cudaSuccess) return noalloc_fail(LBL_ERR_CUDA, std::string("analysis launch: ") + cudaGetErrorString(e));
    if (host_stats) {
        e = cudaMemcpyAsync(host_stats, stats, sizeof(int) * 4, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return noalloc_fail(LBL_ERR_CUDA, std::string("counters: ") + cudaGetErrorString(e));
        if (host_stats[2]) return noalloc_fail(LBL_ERR_NAN, "NaN in the LETKF analysis");
    }
    return LBL_OK;
}
}  // namespace
