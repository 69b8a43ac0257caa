// ref_letkf_harness.cu -- ORACLE TOOLING (test infrastructure only).
//
// One LETKF analysis of given inputs by the reference's own call sequence
// (ref_letkf_solver.cu, which says what of the reference it runs and restates).
//
// usage: ref_letkf <in.bin> <out.bin>
//   in:  int32 nx, ny, M, j0, j1; float32 f[M][9][ny][nx]; ro, uo, vo [ny][nx]
//   out: int32 nx, ny, M, j0, j1, evd (0 syevjBatched, 1 per-matrix syevj);
//        float32 fa[M][9][ny][nx] (the analysis where computed, the input elsewhere);
//        float32 lambda[ny][nx][M] (eigenvalues in cuSOLVER's order; 0 where not computed)
// Only the ranks whose points meet rows [j0, j1) are computed.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

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

using real = float;
static constexpr int n_stt = 9;

static std::vector<char> read_all(const char* path) {
    std::FILE* fp = std::fopen(path, "rb");
    if (!fp) { std::fprintf(stderr, "cannot read %s\n", path); std::exit(1); }
    std::vector<char> buf;
    char tmp[1 << 16];
    size_t n;
    while ((n = std::fread(tmp, 1, sizeof(tmp), fp)) > 0) buf.insert(buf.end(), tmp, tmp + n);
    std::fclose(fp);
    return buf;
}

int main(int argc, char** argv) {
    if (argc != 3) {
        std::fprintf(stderr, "usage: %s <in.bin> <out.bin>\n", argv[0]);
        return 1;
    }
    const std::vector<char> in = read_all(argv[1]);
    int hdr[5];
    if (in.size() < sizeof(hdr)) { std::fprintf(stderr, "short input\n"); return 1; }
    std::memcpy(hdr, in.data(), sizeof(hdr));
    const int nx = hdr[0], ny = hdr[1], M = hdr[2], j0 = hdr[3], j1 = hdr[4];
    const size_t nxy = size_t(nx) * ny;
    if (nx < 1 || ny < 1 || M < 2 || ny % M || nx > 1024 || ny > 65535 || j0 < 0 || j1 > ny || j0 >= j1) {
        std::fprintf(stderr, "bad header\n");
        return 1;
    }
    const size_t need = sizeof(hdr) + sizeof(real) * (size_t(M) * n_stt * nxy + 3 * nxy);
    if (in.size() != need) { std::fprintf(stderr, "input size %zu, expected %zu\n", in.size(), need); return 1; }
    const real* h_f = reinterpret_cast<const real*>(in.data() + sizeof(hdr));
    const real* h_obs = h_f + size_t(M) * n_stt * nxy;

    std::vector<real*> f(M), fa(M);
    for (int k = 0; k < M; k++) {
        CK(cudaMalloc(&f[k], sizeof(real) * n_stt * nxy));
        CK(cudaMalloc(&fa[k], sizeof(real) * n_stt * nxy));
        CK(cudaMemcpy(f[k], h_f + size_t(k) * n_stt * nxy, sizeof(real) * n_stt * nxy, cudaMemcpyHostToDevice));
        CK(cudaMemcpy(fa[k], f[k], sizeof(real) * n_stt * nxy, cudaMemcpyDeviceToDevice));
    }
    real *ro, *uo, *vo, *lam;
    CK(cudaMalloc(&ro, sizeof(real) * nxy));
    CK(cudaMalloc(&uo, sizeof(real) * nxy));
    CK(cudaMalloc(&vo, sizeof(real) * nxy));
    CK(cudaMalloc(&lam, sizeof(real) * nxy * M));
    CK(cudaMemset(lam, 0, sizeof(real) * nxy * M));
    CK(cudaMemcpy(ro, h_obs, sizeof(real) * nxy, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(uo, h_obs + nxy, sizeof(real) * nxy, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(vo, h_obs + 2 * nxy, sizeof(real) * nxy, cudaMemcpyHostToDevice));
    const int evd = refletkf::analyse(std::vector<const float*>(f.begin(), f.end()), fa, ro, uo, vo, nx, ny, j0, j1,
                                      lam);

    std::FILE* fp = std::fopen(argv[2], "wb");
    if (!fp) { std::fprintf(stderr, "cannot write %s\n", argv[2]); return 1; }
    const int ohdr[6] = {nx, ny, M, j0, j1, evd};
    std::fwrite(ohdr, sizeof(int), 6, fp);
    std::vector<real> h(n_stt * nxy);
    for (int k = 0; k < M; k++) {
        CK(cudaMemcpy(h.data(), fa[k], sizeof(real) * h.size(), cudaMemcpyDeviceToHost));
        std::fwrite(h.data(), sizeof(real), h.size(), fp);
    }
    std::vector<real> hl(nxy * M);
    CK(cudaMemcpy(hl.data(), lam, sizeof(real) * hl.size(), cudaMemcpyDeviceToHost));
    std::fwrite(hl.data(), sizeof(real), hl.size(), fp);
    std::fclose(fp);
    std::printf("ref_letkf: nx=%d ny=%d M=%d rows [%d,%d) evd=%s\n", nx, ny, M, j0, j1,
                evd ? "per-matrix syevj (EigenG stand-in)" : "syevjBatched");
    return 0;
}
