// ref_lbm_harness.cu -- ORACLE TOOLING (test infrastructure only).
//
// A driver of our own around the reference's unmodified LBM sources
// (src/lbm.cu, src/data.cu, compiled from where they lie by oracle/Makefile).  It
// builds one reference `data` object (data.h:45-64: IC + forcing init) for a given
// ensemble id and calls the reference's `update()` (lbm.h:16-29) step by step,
// dumping the reference's own arrays (f, r, u, v, force_x, force_y, the cuRAND
// normal buffer and its cursor) as raw little-endian float32 files.  The outputs
// pin the CPU oracle and the CUDA engine against the reference itself.
//
// usage: ref_lbm <out_dir> <ensemble_id> <nsteps> <dump_step>[,<dump_step>...]
//        ref_lbm time <ensemble_id> <nsteps> <warmup> [<ready_file> <go_file>]
//
// The `time` form runs `warmup` untimed steps, then (when given the two files)
// creates <ready_file> and waits, at most 300 s, for <go_file> to appear, so that
// several such processes sharing one GPU start their timed steps together, as the
// reference's one-rank-per-member runs do.  It prints
//   ref_lbm_time <ensemble_id> <nsteps> <t0_ns> <t1_ns>
// with CLOCK_REALTIME stamps around the timed steps (the end after a device sync).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <set>
#include <sstream>
#include <string>
#include <vector>

#include <unistd.h>

#include <cuda_runtime.h>

#include "config.h"
#include "data.h"
#include "lbm.h"

static void dump(const std::string& name, const void* p, size_t bytes) {
    std::FILE* fp = std::fopen(name.c_str(), "wb");
    if (!fp) { std::fprintf(stderr, "cannot write %s\n", name.c_str()); std::exit(1); }
    std::fwrite(p, 1, bytes, fp);
    std::fclose(fp);
}

static void dump_state(data& dat, const std::string& dir, int step) {
    cudaDeviceSynchronize();
    const std::string pre = dir + "/s" + std::to_string(step) + "_";
    const size_t nxy = size_t(config::nx) * config::ny;
    dump(pre + "f.f32", dat.d().f.data(), sizeof(real) * nxy * config::Q);
    dump(pre + "r.f32", dat.d().r.data(), sizeof(real) * nxy);
    dump(pre + "u.f32", dat.d().u.data(), sizeof(real) * nxy);
    dump(pre + "v.f32", dat.d().v.data(), sizeof(real) * nxy);
    dump(pre + "fx.f32", dat.d0().force_x.data(), sizeof(real) * nxy);
    dump(pre + "fy.f32", dat.d0().force_y.data(), sizeof(real) * nxy);
    const int cursor = dat.d0().i_rand_outdated;
    dump(pre + "cursor.i32", &cursor, sizeof(int));
}

static long long now_ns() {
    timespec ts;
    clock_gettime(CLOCK_REALTIME, &ts);
    return ts.tv_sec * 1000000000LL + ts.tv_nsec;
}

static int time_steps(int argc, char** argv) {
    const int id = std::atoi(argv[2]);
    const int nsteps = std::atoi(argv[3]);
    const int warmup = std::atoi(argv[4]);
    auto dat = data(id);
    for (int s = 0; s < warmup; s++) update(dat, s);
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) { std::fprintf(stderr, "CUDA error: %s\n", cudaGetErrorString(e)); return 1; }
    if (argc >= 7) {
        std::FILE* fp = std::fopen(argv[5], "w");
        if (!fp) { std::fprintf(stderr, "cannot write %s\n", argv[5]); return 1; }
        std::fclose(fp);
        const long long limit = now_ns() + 300LL * 1000000000LL;
        while (access(argv[6], F_OK) != 0) {
            if (now_ns() > limit) { std::fprintf(stderr, "ref_lbm: no start signal within 300 s\n"); return 3; }
            usleep(100);
        }
    }
    const long long t0 = now_ns();
    for (int s = warmup; s < warmup + nsteps; s++) update(dat, s);
    e = cudaDeviceSynchronize();
    const long long t1 = now_ns();
    if (e != cudaSuccess) { std::fprintf(stderr, "CUDA error: %s\n", cudaGetErrorString(e)); return 1; }
    std::printf("ref_lbm_time %d %d %lld %lld\n", id, nsteps, t0, t1);
    return 0;
}

int main(int argc, char** argv) {
    if (argc >= 5 && std::strcmp(argv[1], "time") == 0) return time_steps(argc, argv);
    if (argc < 5) { std::fprintf(stderr, "usage: %s out_dir ensemble_id nsteps dumps\n", argv[0]); return 2; }
    const std::string dir = argv[1];
    const int id = std::atoi(argv[2]);
    const int nsteps = std::atoi(argv[3]);
    std::set<int> dumps;
    {
        std::stringstream ss(argv[4]);
        std::string tok;
        while (std::getline(ss, tok, ',')) dumps.insert(std::atoi(tok.c_str()));
    }
    auto dat = data(id);
    cudaDeviceSynchronize();
    {  // forcing tables and the first normal buffer (serves the first 1023 forcing calls)
        auto& d0 = dat.d0();
        const int n = int(d0.force_amp.size());
        dump(dir + "/modes_kx.f32", d0.force_kx.data(), sizeof(real) * n);
        dump(dir + "/modes_ky.f32", d0.force_ky.data(), sizeof(real) * n);
        dump(dir + "/modes_amp.f32", d0.force_amp.data(), sizeof(real) * n);
        std::vector<float> buf(d0.n_rand_buf);
        cudaMemcpy(buf.data(), d0.force_theta_d, sizeof(float) * buf.size(), cudaMemcpyDeviceToHost);
        dump(dir + "/normals.f32", buf.data(), sizeof(float) * buf.size());
    }
    if (dumps.count(0)) dump_state(dat, dir, 0);
    for (int s = 1; s <= nsteps; s++) {
        update(dat, s - 1);
        if (dumps.count(s)) dump_state(dat, dir, s);
    }
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) { std::fprintf(stderr, "CUDA error: %s\n", cudaGetErrorString(e)); return 1; }
    std::printf("ref_lbm: id %d, %d steps, dumps in %s\n", id, nsteps, dir.c_str());
    return 0;
}
