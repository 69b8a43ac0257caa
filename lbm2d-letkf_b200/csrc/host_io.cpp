// host_io.cpp -- host-side parts of the path that the reference runs on the CPU:
// raw .dat field files (io.cu:26-44), zero-padded step names
// (util/stringutils.hpp:10-20), host FP32 vorticity (io.cu:61-86), OBSERVE noise
// and NaN pruning (io.cu:160-246), and the "#tag,sec" tag timers
// (util/timer.hpp:32-72).  These run in FP32 on the host exactly like the
// reference so that OBSERVE output is bit-identical.
#include <sys/stat.h>
#include <sys/time.h>

#include <cerrno>
#include <cmath>
#include <cstdio>
#include <iomanip>
#include <random>
#include <sstream>

#include "lbl_internal.h"

namespace lbl {

std::string to_string_aligned(int t, int digits) {
    std::stringstream ss;
    ss << std::setfill('0') << std::setw(digits) << t;
    return ss.str();
}

int write_dat(const std::string& fname, const float* p, size_t n, std::string& err) {
    std::FILE* fp = std::fopen(fname.c_str(), "wb");
    if (!fp) { err = "could not open file: " + fname; return LBL_ERR_IO; }
    const size_t w = std::fwrite(p, sizeof(float), n, fp);
    std::fclose(fp);
    if (w != n) { err = "IOError: fwrite failed: " + fname; return LBL_ERR_IO; }
    return LBL_OK;
}

int read_dat(const std::string& fname, float* p, size_t n, std::string& err) {
    std::FILE* fp = std::fopen(fname.c_str(), "rb");
    if (!fp) { err = "IOError: could not open file: " + fname; return LBL_ERR_IO; }
    const size_t r = std::fread(p, sizeof(float), n, fp);
    std::fclose(fp);
    if (r != n) { err = "IOError: short read: " + fname; return LBL_ERR_IO; }
    return LBL_OK;
}

int mkdir_p(const std::string& path) {
    std::string cur;
    for (size_t i = 0; i <= path.size(); i++) {
        if (i == path.size() || path[i] == '/') {
            if (!cur.empty() && ::mkdir(cur.c_str(), 0755) != 0 && errno != EEXIST) return -1;
        }
        if (i < path.size()) cur.push_back(path[i]);
    }
    return 0;
}

void vorticity_host(int nx, int ny, float dx, const float* u, const float* v, float* vor) {
    for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
            const int iw = (i - 1 + nx) % nx, ie = (i + 1) % nx, js = (j - 1 + ny) % ny, jn = (j + 1) % ny;
            const float us = u[i + nx * js], un = u[i + nx * jn];
            const float uy = (un - us) / (2 * dx);
            const float vw = v[iw + nx * j], ve = v[ie + nx * j];
            const float vx = (ve - vw) / (2 * dx);
            vor[i + nx * j] = vx - uy;
        }
}

void* obs_engine_new(uint32_t seed) { return new std::mt19937(seed); }
void obs_engine_free(void* e) { delete static_cast<std::mt19937*>(e); }

void observe_host(void* engine, int nx, int ny, int p, float er, float eu, const float* r, const float* u,
                  const float* v, float* ro, float* uo, float* vo, float* voro, float dx) {
    auto& eng = *static_cast<std::mt19937*>(engine);
    std::normal_distribution<float> dist(0, 1);  // fresh per call, like io.cu:322
    const size_t nxy = size_t(nx) * ny;
    for (size_t ij = 0; ij < nxy; ij++) {
        ro[ij] = r[ij] + er * dist(eng);
        uo[ij] = u[ij] + eu * dist(eng);
        vo[ij] = v[ij] + eu * dist(eng);
    }
    vorticity_host(nx, ny, dx, uo, vo, voro);
    for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++)
            if (i % p != 0 || j % p != 0) {
                const size_t ij = i + size_t(nx) * j;
                ro[ij] = NAN; uo[ij] = NAN; vo[ij] = NAN; voro[ij] = NAN;
            }
}

double wall_time() {
    timeval tv;
    gettimeofday(&tv, nullptr);
    return tv.tv_sec + 1e-6 * tv.tv_usec;
}

void timer_transit(TimerMap& t, const std::string& tag) {
    const double now = wall_time();
    if (t.t0 == 0) t.t0 = now;
    t.map[t.cur] += now - t.t0;
    t.cur = tag;
    t.t0 = now;
}

void timer_add(TimerMap& t, const std::string& tag, double sec) { t.map[tag] += sec; }

std::string timer_csv(const TimerMap& t) {
    std::ostringstream os;
    os << "#tag,sec" << std::endl;
    for (const auto& m : t.map) os << m.first << ',' << m.second << std::endl;
    return os.str();
}

}  // namespace lbl
