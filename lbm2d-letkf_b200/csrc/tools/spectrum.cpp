// lbl_spectrum -- the energy spectrum of postprocess/fourier.ipynb cell 2, averaged
// over the output steps t0, t0 + dt, ... <= t1 of one directory (the notebook's
// sub(): steps 1000..2000 by 10).  Prints "k,E(k)" for k = 0..nx/2 and the
// notebook's energy-contribution ratio R(kf) = sum_{k<kf} E / sum E.
//
// usage: lbl_spectrum <dir> [--t0=1000] [--t1=2000] [--dt=10] [--kf=4]
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../../include/lbl.h"

static bool load(const std::string& path, std::vector<float>& a) {
    std::FILE* fp = std::fopen(path.c_str(), "rb");
    if (!fp) return false;
    std::fseek(fp, 0, SEEK_END);
    const long n = std::ftell(fp) / 4;
    std::fseek(fp, 0, SEEK_SET);
    a.resize(size_t(n));
    const bool ok = n > 0 && std::fread(a.data(), 4, a.size(), fp) == a.size();
    std::fclose(fp);
    return ok;
}

int main(int argc, char** argv) {
    int t0 = 1000, t1 = 2000, dt = 10, kf = 4;
    const char* dir = nullptr;
    for (int a = 1; a < argc; a++) {
        if (std::strncmp(argv[a], "--t0=", 5) == 0) t0 = std::atoi(argv[a] + 5);
        else if (std::strncmp(argv[a], "--t1=", 5) == 0) t1 = std::atoi(argv[a] + 5);
        else if (std::strncmp(argv[a], "--dt=", 5) == 0) dt = std::atoi(argv[a] + 5);
        else if (std::strncmp(argv[a], "--kf=", 5) == 0) kf = std::atoi(argv[a] + 5);
        else dir = argv[a];
    }
    if (!dir || dt < 1 || t1 < t0) {
        std::fprintf(stderr, "usage: lbl_spectrum <dir> [--t0=1000] [--t1=2000] [--dt=10] [--kf=4]\n");
        return 2;
    }
    std::vector<double> mean;
    int count = 0, nx = 0;
    for (int t = t0; t <= t1; t += dt) {
        char name[64];
        std::vector<float> u, v;
        std::snprintf(name, sizeof(name), "/u_step%010d.dat", t);
        const bool ok_u = load(std::string(dir) + name, u);
        std::snprintf(name, sizeof(name), "/v_step%010d.dat", t);
        if (!ok_u || !load(std::string(dir) + name, v) || u.size() != v.size()) {
            std::fprintf(stderr, "lbl_spectrum: cannot read step %d in %s\n", t, dir);
            return 1;
        }
        nx = int(std::lround(std::sqrt(double(u.size()))));
        if (size_t(nx) * nx != u.size()) { std::fprintf(stderr, "lbl_spectrum: grid is not square\n"); return 1; }
        std::vector<double> ek(size_t(nx / 2 + 1));
        lbl_energy_spectrum(u.data(), v.data(), nx, nx, ek.data());
        if (mean.empty()) mean.assign(ek.size(), 0.0);
        for (size_t k = 0; k < ek.size(); k++) mean[k] += std::fabs(ek[k]);
        count++;
    }
    double tot = 0, low = 0;
    for (size_t k = 0; k < mean.size(); k++) {
        mean[k] /= count;
        tot += mean[k];
        if (int(k) < kf) low += mean[k];
        std::printf("%zu,%.10e\n", k, mean[k]);
    }
    std::fprintf(stderr, "R(kf): %.6f\n", tot > 0 ? low / tot : 0.0);
    return 0;
}
