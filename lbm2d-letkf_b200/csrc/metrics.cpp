// metrics.cpp -- the reference's evaluation measures, as host functions of the C ABI:
//   lbl_bindiff         RMSE of (u, v) between two output directories (bindiff/main.cpp:27-69)
//   lbl_ensemble_stat   spread and RMSE of the ensemble mean against the nature run
//                       (ensemble_stat/main.cpp:33-170), grid size taken from the files
//   lbl_energy_spectrum shell-summed spectrum of postprocess/fourier.ipynb cell 2
// They read the .dat files that lbl_output writes (raw float32, nx*ny, row-major).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "lbl_internal.h"

namespace {

void set_err(char* err, size_t cap, const std::string& msg) {
    if (err && cap > 0) {
        const size_t n = std::min(cap - 1, msg.size());
        std::memcpy(err, msg.data(), n);
        err[n] = '\0';
    }
}

std::string step_name(const std::string& dir, const char* var, int step) {
    char buf[64];
    std::snprintf(buf, sizeof(buf), "/%s_step%010d.dat", var, step);
    return dir + buf;
}

// whole file as float32; false if it cannot be read
bool read_all(const std::string& path, std::vector<float>& out) {
    std::FILE* fp = std::fopen(path.c_str(), "rb");
    if (!fp) return false;
    std::fseek(fp, 0, SEEK_END);
    const long bytes = std::ftell(fp);
    std::fseek(fp, 0, SEEK_SET);
    if (bytes < 0 || bytes % 4 != 0) { std::fclose(fp); return false; }
    out.resize(size_t(bytes) / 4);
    const size_t got = out.empty() ? 0 : std::fread(out.data(), 4, out.size(), fp);
    std::fclose(fp);
    return got == out.size();
}

}  // namespace

extern "C" {

int lbl_bindiff(const char* dir0, const char* dir1, int step, double* rmse, long long* count, char* err,
                size_t err_cap) {
    if (!dir0 || !dir1 || !rmse || step < 0) { set_err(err, err_cap, "null argument"); return LBL_ERR_ARG; }
    long double sum_sq_error = 0;
    long long n = 0;
    for (const char* var : {"u", "v"}) {                            // bindiff/main.cpp:20-25 (default)
        std::vector<float> a, b;
        const std::string fa = step_name(dir0, var, step), fb = step_name(dir1, var, step);
        if (!read_all(fa, a)) { set_err(err, err_cap, "could not read file: " + fa); return LBL_ERR_IO; }
        if (!read_all(fb, b)) { set_err(err, err_cap, "could not read file: " + fb); return LBL_ERR_IO; }
        const size_t m = std::min(a.size(), b.size());           // reads pairwise until either file ends
        for (size_t i = 0; i < m; i++) {
            const float e = a[i] - b[i];                            // real arithmetic (main.cpp:57-59)
            sum_sq_error += e * e;
            n++;
        }
    }
    *rmse = double(std::sqrt(sum_sq_error / n));
    if (count) *count = n;
    return LBL_OK;
}

int lbl_ensemble_stat(const char* nature_dir, const char* ens_dir, int n_ens, int step, double* out, char* err,
                      size_t err_cap) {
    if (!nature_dir || !ens_dir || !out || n_ens < 1 || n_ens > 9999 || step < 0) {
        set_err(err, err_cap, "bad argument");
        return LBL_ERR_ARG;
    }
    const char* vars[3] = {"u", "v", "rho"};
    std::vector<float> nat[3];
    for (int k = 0; k < 3; k++) {
        const std::string f = step_name(std::string(nature_dir) + "/ens0000", vars[k], step);
        if (!read_all(f, nat[k])) { set_err(err, err_cap, "could not read file: " + f); return LBL_ERR_IO; }
    }
    const size_t nxy = nat[0].size();                               // the grid comes from the data
    if (nxy == 0 || nat[1].size() != nxy || nat[2].size() != nxy) {
        set_err(err, err_cap, "nature files differ in size");
        return LBL_ERR_IO;
    }
    std::vector<std::vector<float>> ens(size_t(n_ens) * 3);
    for (int m = 0; m < n_ens; m++) {
        char d[32];
        std::snprintf(d, sizeof(d), "/ens%04d", m);
        for (int k = 0; k < 3; k++) {
            const std::string f = step_name(std::string(ens_dir) + d, vars[k], step);
            std::vector<float>& a = ens[size_t(m) * 3 + k];
            if (!read_all(f, a)) { set_err(err, err_cap, "could not read file: " + f); return LBL_ERR_IO; }
            if (a.size() != nxy) { set_err(err, err_cap, "size mismatch: " + f); return LBL_ERR_IO; }
        }
    }
    // per-cell mean and standard deviation in long double, kept as float (main.cpp:112-138)
    std::vector<float> mean[3], sd[3];
    for (int k = 0; k < 3; k++) {
        mean[k].resize(nxy);
        sd[k].resize(nxy);
        for (size_t i = 0; i < nxy; i++) {
            long double s = 0, ss = 0;
            for (int m = 0; m < n_ens; m++) {
                const long double x = ens[size_t(m) * 3 + k][i];
                s += x;
                ss += x * x;
            }
            const long double mu = s / n_ens, var = ss / n_ens - mu * mu;
            mean[k][i] = float(mu);
            sd[k][i] = float(var <= 0 ? 0 : std::sqrt(var));        // sqrt_epsilon (main.cpp:27-29)
        }
    }
    // spread and RMSE against nature: (u, v) together, rho alone (main.cpp:139-170)
    long double sp_vel = 0, se_vel = 0, sp_rho = 0, se_rho = 0, mx = 0;
    for (size_t i = 0; i < nxy; i++) {
        for (int k = 0; k < 2; k++) {
            const long double cm = mean[k][i], cs = sd[k][i], e = cm - (long double)nat[k][i];
            sp_vel += cs * cs;
            se_vel += e * e;
            mx = std::max(mx, cm);
        }
        const long double cm = mean[2][i], cs = sd[2][i], e = cm - (long double)nat[2][i];
        sp_rho += cs * cs;
        se_rho += e * e;
    }
    out[0] = double(std::sqrt(sp_vel / (2 * nxy)));   // spread
    out[1] = double(std::sqrt(se_vel / (2 * nxy)));   // rmse
    out[2] = double(std::sqrt(sp_rho / nxy));         // rho_spread
    out[3] = double(std::sqrt(se_rho / nxy));         // rho_rmse
    out[4] = double(mx);                              // max(debug)
    return LBL_OK;
}

int lbl_energy_spectrum(const float* u, const float* v, int nx, int ny, double* ek) {
    if (!u || !v || !ek || nx < 2 || ny < 2) return LBL_ERR_ARG;
    // fourier.ipynb cell 2: F = fftn(.)/nx/ny over the [ny][nx] field; for the
    // non-negative wavenumbers i (rows), j (columns) <= kmax = nx/2, shell
    // k = int(sqrt(i^2 + j^2) + 0.5) <= kmax collects |(Fu^2 + Fv^2)/2| (complex squares).
    const int kmax = nx / 2;
    std::vector<double> cx(nx), sx(nx), cy(ny), sy(ny);
    for (int m = 0; m < nx; m++) { cx[m] = std::cos(2 * M_PI * m / nx); sx[m] = std::sin(2 * M_PI * m / nx); }
    for (int m = 0; m < ny; m++) { cy[m] = std::cos(2 * M_PI * m / ny); sy[m] = std::sin(2 * M_PI * m / ny); }
    const int nj = kmax + 1, ni = std::min(kmax, ny - 1) + 1;
    auto dft = [&](const float* a, std::vector<double>& re, std::vector<double>& im) {
        std::vector<double> r1(size_t(ny) * nj), i1(size_t(ny) * nj);
        for (int y = 0; y < ny; y++)                                  // along x: columns j
            for (int j = 0; j < nj; j++) {
                double sr = 0, si = 0;
                for (int x = 0; x < nx; x++) {
                    const int t = int((long long)j * x % nx);
                    sr += a[size_t(y) * nx + x] * cx[t];
                    si -= a[size_t(y) * nx + x] * sx[t];
                }
                r1[size_t(y) * nj + j] = sr;
                i1[size_t(y) * nj + j] = si;
            }
        re.assign(size_t(ni) * nj, 0.0);
        im.assign(size_t(ni) * nj, 0.0);
        for (int i = 0; i < ni; i++)                                  // along y: rows i
            for (int y = 0; y < ny; y++) {
                const int t = int((long long)i * y % ny);
                const double c = cy[t], s = -sy[t];
                for (int j = 0; j < nj; j++) {
                    const double ar = r1[size_t(y) * nj + j], ai = i1[size_t(y) * nj + j];
                    re[size_t(i) * nj + j] += ar * c - ai * s;
                    im[size_t(i) * nj + j] += ar * s + ai * c;
                }
            }
        const double norm = 1.0 / (double(nx) * ny);
        for (auto& x : re) x *= norm;
        for (auto& x : im) x *= norm;
    };
    std::vector<double> ur, ui, vr, vi;
    dft(u, ur, ui);
    dft(v, vr, vi);
    for (int k = 0; k <= kmax; k++) ek[k] = 0;
    for (int i = 0; i < ni; i++)
        for (int j = 0; j < nj; j++) {
            const int k = int(std::sqrt(double(i * i + j * j)) + 0.5);
            if (k > kmax) continue;
            const size_t o = size_t(i) * nj + j;
            const double re = 0.5 * (ur[o] * ur[o] - ui[o] * ui[o] + vr[o] * vr[o] - vi[o] * vi[o]);
            const double im = 0.5 * (2 * ur[o] * ui[o] + 2 * vr[o] * vi[o]);
            ek[k] += std::sqrt(re * re + im * im);
        }
    return LBL_OK;
}

}  // extern "C"
