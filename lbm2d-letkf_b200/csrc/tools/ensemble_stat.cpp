// lbl_ensemble_stat -- spread and RMSE of the ensemble mean against the nature run for
// every output step t <= t_iter with t % skip == 0, in the reference tool's argument
// order and output format (ensemble_stat/main.cpp).  The grid size comes from the
// files; the member count is --n_ens (the reference's -D N_ENS), by default the
// number of consecutive ens%04d directories found.
//
// usage: lbl_ensemble_stat <nature_prefix> <ensemble_prefix> <t_iter> [--n_ens=N] [--skip=10]
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>

#include <sys/stat.h>

#include "../../../include/lbl.h"

int main(int argc, char** argv) {
    int skip = 10, n_ens = 0;
    const char* pos[3] = {nullptr, nullptr, nullptr};
    int np = 0;
    for (int a = 1; a < argc; a++) {
        if (std::strncmp(argv[a], "--skip=", 7) == 0) skip = std::atoi(argv[a] + 7);
        else if (std::strncmp(argv[a], "--n_ens=", 8) == 0) n_ens = std::atoi(argv[a] + 8);
        else if (np < 3) pos[np++] = argv[a];
    }
    if (np < 3 || skip < 1) {
        std::fprintf(stderr, "usage: lbl_ensemble_stat <nature_prefix> <ensemble_prefix> <t_iter> [--n_ens=N] [--skip=10]\n");
        return 2;
    }
    if (n_ens <= 0) {
        struct stat st;
        char d[64];
        while (n_ens < 9999) {
            std::snprintf(d, sizeof(d), "/ens%04d", n_ens);
            if (stat((std::string(pos[1]) + d).c_str(), &st) != 0) break;
            n_ens++;
        }
    }
    std::cout << "dirinfo: nature=" << pos[0] << " -- " << "ensemble=" << pos[1] << std::endl;
    const int t_iter = std::atoi(pos[2]);
    char err[512];
    for (int t = 0; t <= t_iter; t++) {
        if (t % skip != 0) continue;
        double s[5];
        if (lbl_ensemble_stat(pos[0], pos[1], n_ens, t, s, err, sizeof(err)) != LBL_OK) {
            std::cout << err << std::endl;
            return 1;
        }
        std::cout << "t_step, spread, rmse, rho_spread, rho_rmse, max(debug) = " << t << ", " << s[0] << ", " << s[1]
                  << ", " << s[2] << ", " << s[3] << ", " << s[4] << std::endl;
        std::cerr << t << ", " << s[0] << ", " << s[1] << ", " << s[2] << ", " << s[3] << std::endl;
    }
    return 0;
}
