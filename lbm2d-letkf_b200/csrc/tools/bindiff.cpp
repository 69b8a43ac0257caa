// lbl_bindiff -- RMSE of (u, v) between two output directories for every output step
// t <= t_iter with t % skip == 0, in the reference tool's argument order and output
// format (bindiff/main.cpp): stdout "t,rmse", stderr "t: rmse (count = n)".
//
// usage: lbl_bindiff <dir0> <dir1> <t_iter> [--skip=10]
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>

#include "../../../include/lbl.h"

int main(int argc, char** argv) {
    int skip = 10;  // ioprune (bindiff/main.cpp:28)
    const char* pos[3] = {nullptr, nullptr, nullptr};
    int np = 0;
    for (int a = 1; a < argc; a++) {
        if (std::strncmp(argv[a], "--skip=", 7) == 0) skip = std::atoi(argv[a] + 7);
        else if (np < 3) pos[np++] = argv[a];
    }
    if (np < 3 || skip < 1) {
        std::fprintf(stderr, "usage: lbl_bindiff <dir0> <dir1> <t_iter> [--skip=10]\n");
        return 2;
    }
    const int t_iter = std::atoi(pos[2]);
    char err[512];
    for (int t = 0; t <= t_iter; t++) {
        if (t % skip != 0) continue;
        double rmse = 0;
        long long count = 0;
        if (lbl_bindiff(pos[0], pos[1], t, &rmse, &count, err, sizeof(err)) != LBL_OK) {
            std::cerr << err << std::endl;
            return 1;
        }
        std::cerr << t << ": " << rmse << " (count = " << count << ")" << std::endl;
        std::cout << t << "," << rmse << std::endl;
    }
    return 0;
}
