// lbl_run.cpp -- host driver replacing the reference's main() (src/main.cu:22-155)
// for the forecast-and-assimilate path.  All M members run in this one process on
// one GPU through liblbl's C ABI; run modes, loop order, the spin-up, the
// DROP_FORMER_HALF_TIMER rule, the io/ file layout and the elapsed_time CSVs
// follow the reference.
//
// usage: lbl_run --mode=NATURE|OBSERVE|DA_LETKF|DA_NUDGING [--nx=256] [--n_ens=M] [--KEY=VALUE ...] [ens_offset]
//   KEY is one of the reference's knobs: DAPRUNE IOPRUNE DA_XYPRUNE LETKF_RLOC_LEN
//   LETKF_COVINF OBS_ERROR_RHO OBS_ERROR_U DA_DUMMY DA_QUADRA DA_NUD_RATE DA_OBS_UV, or
//   SPINUP ITER_MAIN IIITER CS NU TAU IC (reference|k4exp) IC_AMP
//   ENS_INIT (independent|perturbed) ENS_PERTURB PREFIX DEVICE
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/lbl.h"

namespace {

int check(lbl_ctx* ctx, int rc, const char* what) {
    if (rc != LBL_OK) {
        std::fprintf(stderr, "lbl_run: %s failed (%d): %s\n", what, rc, ctx ? lbl_last_error(ctx) : "");
        std::exit(1);
    }
    return rc;
}

bool starts(const std::string& a, const char* p) { return a.rfind(p, 0) == 0; }

std::string timer_text(lbl_ctx* ctx, int which) {
    const int n = lbl_timer_csv(ctx, which, nullptr, 0);
    std::vector<char> buf(size_t(n) + 1);
    lbl_timer_csv(ctx, which, buf.data(), buf.size());
    return std::string(buf.data());
}

double timer_get(const std::string& csv, const std::string& tag) {
    size_t pos = csv.find("\n" + tag + ",");
    if (pos == std::string::npos) return 0.0;
    return std::atof(csv.c_str() + pos + tag.size() + 2);
}

}  // namespace

int main(int argc, char** argv) {
    std::string mode_s = "NATURE", prefix = "io";
    int nx = 256, M = 1, ofs = 0, device = 0;
    std::vector<std::pair<std::string, std::string>> kv;
    for (int a = 1; a < argc; a++) {
        std::string s = argv[a];
        if (starts(s, "--")) {
            const size_t eq = s.find('=');
            const std::string k = s.substr(2, eq == std::string::npos ? std::string::npos : eq - 2);
            const std::string v = eq == std::string::npos ? "1" : s.substr(eq + 1);
            if (k == "mode") mode_s = v;
            else if (k == "nx") nx = std::atoi(v.c_str());
            else if (k == "n_ens") M = std::atoi(v.c_str());
            else if (k == "PREFIX") prefix = v;
            else if (k == "DEVICE") device = std::atoi(v.c_str());
            else kv.emplace_back(k, v);
        } else {
            ofs = std::atoi(s.c_str());  // main.cu:42-45: argv[1] = ensemble offset
        }
    }
    const int mode = mode_s == "OBSERVE"      ? LBL_MODE_OBSERVE
                     : mode_s == "DA_LETKF"   ? LBL_MODE_DA_LETKF
                     : mode_s == "DA_NUDGING" ? LBL_MODE_DA_NUDGING
                                              : LBL_MODE_NATURE;
    const bool da = mode == LBL_MODE_DA_LETKF || mode == LBL_MODE_DA_NUDGING;  // DATA_ASSIMILATION
    lbl_config cfg;
    lbl_config_default(&cfg, mode, nx, M);
    for (auto& p : kv) {
        const std::string& k = p.first;
        const char* v = p.second.c_str();
        if (k == "DAPRUNE") cfg.daprune = std::atoi(v);
        else if (k == "IOPRUNE") cfg.ioprune = std::atoi(v);
        else if (k == "DA_XYPRUNE") cfg.da_xyprune = std::atoi(v);
        else if (k == "LETKF_RLOC_LEN") cfg.letkf_rloc_len = std::atoi(v);
        else if (k == "LETKF_COVINF") cfg.letkf_covinf = std::atof(v);
        else if (k == "OBS_ERROR_RHO") cfg.obs_error_rho = std::atof(v);
        else if (k == "OBS_ERROR_U") cfg.obs_error_u = std::atof(v);
        else if (k == "SPINUP") cfg.spinup = std::atoi(v);
        else if (k == "ITER_MAIN") cfg.iter_main = std::atoi(v);
        else if (k == "IITER") cfg.iiter = std::atoi(v);
        else if (k == "CS") cfg.cs = std::atof(v);
        else if (k == "NU") cfg.nu = std::atof(v);
        else if (k == "TAU") cfg.tau = std::atof(v);
        else if (k == "IC") cfg.ic_kind = std::string(v) == "k4exp" ? LBL_IC_K4EXP : LBL_IC_REFERENCE;
        else if (k == "IC_AMP") cfg.ic_amp = std::atof(v);
        else if (k == "ENS_INIT") cfg.ens_init = std::string(v) == "perturbed" ? LBL_ENS_PERTURBED : LBL_ENS_INDEPENDENT;
        else if (k == "ENS_PERTURB") cfg.ens_perturb = std::atof(v);
        else if (k == "DA_DUMMY") cfg.da_dummy = std::atoi(v);
        else if (k == "DA_QUADRA") cfg.da_quadra = std::atoi(v);
        else if (k == "DA_NUD_RATE") cfg.da_nud_rate = std::atof(v);
        else if (k == "DA_OBS_UV") cfg.da_obs_ruv = std::atoi(v) ? 0 : 1;
        else { std::fprintf(stderr, "lbl_run: unknown option --%s\n", k.c_str()); return 2; }
    }

    lbl_ctx* ctx = nullptr;
    const int rc = lbl_create(&cfg, device, &ctx);
    if (rc != LBL_OK) {
        std::fprintf(stderr, "lbl_run: lbl_create failed (%d): %s\n", rc, ctx ? lbl_last_error(ctx) : "");
        lbl_destroy(ctx);
        return 1;
    }
    const int T = LBL_TIMER_MAIN;
    std::printf("mode: %s, nx = %d, members = %d, iiter = %d\n", mode_s.c_str(), nx, M, cfg.iiter);
    lbl_timer_transit(ctx, T, "unit tests");
    lbl_timer_transit(ctx, T, "allocate data");
    check(ctx, lbl_init(ctx, ofs), "lbl_init");
    if (cfg.spinup > 0) {
        lbl_timer_transit(ctx, T, "spinup");
        std::printf("spin-up ...\n");
        check(ctx, lbl_update(ctx, -cfg.spinup, cfg.spinup), "spin-up");
        std::printf("spin-up finished\n");
    }
    lbl_timer_transit(ctx, T, "_main");
    const int iter_total = (mode == LBL_MODE_OBSERVE || (da && cfg.da_dummy)) ? cfg.iter_main + 1  // config.h:144-151
                                                                                : cfg.iter_main;
    for (int tt = 0; tt < iter_total / cfg.iiter + 1; tt++) {
        const int t = tt * cfg.iiter;
        if (mode == LBL_MODE_DA_LETKF && t == iter_total / 2) {  // DROP_FORMER_HALF_TIMER, main.cu:85-92
            lbl_timer_clear(ctx, T);
            lbl_timer_clear(ctx, LBL_TIMER_LETKF);
        }
        if (da && !cfg.da_dummy) {                                   // main.cu:94
            lbl_timer_transit(ctx, T, "DA");
            if (t > 0) check(ctx, lbl_assimilate_files(ctx, t, prefix.c_str()), "assimilate");
            lbl_timer_transit(ctx, T, "_sync.DA");
        }
        lbl_timer_transit(ctx, T, "output");
        check(ctx, lbl_output_async(ctx, t, prefix.c_str()), "output");  // files written beside the next steps
        lbl_timer_transit(ctx, T, "_sync.output");
        lbl_timer_transit(ctx, T, "forecast");
        check(ctx, lbl_update(ctx, t, cfg.iiter), "forecast");
        lbl_timer_transit(ctx, T, "_sync.forecast");
    }
    lbl_timer_transit(ctx, T, "_ignored");
    check(ctx, lbl_sync(ctx), "output");  // the last files are written and their status known

    const std::string main_csv = timer_text(ctx, T);
    const double fc = timer_get(main_csv, "forecast"), out = timer_get(main_csv, "output"), t_da = timer_get(main_csv, "DA");
    std::printf("\nElapsed time%s:\n%s", mode == LBL_MODE_DA_LETKF ? " for latter half loop" : "", main_csv.c_str());
    const double lu = double(nx) * nx * iter_total;
    // main.cu:128-133 prints these per member with the full iter_total (2x overstated
    // in DA_LETKF, where the timers cover the latter half only); the ensemble rates
    // below count every member and the steps the timers actually cover.
    std::printf("core MLUPS (reference formula, per member): %g\n", 1e-6 * lu / fc);
    std::printf("total MLUPS (reference formula, per member): %g\n", 1e-6 * lu / (fc + out + t_da));
    const double covered = mode == LBL_MODE_DA_LETKF ? 0.5 : 1.0;
    std::printf("ensemble GLUPS (forecast tag): %g\n", 1e-9 * lu * M * covered / fc);
    if (mode == LBL_MODE_DA_LETKF) std::printf("LETKF breakdown:\n%s", timer_text(ctx, LBL_TIMER_LETKF).c_str());

    auto fout = [&](const std::string& name, const std::string& text) {
        std::FILE* fp = std::fopen(name.c_str(), "w");
        if (!fp) { std::fprintf(stderr, "lbl_run: cannot write %s\n", name.c_str()); return; }
        std::fputs(text.c_str(), fp);
        std::fclose(fp);
    };
    fout(prefix + "/elapsed_time_rank0.csv", main_csv);
    if (mode == LBL_MODE_DA_LETKF) fout(prefix + "/letkf_elapsed_time_rank0.csv", timer_text(ctx, LBL_TIMER_LETKF));
    lbl_destroy(ctx);
    return 0;
}
