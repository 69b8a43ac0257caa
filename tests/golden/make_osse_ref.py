"""Generate tests/golden/ref_osse_p4r1.npz: a whole DA_LETKF experiment run by the
reference's own code and by the engine on identical observations, so that their
analysis RMSE can be compared.

The reference side is oracle/_ref/ref_osse_p4r1 (oracle/ref_osse_harness.cu): the
nature run and 16 members as reference `data` objects advanced by the reference's
update() (src/lbm.cu, src/data.cu compiled unmodified), every 100 steps the members
analysed by the reference's LETKF call sequence (letkf.cu glue, letkf_solver.h's cuBLAS /
cuSOLVER calls) with the 256^2 x 16 workload's DA settings (DA_XYPRUNE 4,
LETKF_RLOC_LEN 1, LETKF_COVINF 1.1, OBS_ERROR_U 0.1, OBS_ERROR_RHO 0.01), observations
of the nature run's macros at every 4th point plus seeded noise.  It writes each cycle's observations and true (u, v).

The engine side replays them through the C ABI: the same configuration (the reference's
default physics, 256^2, 16 members with the reference's member initial conditions),
lbl_update for 100 steps, lbl_rmse_uv for the forecast, lbl_assimilate with the
reference's observation fields, lbl_rmse_uv for the analysis.  compat_stale_v is off so
that the analysis macros carry the analysis v (the reference's stale v reaches only
output: its update() recomputes every macro from the populations).

Both RMSEs are of the ensemble-mean (u, v) against the nature run's over the grid.
Stored: meta (JSON), ref_forecast, ref_analysis, engine_forecast, engine_analysis (one
value per cycle).  Needs a CUDA GPU and `make -C oracle ref REF_SRC=<reference src/>`.
Usage:  python tests/golden/make_osse_ref.py [--cycles 100] [--out tests/golden]
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "lbm2d-letkf_b200"))

import lbl  # noqa: E402

NX, M, STEPS, SEED = 256, 16, 100, 2025


def read_ref(path, cycles):
    nxy = NX * NX
    rec = 4 + 5 * 4 * nxy + 16
    raw = np.fromfile(path, np.uint8)
    assert raw.size == rec * cycles, (raw.size, rec * cycles)
    out = []
    for c in range(cycles):
        b = raw[c * rec:(c + 1) * rec]
        assert int(b[:4].view(np.int32)[0]) == c + 1
        f = b[4:4 + 5 * 4 * nxy].view(np.float32).reshape(5, NX, NX)
        fr, ar = b[4 + 5 * 4 * nxy:].view(np.float64)
        out.append((f[0].copy(), f[1].copy(), f[2].copy(), f[3].copy(), f[4].copy(), float(fr), float(ar)))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--cycles", type=int, default=100)
    ap.add_argument("--out", default=HERE)
    args = ap.parse_args()
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_osse_p4r1")
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "osse.bin")
        t0 = time.time()
        subprocess.run([exe, str(M), str(args.cycles), str(STEPS), str(SEED), path], check=True,
                       stdout=subprocess.DEVNULL)
        t_ref = time.time() - t0
        cyc = read_ref(path, args.cycles)
    cfg = lbl.config_default("DA_LETKF", NX, M, da_xyprune=4, letkf_rloc_len=1, letkf_covinf=1.1, obs_error_u=0.1,
                             obs_error_rho=0.01, iiter=20, daprune=5, compat_stale_v=0)
    e = lbl.Ensemble(cfg)
    e.init(0)
    eng_f, eng_a = [], []
    t0 = time.time()
    for c, (ro, uo, vo, ut, vt, _, _) in enumerate(cyc, start=1):
        e.update((c - 1) * STEPS, STEPS)
        eng_f.append(e.rmse_uv(ut, vt))
        e.assimilate(c * STEPS, ro, uo, vo)
        eng_a.append(e.rmse_uv(ut, vt))
    t_eng = time.time() - t0
    stats = e.letkf_stats()
    e.close()
    ref_f = np.array([x[5] for x in cyc])
    ref_a = np.array([x[6] for x in cyc])
    eng_f, eng_a = np.array(eng_f), np.array(eng_a)
    half = slice(args.cycles // 2, None)
    meta = {"grid": NX, "members": M, "steps_per_cycle": STEPS, "cycles": args.cycles, "obs_seed": SEED,
            "da": "DA_XYPRUNE 4, LETKF_RLOC_LEN 1, LETKF_COVINF 1.1, OBS_ERROR_U 0.1, OBS_ERROR_RHO 0.01",
            "physics": "the reference's defaults (Cs 0.2, nu 1e-4, band-limited IC); members: ensemble ids 334 + k",
            "reference": "oracle/_ref/ref_osse_p4r1 (oracle/ref_osse_harness.cu)",
            "engine_letkf_stats": stats, "wall_s": {"reference": t_ref, "engine": t_eng},
            "mean_analysis_rmse_second_half": {"reference": float(ref_a[half].mean()),
                                               "engine": float(eng_a[half].mean())},
            "mean_forecast_rmse_second_half": {"reference": float(ref_f[half].mean()),
                                               "engine": float(eng_f[half].mean())}}
    path = os.path.join(args.out, "ref_osse_p4r1.npz")
    np.savez_compressed(path, meta=json.dumps(meta), ref_forecast=ref_f, ref_analysis=ref_a, engine_forecast=eng_f,
                        engine_analysis=eng_a)
    print(json.dumps(meta))


if __name__ == "__main__":
    main()
