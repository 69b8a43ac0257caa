"""The learned eddy-viscosity closure around the engine (include/lbl.h, lbl_closure_*):
training data from box-filtered fine runs that the engine itself computes, GPU
training, the saved parameters, and the comparison against plain Smagorinsky.

The closure has no counterpart in the reference, whose eddy viscosity is the fixed
Smagorinsky term of lbm.cu:42-60.  A coarse run (the 256^2 DA configuration) uses
nu_t = m (cs dx)^2 |S| with m from a 6-32-32-1 MLP of the local velocity-gradient
invariants; the training target is the m that makes the Smagorinsky stress match
the subgrid stress of an 8x box filter of a 2048^2 run with the same physics.

    python -m lbl.closure train --out lbm2d-letkf_b200/lbl/closure_c4.npz
    python -m lbl.closure eval --params lbm2d-letkf_b200/lbl/closure_c4.npz
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

import lbl

Q = 9
EX = np.array([(q % 3) - 1 for q in range(Q)], np.float64)
EY = np.array([(q // 3) - 1 for q in range(Q)], np.float64)
W = np.array([4 / 9 if EX[q] == 0 and EY[q] == 0 else (1 / 9 if EX[q] == 0 or EY[q] == 0 else 1 / 36)
              for q in range(Q)])
DEFAULT_PARAMS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "closure_c4.npz")


def phys(cfg) -> dict:
    """c, dx, dt, nu of a configuration, as the engine derives them (FP32 constants)."""
    c = np.float32(cfg.u_ref) / np.float32(cfg.cfl)
    dx = np.float32(cfg.h_ref) / np.float32(cfg.ny - 1)
    dt = dx / c
    nu = np.float32((cfg.tau - 0.5) * float(c) * float(c) * float(dt) / 3.0 if cfg.tau > 0 else cfg.nu)
    return {"c": float(c), "dx": float(dx), "dt": float(dt), "nu": float(nu)}


def coarse_config(nx: int = 256, n_ens: int = 16, mode: str = "DA_LETKF", **kw):
    """The DA configuration the closure serves: 256^2, Cs 0.1, tau 0.51, K4EXP IC at rms
    1, observations every 4th point, GC radius 4 cells, inflation 1.1."""
    args = dict(da_xyprune=4, letkf_rloc_len=1, letkf_covinf=1.1, obs_error_u=0.1, obs_error_rho=0.01, daprune=5,
                cs=0.1, tau=0.51, ic_kind=lbl.IC_K4EXP, ic_amp=1.0, ens_init=lbl.ENS_PERTURBED, ens_perturb=0.1)
    args.update(kw)
    return lbl.config_default(mode, nx, n_ens, **args)


def fine_config(coarse, filter: int, members: int):
    """A NATURE run filter times finer with the coarse run's physics: the same domain,
    IC spectrum and molecular viscosity (tau follows from nu), and the same forcing
    and friction per unit time.  The engine applies both per step (lbm.h:41-70): the
    random force is drawn afresh every step, so its energy input per unit time goes
    as fkf^2 dt and fkf scales with sqrt(dt_coarse / dt_fine); the friction removes
    friction_rate of the velocity per step, so friction_rate scales with dt_fine /
    dt_coarse."""
    f = lbl.config_default("NATURE", coarse.nx * filter, members)
    for k in ("cs", "cfl", "rho_ref", "u_ref", "h_ref", "kf", "ic_kind", "ic_amp", "force_seed"):
        setattr(f, k, getattr(coarse, k))
    f.tau = 0.0
    f.nu = phys(coarse)["nu"]
    ratio = phys(coarse)["dt"] / phys(f)["dt"]
    f.fkf = coarse.fkf * np.sqrt(ratio)
    f.friction_rate = coarse.friction_rate / ratio
    return f


def feq_populations(rho, u, v, c: float) -> np.ndarray:
    """Equilibrium populations [9][ny][nx] of (rho, u, v) (lbm.h:31-39)."""
    rho, u, v = (np.asarray(a, np.float64) for a in (rho, u, v))
    uu = (u * u + v * v) / (c * c)
    f = np.empty((Q,) + u.shape)
    for q in range(Q):
        uc = (EX[q] * u + EY[q] * v) / c
        f[q] = rho * W[q] * (1 + 3 * uc + 4.5 * uc * uc - 1.5 * uu)
    return f.astype(np.float32)


def box(a, f: int) -> np.ndarray:
    ny, nx = a.shape
    return np.asarray(a, np.float64).reshape(ny // f, f, nx // f, f).mean(axis=(1, 3))


def save_params(path: str, params, meta: dict):
    np.savez(path, params=np.asarray(params, np.float32), meta=json.dumps(meta))


def load_params(path: str = DEFAULT_PARAMS):
    """(params [1313] float32, metadata dict) of a saved closure."""
    with np.load(path) as z:
        return z["params"].astype(np.float32), json.loads(str(z["meta"]))


def _mem_available() -> int:
    try:
        for line in open("/proc/meminfo"):
            if line.startswith("MemAvailable:"):
                return int(line.split()[1]) * 1024
    except OSError:
        pass
    return 1 << 62


def train(coarse=None, filter: int = 8, members: int = 64, snapshots: int = 64, spinup: int = 20000,
          spacing: int = 800, iters=(6000, 3000, 3000), lrs=(2e-3, 7e-4, 2e-4), batch: int = 65536, seed: int = 1,
          device: int = 0, log=print):
    """Generate the box-filtered training set and train the closure on the GPU.
    Returns (params, report)."""
    coarse = coarse if coarse is not None else coarse_config()
    fine = fine_config(coarse, filter, members)
    nc = (fine.nx // filter) * (fine.ny // filter)
    need = 2.5 * 28 * nc * members * snapshots
    if need > _mem_available():
        snapshots = max(4, int(snapshots * _mem_available() / need))
        log(f"host memory: snapshots per member reduced to {snapshots}")
    t0 = time.time()
    feat, tgt = lbl.closure_generate(fine, filter, spinup, snapshots, spacing, device)
    t_gen = time.time() - t0
    log(f"generated {len(tgt)} samples ({members * snapshots} snapshots of {fine.nx}^2 filtered {filter}x) "
        f"in {t_gen:.1f} s; target mean {tgt.mean():.3f} sd {tgt.std():.3f}")
    rng = np.random.default_rng(seed)
    # hold out whole snapshots: consecutive cells are correlated
    snap = np.arange(len(tgt)) // nc
    val_snaps = rng.choice(members * snapshots, max(1, members * snapshots // 10), replace=False)
    is_val = np.isin(snap, val_snaps)
    tr, va = np.flatnonzero(~is_val), np.flatnonzero(is_val)
    ftr, ttr = np.ascontiguousarray(feat[tr]), np.ascontiguousarray(tgt[tr])
    w, curves = None, []
    t0 = time.time()
    for k, (n_it, lr) in enumerate(zip(iters, lrs)):
        w, curve = lbl.closure_train(ftr, ttr, n_it, batch, lr, seed + k, device, init=w)
        curves.append(curve)
        log(f"stage {k}: lr {lr:g}, {n_it} iterations, minibatch loss {curve[:20].mean():.4f} -> "
            f"{curve[-50:].mean():.4f}")
    t_train = time.time() - t0
    m_va = lbl.closure_infer(w, feat[va], 0, device)
    t_va = tgt[va].astype(np.float64)
    rep = {
        "fine_grid": fine.nx, "filter": filter, "members": members, "snapshots_per_member": snapshots,
        "snapshots": members * snapshots, "samples": int(len(tgt)), "spinup_steps": spinup,
        "spacing_steps": spacing, "fine_nu": fine.nu, "fine_tau": 0.5 + 3 * fine.nu / (phys(fine)["c"] * phys(fine)["dx"]),
        "generate_s": t_gen, "train_s": t_train, "iters": list(iters), "lrs": list(lrs), "batch": batch,
        "target_mean": float(tgt.mean()), "target_sd": float(tgt.std()),
        "val_samples": int(len(va)),
        "val_mse_mlp": float(np.mean((m_va - t_va) ** 2)),
        "val_mse_smagorinsky": float(np.mean((1.0 - t_va) ** 2)),
        "val_mse_best_constant": float(np.var(t_va)),
        "val_corr": float(np.corrcoef(m_va, t_va)[0, 1]),
        "loss_curve": [float(c) for c in np.concatenate(curves)[::50]],
        "nu_ref": phys(fine)["nu"], "dx_ref": float(coarse.h_ref / 255.0),
    }
    log(f"validation MSE: MLP {rep['val_mse_mlp']:.4f}, Smagorinsky (m=1) {rep['val_mse_smagorinsky']:.4f}, "
        f"best constant {rep['val_mse_best_constant']:.4f}; corr {rep['val_corr']:.3f}")
    return w, rep


def spectrum_error(e_run, e_ref, kmax: int) -> float:
    """Mean |log10(E_run / E_ref)| over shells 1..kmax."""
    k = np.arange(1, kmax + 1)
    return float(np.mean(np.abs(np.log10(np.maximum(e_run[k], 1e-300) / np.maximum(e_ref[k], 1e-300)))))


def evaluate(params=None, meta=None, filter: int = 8, spinup: int = 20000, cycles: int = 100, members: int = 16,
             spectrum_every: int = 5, seed: int = 0, device: int = 0, log=print, refresh: int = 1):
    """The closure against plain Smagorinsky in the coarse configuration, with the
    box-filtered fine run as the truth (an imperfect-model experiment: neither coarse
    model represents the truth exactly).

    * analysis RMSE: two DA_LETKF ensembles (members, 256^2) started from the filtered
      truth plus 10 % random-phase perturbations; every 100 coarse steps both
      assimilate the same noisy observations of the filtered truth (u, v, rho every
      4th point, sigma 0.1 / 0.01) and the RMSE of the analysis mean against the
      filtered truth is recorded;
    * spectrum: two free coarse runs from the filtered truth; their energy spectra
      and the filtered truth's, averaged over the run, and the mean |log10| error.
    refresh: the network runs every `refresh` steps and each cell's multiplier is held
    between (lbl_set_closure_refresh).  Returns the report dict."""
    if params is None:
        params, meta = load_params()
    coarse = coarse_config(n_ens=members)
    fine = fine_config(coarse, filter, 1)
    ratio = phys(coarse)["dt"] / phys(fine)["dt"]
    nat = lbl.Ensemble(fine, device)
    nat.init(0)
    nat.update(0, spinup)
    tf, done_f = spinup, 0

    def truth():
        r, u, v, _ = nat.get_fields(0)
        return box(r, filter).astype(np.float32), box(u, filter).astype(np.float32), box(v, filter).astype(np.float32)

    rt, ut, vt = truth()
    c = phys(coarse)["c"]
    pert = lbl.Ensemble(lbl.config_default("NATURE", coarse.nx, members, ic_kind=coarse.ic_kind, ic_amp=coarse.ic_amp),
                        device)
    pert.init(1000)
    dvel = [pert.get_fields(m)[1:3] for m in range(members)]
    pert.close()
    setups = (("smagorinsky", None), ("mlp", params))
    da, free = {}, {}
    for name, w in setups:
        e = lbl.Ensemble(coarse, device)
        e.init(0)
        f1 = lbl.Ensemble(coarse_config(n_ens=1, mode="NATURE"), device)
        f1.init(0)
        if w is not None:
            e.set_closure(w, meta["nu_ref"], meta["dx_ref"])
            f1.set_closure(w, meta["nu_ref"], meta["dx_ref"])
            e.set_closure_refresh(refresh)
            f1.set_closure_refresh(refresh)
        for m in range(members):
            e.set_f(m, feq_populations(rt, ut + coarse.ens_perturb * dvel[m][0], vt + coarse.ens_perturb * dvel[m][1], c))
        f1.set_f(0, feq_populations(rt, ut, vt, c))
        da[name], free[name] = e, f1
    rng = np.random.default_rng(seed)
    rmse = {n: [] for n, _ in setups}
    spec = {n: [] for n in ["truth"] + [n for n, _ in setups]}
    t0 = time.time()
    for cyc in range(cycles):
        n_f = int(round((cyc + 1) * 100 * ratio)) - done_f  # fine steps for 100 coarse steps
        nat.update(tf, n_f)
        tf += n_f
        done_f += n_f
        rt, ut, vt = truth()
        ro = rt + rng.normal(0, coarse.obs_error_rho, rt.shape).astype(np.float32)
        uo = ut + rng.normal(0, coarse.obs_error_u, ut.shape).astype(np.float32)
        vo = vt + rng.normal(0, coarse.obs_error_u, vt.shape).astype(np.float32)
        t = cyc * 100
        for name, _ in setups:
            da[name].update(t, 100)
            da[name].assimilate(t + 100, ro, uo, vo)
            rmse[name].append(da[name].rmse_uv(ut, vt))
            free[name].update(t, 100)
        if (cyc + 1) % spectrum_every == 0:
            spec["truth"].append(lbl.energy_spectrum(ut, vt))
            for name, _ in setups:
                _, u, v, _ = free[name].get_fields(0)
                spec[name].append(lbl.energy_spectrum(u, v))
    wall = time.time() - t0
    half = cycles // 2
    es = {n: np.mean(v, axis=0) for n, v in spec.items()}
    kq, kh = coarse.nx // 4, coarse.nx // 2 - 1
    rep = {
        "cycles": cycles, "members": members, "fine_grid": fine.nx, "filter": filter, "spinup_fine_steps": spinup,
        "closure_refresh_steps": refresh,
        "dt_ratio": ratio, "wall_s": wall,
        "rmse_mean_second_half": {n: float(np.mean(v[half:])) for n, v in rmse.items()},
        "rmse_final": {n: float(v[-1]) for n, v in rmse.items()},
        "rmse_series": {n: [float(x) for x in v] for n, v in rmse.items()},
        f"spectrum_error_k1_to_{kq}": {n: spectrum_error(es[n], es["truth"], kq) for n, _ in setups},
        f"spectrum_error_k1_to_{kh}": {n: spectrum_error(es[n], es["truth"], kh) for n, _ in setups},
        "spectra": {n: [float(x) for x in v] for n, v in es.items()},
    }
    for d in (da, free):
        for e in d.values():
            e.close()
    nat.close()
    log(json.dumps({k: v for k, v in rep.items() if k not in ("rmse_series", "spectra")}))
    return rep


def _cli_eval(a):
    w, meta = load_params(a.params)
    rep = evaluate(w, meta, filter=meta.get("filter", 8), spinup=a.spinup, cycles=a.cycles, members=a.members,
                   refresh=a.refresh)
    if a.out:
        with open(a.out, "w") as f:
            json.dump(rep, f, indent=1)


def _cli_train(a):
    w, rep = train(filter=a.filter, members=a.members, snapshots=a.snapshots, spinup=a.spinup, spacing=a.spacing,
                   iters=tuple(a.iters), lrs=tuple(a.lrs), batch=a.batch, seed=a.seed)
    save_params(a.out, w, rep)
    print(json.dumps({k: v for k, v in rep.items() if k != "loss_curve"}))


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    sub = ap.add_subparsers(dest="cmd", required=True)
    t = sub.add_parser("train", help="generate box-filtered data and train the closure")
    t.add_argument("--filter", type=int, default=8)
    t.add_argument("--members", type=int, default=64)
    t.add_argument("--snapshots", type=int, default=64, help="snapshots per member")
    t.add_argument("--spinup", type=int, default=20000, help="fine steps before the first snapshot")
    t.add_argument("--spacing", type=int, default=800, help="fine steps between snapshots")
    t.add_argument("--iters", type=int, nargs="+", default=[6000, 3000, 3000])
    t.add_argument("--lrs", type=float, nargs="+", default=[2e-3, 7e-4, 2e-4])
    t.add_argument("--batch", type=int, default=65536)
    t.add_argument("--seed", type=int, default=1)
    t.add_argument("--out", default=DEFAULT_PARAMS)
    e = sub.add_parser("eval", help="closure vs Smagorinsky: analysis RMSE and spectrum against filtered truth")
    e.add_argument("--params", default=DEFAULT_PARAMS)
    e.add_argument("--spinup", type=int, default=20000)
    e.add_argument("--cycles", type=int, default=100)
    e.add_argument("--members", type=int, default=16)
    e.add_argument("--refresh", type=int, default=1,
                   help="run the network every this many steps and hold the multipliers between")
    e.add_argument("--out", default=None, help="write the full report (series, spectra) as JSON")
    a = ap.parse_args()
    if a.cmd == "train":
        _cli_train(a)
    else:
        _cli_eval(a)


if __name__ == "__main__":
    main()
