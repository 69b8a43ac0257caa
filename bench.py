#!/usr/bin/env python
"""bench.py -- DA cycles/s of the LBM2D-LETKF forecast-and-assimilate cycle on B200.

Workload (the DA_LETKF OSSE at M=16, 256^2): 16 members resident on one GPU, D2Q9
BGK + Smagorinsky (Cs 0.1, tau 0.51), forcing as config.h (kf 4, fkf 5.6), IC
E(k) ~ k^4 exp(-2 (k/4)^2) at rms 0.05 lattice (1.0 physical), ensemble = nature IC
+ 10% random-phase perturbations; observations (u, v, rho) every 4th point
(4,096 sites) with sigma_u = 0.1 x rms velocity; Gaspari-Cohn R-localisation over
a 4-cell radius (DA_XYPRUNE=4, LETKF_RLOC_LEN=1, 75 observations per point);
inflation 1.1; one analysis every 100 steps (DAPRUNE=5 x iiter=20).

One bench "step" = one DA cycle = the LETKF analysis + 100 LBM steps.

  value     cycles/s with the observations already resident on the device
            (lbl_cycle_async with NULL observation pointers), device time from
            CUDA events on the engine's stream, max over ranks
  e2e       the same through the public C ABI with host buffers every cycle:
            observation fields from pinned host arrays (compacted into pinned staging, H2D),
            cycle graph, and the forecast RMSE of the ensemble-mean velocity
            against the nature run read back (lbl_rmse_uv)
  roofline  the fused stream-collide kernel (the dominant kernel): 72 B per
            lattice update (9 float loads + 9 float stores) x M*nx*ny per launch
            / the average launch time from CUDA events (lbl_profile_step)
  cpu_baseline  the FP64 OpenMP oracle on this host's cores, bounded sample
  analysis_roofline  the LETKF analysis phase against the nominal FP32 SIMT peak
            (algorithmic flops per grid point: Gram 2 n_obs M^2, transform
            2*9*M^2 + 4 M^3, Jacobi 18 M M(M-1)/2 per sweep)

  roofline_hbm, c2_cycles_per_s, c4_cycles_per_s  (default C1 line on one GPU)
            two side legs timed the same way: C2 (512^2 x 64, 604 MB population
            buffers, so the stream-collide launches inside its cycles are
            HBM-bound) and C4 (C1 with the learned closure)

`--impl reference` is the reference arm.  At the C1 shape it runs the reference's
own code on this GPU (oracle/_ref/ref_osse_p4r1, built from the reference's sources
here): one step is one whole DA cycle, its LBM (src/lbm.cu, src/data.cu, unmodified)
for the 16 members x 100 steps and its LETKF call sequence (letkf.cu glue and
letkf_solver.h's cuBLAS / cuSOLVER calls, restated because those two files need MPI
and HDF5), as one process.  The reference has no CPU implementation; the FP64 OpenMP
restatement of its path in oracle/ on the host cores is the line's cpu_baseline
(configured by the oracle's own restatement of config.h: the product library is
never loaded in that arm), and the value where the reference's build cannot serve the
workload.  The line also carries `reference_build`: the reference's forecast alone run
as M processes sharing the GPU, one per member as its one-MPI-rank-per-member runs
do, and the cycles/s bound it implies (`reference_build_bound_cycles_per_s`).

Multi-GPU: by default replicas (one independent experiment per GPU, no collective on
the data path); `value` is the cycles of all ranks / the slowest rank's time.
`--shard slab` instead splits the workload's one experiment into y-bands, one per GPU
(lbl.slab: all members of a band of rows per GPU, halo rows exchanged by NCCL send /
receive); its value is that one experiment's cycles/s ("scaling": "strong").
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "lbm2d-letkf_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

NX = 256
M = 16
STEPS_PER_CYCLE = 100
P_OBS = 4
METRIC = "DA cycles/s"
UNIT = "cycles/s"
WORKLOADS = {
    "C1": (256, 16, "DA_LETKF OSSE, M=16 members resident on 1 GPU, 256x256 D2Q9 BGK+Smagorinsky (Cs 0.1, tau 0.51), "
                    "obs (u,v,rho) every 4th point (4096 sites), GC localisation radius 4 cells (75 obs/point), "
                    "inflation 1.1, 100 LBM steps + 1 LETKF analysis per cycle, FP32"),
    "C2": (512, 64, "DA_LETKF OSSE, M=64 members resident on 1 GPU, 512x512 D2Q9 BGK+Smagorinsky (Cs 0.1, tau 0.51), "
                    "obs (u,v,rho) every 4th point (16384 sites), GC localisation radius 4 cells (75 obs/point), "
                    "inflation 1.1, 100 LBM steps + 1 LETKF analysis per cycle, FP32 storage"),
    "C4": (256, 16, "DA_LETKF OSSE as C1 (M=16, 256x256, obs every 4th point, GC radius 4, inflation 1.1, 100 steps + "
                    "1 analysis per cycle, FP32) with the learned closure in the stream-collide: nu_t = m (Cs dx)^2 |S|, "
                    "m from a 6-32-32-1 GELU/softplus MLP (BF16 parameters, FP16 tensor-core operands, FP32 sums) "
                    "trained on 4096 8x-box-filtered 2048^2 snapshots; nature run plain Smagorinsky"),
}
CLOSURE = False  # the ensemble (and the CPU baselines) use the trained closure (workload C4)
CLOSURE_REFRESH = 20  # the closure's network runs every this many steps (lbl_set_closure_refresh)
WORKLOAD = WORKLOADS["C1"][2]


STORAGE = 0  # lbl_config.storage of the ensemble (the nature run stays FP32)
GRAM = 0     # lbl_config.gram of the ensemble: 0 FP32, 1 BF16 tensor cores (32 < M <= 64)
LBM_VARIANT = 0  # lbl_config.lbm_variant of the ensemble and the nature run (0: the library's choice)
PREFETCH = None  # the stream-collide's march form (lbl_set_stream_collide_shape), None: the library's choice


def workload_config(lib, mode="DA_LETKF", n_ens=None):
    """The workload's lbl_config; `lib` is the product package (lbl) or, for the CPU
    reference arm, the oracle module, which has its own restatement of config.h."""
    return lib.config_default(
        mode, NX, M if n_ens is None else n_ens, da_xyprune=P_OBS, letkf_rloc_len=1, letkf_covinf=1.1, obs_error_u=0.1,
        obs_error_rho=0.01, iiter=20, daprune=5, cs=0.1, tau=0.51, ic_kind=lib.IC_K4EXP, ic_amp=1.0,
        ens_init=lib.ENS_PERTURBED, ens_perturb=0.1, storage=STORAGE if mode != "NATURE" else 0,
        gram=GRAM if mode == "DA_LETKF" else 0, lbm_variant=LBM_VARIANT)


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def stream_collide_kernel(ens):
    """The stream-collide kernel the context runs and its launch shape."""
    shape = ens.launch_shape()
    if CLOSURE:
        return "lbm_step_kernel_closure", shape
    return ("lbm_step_vec_kernel" if shape["columns_per_thread"] > 1 else "lbm_step_kernel"), shape


def ncu_traffic(kernel, nx=None, m=None, storage=None):
    """DRAM bytes per stream-collide launch from the committed ncu summary
    profiles/<kernel>[_f16]_<nx>x<nx>_M<m>.md, if there is one."""
    nx = NX if nx is None else nx
    m = M if m is None else m
    storage = STORAGE if storage is None else storage
    path = os.path.join(ROOT, "profiles", f"{kernel}{'_f16' if storage else ''}_{nx}x{nx}_M{m}.md")
    try:
        for line in open(path):
            if line.startswith("traffic_bytes_per_launch:"):
                return float(line.split(":")[1])
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi clock/throttle samples while the timed region runs."""

    QUERY = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc:
            time.sleep(0.15)
            self.proc.terminate()
            out, _ = self.proc.communicate(timeout=10)
            self.lines = [l for l in out.strip().split("\n") if l.strip()]

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            p = [x.strip() for x in l.split(",")]
            try:
                sm.append(float(p[0]))
                mx.append(float(p[1]))
            except (ValueError, IndexError):
                continue
            for n, v in zip(names, p[4:8]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def make_observations(lbl, n_cycles, seed=2024):
    """Nature run (member id 0) and its observations at the end of every cycle."""
    nat = lbl.Ensemble(workload_config(lbl, "NATURE", 1))
    nat.init(0)
    rng = np.random.default_rng(seed)
    obs, truth = [], []
    nsite = np.ones((NX, NX), bool)
    nsite[::P_OBS, ::P_OBS] = False
    for _ in range(n_cycles):
        nat.update(0, STEPS_PER_CYCLE)
        r, u, v, _ = nat.get_fields(0)
        ro = (r + 0.01 * rng.standard_normal(r.shape)).astype(np.float32)
        uo = (u + 0.1 * rng.standard_normal(u.shape)).astype(np.float32)
        vo = (v + 0.1 * rng.standard_normal(v.shape)).astype(np.float32)
        for a in (ro, uo, vo):
            a[nsite] = np.nan
        obs.append((ro, uo, vo))
        truth.append((u.copy(), v.copy()))
    nat.close()
    return obs, truth


def cpu_baseline_sample(oracle, obs, threads=None):
    """Oracle (FP64, OpenMP, this host's cores) on a bounded sample of one cycle:
    4 LBM steps of the whole 16-member ensemble + the analysis of 16 of the 256 rows,
    scaled to a full cycle (25x the steps, 16x the rows)."""
    nthreads = oracle.set_threads(threads or os.cpu_count())
    o = with_closure(oracle.Oracle(workload_config(oracle)))
    o.init(0)
    rng = np.random.default_rng(5)
    o.step(1, rng.normal(0, 0.84, 4 * 29).astype(np.float32))  # warm caches / page in
    t0 = time.perf_counter()
    o.step(4, rng.normal(0, 0.84, 4 * 29 * 4).astype(np.float32))
    t_steps = time.perf_counter() - t0
    t0 = time.perf_counter()
    o.assimilate_rows(*obs, 120, 136)
    t_ana = time.perf_counter() - t0
    o.close()
    cycle = 25 * t_steps + 16 * t_ana
    return {"value": 1.0 / cycle, "unit": UNIT, "cores": nthreads, "kind": "port",
            "sample": "4 LBM steps of 16x256^2 + LETKF of 16/256 rows, scaled x25 / x16 to one cycle",
            "lbm_glups": 4 * M * NX * NX / t_steps / 1e9, "analysis_s_per_cycle": 16 * t_ana}


def init_dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws <= 1:
        return None, 0, 1, int(os.environ.get("LOCAL_RANK", "0"))
    import datetime
    import torch
    import torch.distributed as dist
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return dist, dist.get_rank(), ws, local


def reduce_max(dist, x, device):
    """Max of x over ranks (device None: a CPU tensor, for gloo)."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device="cpu" if device is None else f"cuda:{device}")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(world, cycles_per_rank, ms_max):
    """Whole-job cycles/s of `world` independent replicas timed by the slowest rank."""
    return world * cycles_per_rank / (ms_max / 1e3)


def barrier(dist):
    if dist is not None:
        dist.barrier()


def run_engine(args, dist, rank, world, device):
    import lbl
    import oracle
    K, W = args.steps, args.warmup
    obs, truth = make_observations(lbl, W + K + 1)
    ens = with_closure(with_shape(lbl.Ensemble(workload_config(lbl), device=device)))
    ens.init(0)
    T = STEPS_PER_CYCLE
    # first cycle has no analysis (t = 0): bring the ensemble to t = 100
    ens.cycle_async(0, None, None, None, T)
    ens.sync()

    # Timed cycles: the 16-member state (37.7 MB per population buffer) fits in the
    # 126 MB L2, so L2 is flushed (a 256 MB write) between timed cycles, outside the
    # timed intervals; each cycle is timed on the engine's stream with CUDA events.
    # The flush is enqueued on the engine's own stream (lbl_get_stream), ahead of the
    # cycle's start event: the host enqueues the cycle while the flush runs, so the
    # device-timed interval holds the cycle's work and copies, not the host's enqueue.
    import torch
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=f"cuda:{device}")

    def flush_l2_on(e):
        with torch.cuda.stream(torch.cuda.ExternalStream(e.stream(), device=f"cuda:{device}")):
            flush.zero_()

    # the e2e leg's host inputs (observation fields, and the nature fields its RMSE reads)
    # sit in pinned memory, as a caller streaming observations would hold them
    pins = []

    def pinned(a):
        t = torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).pin_memory()
        pins.append(t)
        return t.numpy()

    obs_h = [tuple(pinned(a) for a in o) for o in obs]
    truth_h = [tuple(pinned(a) for a in tr) for tr in truth]

    # ---- value: resident observations --------------------------------------------
    clk = ClockSampler(device).__enter__()  # sampled from warm-up to the end of the timed region
    ens.cycle_async(T, *obs[0], T)  # uploads the observations once
    for c in range(1, W):
        ens.cycle_async((c + 1) * T, None, None, None, T)
    ens.sync()
    torch.cuda.synchronize(device)
    barrier(dist)
    ms = ms_ana = ms_fc = 0.0
    for c in range(K):
        flush_l2_on(ens)
        ens.event_record(0)
        ens.cycle_async((W + c + 1) * T, None, None, None, T)
        ens.event_record(1)
        ms += ens.event_elapsed(0, 1)
        a, f = ens.cycle_phases()
        ms_ana += a
        ms_fc += f
    ens.sync()
    torch.cuda.synchronize(device)
    barrier(dist)
    clk.__exit__(None, None, None)
    ms_max = reduce_max(dist, ms, device)
    value = replica_value(world, K, ms_max)
    stats = ens.letkf_stats()

    # ---- e2e: host observations in, RMSE out, every cycle -----------------------------
    e2e_ens = with_closure(with_shape(lbl.Ensemble(workload_config(lbl), device=device)))
    e2e_ens.init(0)
    e2e_ens.cycle_async(0, None, None, None, T)
    for c in range(W):
        e2e_ens.cycle_async((c + 1) * T, *obs_h[c], T)
        e2e_ens.rmse_uv(*truth_h[c + 1])
    e2e_ens.sync()
    torch.cuda.synchronize(device)
    barrier(dist)
    rmse = []
    ms_e2e = 0.0
    res = torch.zeros(K, dtype=torch.float64).pin_memory()  # the RMSE of each cycle, read back by the host
    res_h = res.numpy()
    for i, c in enumerate(range(W, W + K)):
        flush_l2_on(e2e_ens)
        e2e_ens.event_record(0)
        e2e_ens.cycle_async((c + 1) * T, *obs_h[c], T)
        e2e_ens.rmse_uv_async(*truth_h[c + 1], res_h, i)
        e2e_ens.event_record(1)
        ms_e2e += e2e_ens.event_elapsed(0, 1)
        rmse.append(float(res_h[i]))
    torch.cuda.synchronize(device)
    barrier(dist)
    ms_e2e = reduce_max(dist, ms_e2e, device)
    e2e_value = replica_value(world, K, ms_e2e)
    nsites = (NX // P_OBS) ** 2
    h2d = 3 * nsites * 4 + 2 * NX * NX * 4 + 4 * T
    d2h = 8

    # ---- roofline of the stream-collide kernel, live in the timed cycles ----------------
    # the forecast phase of each cycle graph is T back-to-back stream-collide launches
    ms_step = ms_fc / (K * T)
    bytes_per_launch = (36.0 if STORAGE else 72.0) * M * NX * NX
    achieved = bytes_per_launch / (ms_step * 1e-3) / 1e9
    peak, peak_kind = measured_peak()
    kernel, shape = stream_collide_kernel(ens)
    traffic = ncu_traffic(kernel)
    ens.profile_step(20)
    ms_isolated = ens.profile_step(200)

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": ms_max / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": ("f16 storage, f32 compute" if STORAGE else "f32") + ("; closure f16 mma, f32 sums" if CLOSURE else ""),
        "data": "synthetic (seeded nature run + Gaussian observation noise)",
        "config": {"workload": WORKLOAD, "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
                   "l2": "flushed (256 MB write, on the engine's stream ahead of each cycle's start event) between "
                         "timed cycles, outside the timed intervals",
                   "observations": "value leg reuses the resident observations; e2e uploads them every cycle"},
        "glups": M * NX * NX * T * K * world / (ms_max / 1e3) / 1e9,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "forecast_rmse_uv_last": rmse[-1] if rmse else None},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "kernel": kernel, "shape": shape, "ms_per_launch": ms_step,
                     "algorithmic_bytes_per_launch": bytes_per_launch, "peak_kind": peak_kind,
                     "timed": "forecast phase of the timed cycles (in-graph events), 100 launches per cycle",
                     "ms_per_launch_back_to_back": ms_isolated,
                     "regime": ("L2-resident: the two population buffers (%.1f MB each) fit in the 126 MB L2, so this "
                                "is an L2-fed figure; roofline_hbm is the HBM-bound one" % (bytes_per_launch / 2e6))
                     if bytes_per_launch / 2 < 100e6 else "HBM-bound (population buffers larger than L2)"},
        "phases_ms_per_cycle": {"analysis_with_forcing_beside": ms_ana / K, "forecast": ms_fc / K},
        "analysis_roofline": analysis_roofline(stats, ms_ana / K),
        "gpu_launches": K * (T + 3),
        "letkf": stats,
        "clocks": clk.summary(),
    }
    ens.close()
    e2e_ens.close()
    if world == 1 and not args.no_side_legs and args.workload == "C1" and not STORAGE and not GRAM:
        c2 = side_leg(lbl, "C2", device, flush_l2_on)
        c4 = side_leg(lbl, "C4", device, flush_l2_on)
        line["c2_cycles_per_s"] = c2["cycles_per_s"]
        line["c4_cycles_per_s"] = c4["cycles_per_s"]
        line["c4_over_c1"] = c4["cycles_per_s"] / value
        line["roofline_hbm"] = c2.pop("roofline")
        line["c2"] = c2
        line["c4"] = c4
        line["gpu_launches"] += c2["gpu_launches"] + c4["gpu_launches"]
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_sample(oracle, obs[0])
    return line


def run_slab(args, dist, rank, world, device):
    """The workload's ONE experiment split into y-bands, one band per GPU (lbl.slab): every rank
    holds all members of ~NX/world rows plus 8 halo rows on each side, exchanges 8 rows with each
    neighbour (NCCL send / receive on the engine's stream) every 4 steps and after each analysis,
    and analyses its own rows.  The experiment is the same at every N ("scaling": "strong"); its
    cycles/s is the one experiment's, timed per cycle with CUDA events on each rank's engine
    stream, max over ranks.  One GPU is its own neighbour (the split's whole cost, no transfer)."""
    import lbl
    import torch
    from lbl import slab
    K, W = args.steps, args.warmup
    T = STEPS_PER_CYCLE
    obs, truth = make_observations(lbl, W + 2 * K + 1)
    group = dist.group.WORLD if dist is not None else None
    exp = slab.SlabExperiment(workload_config(lbl), world=world, group=group, device=device)
    band = exp.local[0].ens
    exp.init(0)
    exp.update(0, T)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=f"cuda:{device}")
    stream = torch.cuda.ExternalStream(band.stream(), device=f"cuda:{device}")

    def flush_l2():
        with torch.cuda.stream(stream):
            flush.zero_()

    clk = ClockSampler(device).__enter__()
    for c in range(W):
        exp.assimilate((c + 1) * T, *obs[c])
        exp.update((c + 1) * T, T)
    exp.sync()
    torch.cuda.synchronize(device)
    barrier(dist)

    def timed(c0, with_rmse):
        ms, rmse = 0.0, []
        for c in range(c0, c0 + K):
            flush_l2()
            band.event_record(0)
            exp.assimilate((c + 1) * T, *obs[c])
            exp.update((c + 1) * T, T)
            if with_rmse:
                rmse.append(exp.rmse_uv(*truth[c + 1]))
            band.event_record(1)
            ms += band.event_elapsed(0, 1)
        exp.sync()
        torch.cuda.synchronize(device)
        barrier(dist)
        return reduce_max(dist, ms, device), rmse

    ms, _ = timed(W, False)
    ms_e2e, rmse = timed(W + K, True)
    clk.__exit__(None, None, None)
    halo = exp.halo
    k = halo // 2
    segments = -(-T // exp.segment)  # forcing launches per cycle (lbl_slab_forecast_begin)
    chunks = sum(-(-min(exp.segment, T - i) // k) for i in range(0, T, exp.segment))
    nsites = (NX // P_OBS) ** 2
    line = {
        "metric": METRIC, "value": K / (ms / 1e3), "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": ms / K, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "f16 storage, f32 compute" if STORAGE else "f32",
        "data": "synthetic (seeded nature run + Gaussian observation noise)",
        "config": {"workload": WORKLOAD + f"; ONE experiment split in {world} y-bands",
                   "parallelism": f"y-slab x{world}", "bands": [list(b) for b in exp.bands], "halo_rows": halo,
                   "exchange": (f"{2 * k} rows per neighbour every {k} steps and {halo} after each analysis, "
                                + ("NCCL send / receive" if world > 1 else "the band is its own neighbour")),
                   "l2": "flushed (256 MB write on the engine's stream) between timed cycles, outside the timed "
                         "intervals",
                   "observations": "whole-grid host fields every cycle, each band uploads its rows"},
        "e2e": {"value": K / (ms_e2e / 1e3), "unit": UNIT,
                "h2d_bytes_per_step": 3 * nsites * 4 // world + 2 * NX * NX * 4 // world,
                "d2h_bytes_per_step": 8, "forecast_rmse_uv_last": rmse[-1] if rmse else None},
        # per cycle: forcing, the steps, a pack and an unpack per chunk, then the observation
        # operator, the analysis and the analysis' pack and unpack
        "gpu_launches": K * (segments + T + 2 * chunks + 4),
        "letkf": exp.letkf_stats(),
        "clocks": clk.summary(),
    }
    exp.close()
    return line


def side_leg(lbl, name, device, flush_l2_on, K=10, W=3):
    """One of the other single-GPU workloads, timed like the headline (CUDA events on
    the engine's stream around each cycle, L2 flushed between cycles, observations
    resident): C2 (512^2 x 64, whose 604 MB population buffers make the stream-collide
    HBM-bound; its in-cycle launches give roofline_hbm) or C4 (C1 with the learned
    closure).  Returns cycles/s, phases and, for C2, the stream-collide roofline."""
    global NX, M, CLOSURE, WORKLOAD
    saved = (NX, M, CLOSURE, WORKLOAD)
    NX, M, WORKLOAD = WORKLOADS[name]
    CLOSURE = name == "C4"
    if CLOSURE and CLOSURE_REFRESH > 1:
        WORKLOAD += f"; the network runs every {CLOSURE_REFRESH} steps, each cell's multiplier held between"
    T = STEPS_PER_CYCLE
    try:
        obs, _ = make_observations(lbl, 1)
        ens = with_closure(lbl.Ensemble(workload_config(lbl), device=device))
        ens.init(0)
        ens.cycle_async(0, None, None, None, T)
        ens.cycle_async(T, *obs[0], T)
        for c in range(1, W):
            ens.cycle_async((c + 1) * T, None, None, None, T)
        ens.sync()
        ms = ms_ana = ms_fc = 0.0
        with ClockSampler(device) as clk:
            for c in range(K):
                flush_l2_on(ens)
                ens.event_record(0)
                ens.cycle_async((W + c + 1) * T, None, None, None, T)
                ens.event_record(1)
                ms += ens.event_elapsed(0, 1)
                a, f = ens.cycle_phases()
                ms_ana += a
                ms_fc += f
        ens.sync()
        stats = ens.letkf_stats()
        out = {"workload": WORKLOAD, "cycles_per_s": K / (ms / 1e3), "ms_per_cycle": ms / K, "cycles": K,
               "warmup": W, "phases_ms_per_cycle": {"analysis_with_forcing_beside": ms_ana / K,
                                                    "forecast": ms_fc / K},
               "glups": M * NX * NX * T * K / (ms / 1e3) / 1e9, "letkf": stats, "clocks": clk.summary(),
               "gpu_launches": K * (T + 3)}
        if name == "C2":
            ms_step = ms_fc / (K * T)
            bpl = 72.0 * M * NX * NX
            achieved = bpl / (ms_step * 1e-3) / 1e9
            peak, peak_kind = measured_peak()
            kernel, shape = stream_collide_kernel(ens)
            out["roofline"] = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                               "frac": achieved / peak, "traffic": ncu_traffic(kernel, NX, M, 0),
                               "kernel": kernel, "shape": shape, "grid": f"{NX}x{NX}", "members": M,
                               "ms_per_launch": ms_step, "algorithmic_bytes_per_launch": bpl, "peak_kind": peak_kind,
                               "timed": "forecast phase of the C2 cycles (in-graph events), 100 launches per cycle",
                               "regime": "HBM-bound: two 604 MB population buffers, far larger than the 126 MB L2"}
        ens.close()
        return out
    finally:
        NX, M, CLOSURE, WORKLOAD = saved


def reference_build_forecast(n_proc, nsteps, warmup=50, exe=None):
    """The reference's own LBM (oracle/_ref/ref_lbm, or `exe` speaking its `time`
    protocol) run as n_proc processes sharing the GPU, one ensemble member each,
    started together after their warm-up.  Returns the forecast rate, or
    {"unavailable": why}."""
    import tempfile
    exe = exe or os.path.join(ROOT, "oracle", "_ref", "ref_lbm")
    if not os.path.exists(exe):
        return {"unavailable": "oracle/_ref/ref_lbm not built (it needs the reference sources at build time)"}
    with tempfile.TemporaryDirectory() as tmp:
        go = os.path.join(tmp, "go")
        ready = [os.path.join(tmp, f"ready{k}") for k in range(n_proc)]
        procs = [subprocess.Popen([exe, "time", str(k), str(nsteps), str(warmup), ready[k], go],
                                  stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True) for k in range(n_proc)]

        def stop(why):
            for p in procs:
                if p.poll() is None:
                    p.kill()
            for p in procs:
                p.wait()
            return {"unavailable": why}

        deadline = time.time() + 240
        while not all(os.path.exists(r) for r in ready):
            done = [p for p in procs if p.poll() is not None]
            if done:
                err = done[0].stderr.read().strip().splitlines()
                return stop(f"ref_lbm exited {done[0].returncode}: {err[-1] if err else ''}")
            if time.time() > deadline:
                return stop("ref_lbm processes not ready within 240 s")
            time.sleep(0.005)
        open(go, "w").close()
        spans = []
        for p in procs:
            try:
                out, err = p.communicate(timeout=240)
            except subprocess.TimeoutExpired:
                return stop("ref_lbm timed steps did not end within 240 s")
            rec = [ln.split() for ln in out.splitlines() if ln.startswith("ref_lbm_time")]
            if p.returncode != 0 or not rec:
                return stop(f"ref_lbm exited {p.returncode}: {err.strip()[-200:]}")
            spans.append((int(rec[0][3]), int(rec[0][4])))
    t0 = min(a for a, _ in spans)
    t1 = max(b for _, b in spans)
    sec = (t1 - t0) * 1e-9
    nxy = 256 * 256  # the reference's compiled default grid
    return {"processes": n_proc, "steps_per_process": nsteps, "seconds": sec,
            "ms_per_100_steps": 1e3 * sec * 100 / nsteps, "forecast_glups": n_proc * nxy * nsteps / sec * 1e-9}


def reference_build_line(args):
    """`reference_build` of the reference arm's JSON line (see the module docstring)."""
    nsteps = min(2000, max(200, 20 * args.steps))
    solo = reference_build_forecast(1, nsteps)
    if "unavailable" in solo:
        return solo
    shared = reference_build_forecast(M, nsteps)
    if "unavailable" in shared:
        return shared
    # the better of the two ways to run M members: M processes sharing the GPU, or
    # one process M times over (the single-process time x M, no context switches)
    best = min(shared["ms_per_100_steps"], solo["ms_per_100_steps"] * M)
    return {"kind": "the reference's src/lbm.cu + src/data.cu compiled unmodified (sm_100a, its nvcc flags), "
                    "its update() per step: forcing, streaming + macros, LES, collision",
            "grid": "256x256 (its compiled default; the cost per step does not depend on the flow)",
            "members": M, "shared": shared, "single_process": solo,
            "forecast_ms_per_cycle": best,
            "cycles_per_s_upper_bound": 1e3 / best,
            "note": "forecast only: the reference's LETKF analysis (MPI, HDF5, cuSOLVER) is not built here, "
                    "so its cycles/s is below this bound"}


def reference_osse_cycle(cycles=5, warmup=2, exe=None):
    """The reference's own whole DA cycle on this GPU (oracle/_ref/ref_osse_p4r1 time ...):
    its update() for the M members in turn, then its LETKF call sequence (letkf.cu glue,
    letkf_solver.h's cuBLAS / cuSOLVER calls, ranks in turn) with C1's DA settings, as one
    process; wall time of `cycles` cycles after `warmup`.  Returns its cycles/s, or
    {"unavailable": why}."""
    exe = exe or os.path.join(ROOT, "oracle", "_ref", "ref_osse_p4r1")
    if not os.path.exists(exe):
        return {"unavailable": "oracle/_ref/ref_osse_p4r1 not built (it needs the reference sources at build time)"}
    try:
        out = subprocess.run([exe, "time", str(M), str(cycles), str(STEPS_PER_CYCLE), str(warmup)],
                             capture_output=True, text=True, timeout=900, check=True).stdout
        sec = float(next(l for l in out.splitlines() if l.startswith("ref_osse_time")).split()[4])
    except Exception as e:  # no GPU, or the run failed
        return {"unavailable": f"ref_osse_p4r1 did not run: {type(e).__name__}"}
    return {"cycles_per_s": cycles / sec, "ms_per_cycle": 1e3 * sec / cycles, "cycles": cycles, "warmup": warmup,
            "kind": "the reference's src/lbm.cu + src/data.cu (unmodified) for the 16 members x 100 steps, then its "
                    "LETKF call sequence (oracle/ref_letkf_solver.cu: letkf.cu glue, letkf_solver.h cuBLAS/cuSOLVER "
                    "calls, syevjBatched) with DA_XYPRUNE 4, LETKF_RLOC_LEN 1, covinf 1.1, obs errors 0.1 / 0.01, "
                    "256x256; one process, members and ranks in turn (the reference spreads them over 16 MPI "
                    "processes); its compiled default physics (the cost does not depend on it)"}


def analysis_roofline(stats, ms_phase):
    """The LETKF analysis against the FP32 SIMT peak: algorithmic flops per grid point
    (Gram 2 n_obs M^2, transform 2*9*M^2 + 4 M^3, Jacobi 18 M M(M-1)/2 per sweep at the
    measured mean sweeps) over the analysis phase of the timed cycles, which also holds
    the observation operator and the forcing chunk beside it, so the fraction is a floor.
    The peak is nominal (148 SMs x 128 FP32 lanes x 2 flops x 1965 MHz): the measured
    peaks cover HBM and BF16 tensor cores only."""
    n_obs = 75  # 25 sites x 3 variables at LETKF_RLOC_LEN = 1, p = 4
    sweeps = float(stats.get("mean_sweeps") or 0.0)
    per_point = 2 * n_obs * M * M + 2 * 9 * M * M + 4 * M ** 3 + 18 * M * M * (M - 1) / 2 * sweeps
    flops = per_point * NX * NX
    achieved = flops / (ms_phase * 1e-3) / 1e12
    peak = 148 * 128 * 2 * 1.965e9 / 1e12
    return {"bound": "fp32 simt", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
            "peak_kind": "nominal", "flops_per_point": per_point, "mean_sweeps": sweeps,
            "timed": "analysis phase of the timed cycles (observation operator + analysis, forcing beside it)"}


def run_reference(args, rank, world):
    """The reference arm.  At the C1 shape (256^2, 16 members, plain Smagorinsky) it is
    the reference's own code on this GPU (oracle/_ref/ref_osse_p4r1, built from the
    reference's sources here): one step is one whole DA cycle, its LBM for the 16
    members x 100 steps and its LETKF call sequence; `steps` cycles timed after `warmup`.
    The reference has no CPU implementation; the FP64 OpenMP restatement of the path
    (oracle/) on the host cores is the cpu_baseline, timed on one cycle's work: one
    sample step is 100 LBM steps of one member plus the analysis of ny/M rows of the
    whole ensemble, the row slice moving, so M sample steps are one cycle.  Where the
    reference's build cannot serve the workload the port is the value.  No product
    library is loaded in this process."""
    import oracle
    if rank != 0:
        return None
    T = STEPS_PER_CYCLE
    nthreads = oracle.set_threads(os.cpu_count())
    fc = with_closure(oracle.Oracle(workload_config(oracle, n_ens=1)))   # one member's forecast
    fc.init(0)
    da = with_closure(oracle.Oracle(workload_config(oracle)))            # the ensemble the analysis reads
    da.init(0)
    rng = np.random.default_rng(9)
    obs_nan = np.full((NX, NX), np.nan, np.float32)
    ro, uo, vo = obs_nan.copy(), obs_nan.copy(), obs_nan.copy()
    ro[::P_OBS, ::P_OBS] = 1.0 + 0.01 * rng.standard_normal((NX // P_OBS, NX // P_OBS))
    uo[::P_OBS, ::P_OBS] = rng.standard_normal((NX // P_OBS, NX // P_OBS))
    vo[::P_OBS, ::P_OBS] = rng.standard_normal((NX // P_OBS, NX // P_OBS))
    rows = NX // M
    n_modes = 29  # forcing modes at kf = 4

    def one(k):
        j0 = (k % M) * rows
        t0 = time.perf_counter()
        fc.step(T, rng.normal(0, 0.84, 4 * n_modes * T).astype(np.float32))
        da.assimilate_rows(ro, uo, vo, j0, j0 + rows)
        return time.perf_counter() - t0

    gpu_ref = NX == 256 and M == 16 and not CLOSURE
    port_steps = M if gpu_ref else args.steps  # one whole cycle beside the GPU reference
    one(0)
    sec = [one(1 + k) for k in range(port_steps)]
    port_value = (port_steps / M) / sum(sec)
    fc.close()
    da.close()
    sample = (f"{port_steps} steps of 1/{M} of a cycle: {T} LBM steps of 1 of the {M} members + the LETKF analysis "
              f"of {rows} of the {NX} rows (moving slice; {M} steps = one whole cycle)")
    cpu = {"value": port_value, "unit": UNIT, "cores": nthreads, "kind": "port", "sample": sample,
           "backend": "FP64 OpenMP CPU restatement of the reference path (the reference has no CPU implementation)"}
    ref = reference_osse_cycle(cycles=args.steps, warmup=args.warmup) if gpu_ref else {
        "unavailable": "the reference's build serves 256x256, 16 members, plain Smagorinsky"}
    if "cycles_per_s" in ref:
        value, ms_step, steps, dtype = ref["cycles_per_s"], ref["ms_per_cycle"], args.steps, "f32"
        backend = ("the reference's own code on this GPU (oracle/_ref/ref_osse_p4r1): " + ref["kind"])
        step = "one step = one whole DA cycle (100 LBM steps of the 16 members + one LETKF analysis)"
    else:
        value, ms_step, steps, dtype = port_value, 1e3 * sum(sec) / port_steps, port_steps, "f64"
        backend, step = cpu["backend"], sample
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": dtype, "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD, "backend": backend, "step": step},
            "cpu_baseline": cpu,
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if gpu_ref:
        line["reference_build_cycle"] = ref
        rb = reference_build_line(args)
        line["reference_build"] = rb
        if "cycles_per_s_upper_bound" in rb:
            line["reference_build_bound_cycles_per_s"] = rb["cycles_per_s_upper_bound"]
            line["reference_build_bound_kind"] = (
                "forecast-only upper bound on the reference build's DA cycles/s on this GPU: its own LBM "
                "(src/lbm.cu + src/data.cu, unmodified) for the 16 members x 100 steps as 16 processes or one")
    else:
        line["reference_build"] = {"unavailable": ref["unavailable"]}
    return line


def profile_cycles(args):
    """The workload's cycles only (no timing, no baseline): a clean launch list for ncu."""
    import lbl
    obs, _ = make_observations(lbl, 1)
    ens = with_closure(lbl.Ensemble(workload_config(lbl)))
    ens.init(0)
    T = STEPS_PER_CYCLE
    ens.cycle_async(0, None, None, None, T)
    ens.cycle_async(T, *obs[0], T)
    for c in range(args.warmup + args.steps):
        ens.cycle_async((c + 2) * T, None, None, None, T)
    ens.sync()
    print("profile cycles done:", ens.letkf_stats())
    ens.close()


# The batched form: 8 concurrent independent OSSEs of uneven grid and ensemble sizes
C3_EXPERIMENTS = [(128, 4), (128, 8), (256, 16), (256, 16), (256, 32), (512, 32), (512, 64), (1024, 64)]


def run_batch_graph(args):
    """C3 as one batch (lbl_batch): per cycle one CUDA graph with every experiment's
    analysis and forcing on parallel branches, then each of the 100 steps as one
    launch of the batched persistent stream-collide over all 8 experiments.  The strip
    height is picked by timing candidate heights on two cycles each.  Device time:
    events on the first context's stream, which follows the batch's graphs."""
    global NX, M
    import lbl
    T = STEPS_PER_CYCLE
    K, W = args.steps, args.warmup
    ens, obs = [], []
    for nx, m in C3_EXPERIMENTS:
        NX, M = nx, m
        o, _ = make_observations(lbl, 1)
        e = lbl.Ensemble(workload_config(lbl))
        e.init(0)
        ens.append(e)
        obs.append(o[0])
    t = 0
    tuning = {}
    for sr in (8, 12, 16, 24, 32):
        b = lbl.Batch(ens, sr)
        b.cycle_async(t, obs, T)
        t += T
        for _ in range(2):  # both buffer parities have their graphs
            b.cycle_async(t, None, T)
            t += T
        b.sync()
        ens[0].event_record(0)
        for _ in range(2):
            b.cycle_async(t, None, T)
            t += T
        ens[0].event_record(1)
        b.sync()
        tuning[sr] = ens[0].event_elapsed(0, 1) / 2
        b.close()
    best = min(tuning, key=tuning.get)
    b = lbl.Batch(ens, best)
    b.cycle_async(t, obs, T)
    t += T
    for _ in range(W):
        b.cycle_async(t, None, T)
        t += T
    b.sync()
    ens[0].event_record(0)
    for _ in range(K):
        b.cycle_async(t, None, T)
        t += T
    ens[0].event_record(1)
    b.sync()
    ms = ens[0].event_elapsed(0, 1)
    lu = sum(m * nx ** 2 for nx, m in C3_EXPERIMENTS) * T * K
    line = {"metric": "experiment DA cycles/s (C3 batch)", "value": len(ens) * K / (ms / 1e3), "unit": "cycles/s",
            "n_gpus": 1, "steps": K, "warmup": W, "ms_per_step": ms / K, "higher_is_better": True,
            "dtype": "f32", "data": "synthetic (seeded nature runs + Gaussian observation noise)",
            "config": {"workload": "C3: 8 DA_LETKF OSSEs in one batch, (grid, M) = " +
                       ", ".join(f"{nx}^2 x {m}" for nx, m in C3_EXPERIMENTS) +
                       ", obs every 4th point, GC radius 4 cells, inflation 1.1, 100 LBM steps + 1 analysis per cycle",
                       "concurrency": "one graph per batch cycle: analyses and forcing on parallel branches, one "
                                      "batched persistent stream-collide launch per step for all experiments"},
            "glups": lu / (ms / 1e3) / 1e9,
            "strip_rows": best, "autotune_ms_per_cycle": tuning, "gpu_launches": K * (T + 1 + 3 * len(ens))}
    b.close()
    for e in ens:
        e.close()
    return line


def run_batch(args):
    """C3 as concurrent contexts: every experiment is its own context (own stream,
    cycle graphs, autotuned strip height); their cycles are issued round-robin and run
    concurrently on the GPU.  Device time: each context records events around the
    timed cycles after a full synchronisation, so all start together; the batch time
    is the longest span."""
    global NX, M
    import lbl
    T = STEPS_PER_CYCLE
    K, W = args.steps, args.warmup
    exps = []
    for nx, m in C3_EXPERIMENTS:
        NX, M = nx, m
        obs, _ = make_observations(lbl, 1)
        e = lbl.Ensemble(workload_config(lbl))
        ty, ms_tuned = e.autotune()
        e.init(0)
        e.cycle_async(0, None, None, None, T)
        e.cycle_async(T, *obs[0], T)  # observations resident from here on
        exps.append({"nx": nx, "M": m, "ens": e, "strip_rows": ty, "ms_per_lbm_launch_tuned": ms_tuned,
                     "shape": e.launch_shape()})
    for c in range(W):
        for x in exps:
            x["ens"].cycle_async((c + 2) * T, None, None, None, T)
    for x in exps:
        x["ens"].sync()
    for x in exps:
        x["ens"].event_record(0)
    for c in range(K):
        for x in exps:
            x["ens"].cycle_async((W + c + 2) * T, None, None, None, T)
    spans = []
    for x in exps:
        x["ens"].event_record(1)
        spans.append(x["ens"].event_elapsed(0, 1))
        x["ens"].sync()
    ms = max(spans)
    lu = sum(x["M"] * x["nx"] ** 2 for x in exps) * T * K
    line = {"metric": "experiment DA cycles/s (C3 batch)", "value": len(exps) * K / (ms / 1e3), "unit": "cycles/s",
            "n_gpus": 1, "steps": K, "warmup": W, "ms_per_step": ms / K, "higher_is_better": True,
            "dtype": "f32", "data": "synthetic (seeded nature runs + Gaussian observation noise)",
            "config": {"workload": "C3: 8 concurrent DA_LETKF OSSEs, (grid, M) = " +
                       ", ".join(f"{x['nx']}^2 x {x['M']}" for x in exps) +
                       ", obs every 4th point, GC radius 4 cells, inflation 1.1, 100 LBM steps + 1 analysis per cycle",
                       "concurrency": "one context, stream and per-cycle CUDA graph per experiment"},
            "glups": lu / (ms / 1e3) / 1e9,
            "experiments": [{"nx": x["nx"], "M": x["M"], "strip_rows": x["strip_rows"], "shape": x["shape"],
                             "ms_per_lbm_launch_tuned": x["ms_per_lbm_launch_tuned"],
                             "ms_per_cycle_in_batch": spans[i] / K} for i, x in enumerate(exps)]}
    for x in exps:
        x["ens"].close()
    return line


def closure_params():
    """(params, nu_ref, dx_ref) of the trained closure shipped with the package, read
    with numpy (the CPU reference arm must not import the product)."""
    with np.load(os.path.join(ROOT, "lbm2d-letkf_b200", "lbl", "closure_c4.npz")) as z:
        meta = json.loads(str(z["meta"]))
        return z["params"].astype(np.float32), meta["nu_ref"], meta["dx_ref"]


def with_shape(ens):
    """Apply --prefetch (the stream-collide's march form) to an engine context."""
    if PREFETCH is not None:
        ens.set_launch_shape(PREFETCH, 0)
    return ens


def with_closure(obj):
    """Switch an engine ensemble or an oracle to the trained closure when the workload
    asks for it (the engine with its refresh interval; the oracle evaluates every step)."""
    if CLOSURE:
        obj.set_closure(*closure_params())
        if CLOSURE_REFRESH > 1 and hasattr(obj, "set_closure_refresh"):
            obj.set_closure_refresh(CLOSURE_REFRESH)
    return obj


def lbm_sweep(args):
    """Stream-collide alone at the given grids (NXxM,...): back-to-back launches on the
    engine's stream, CUDA events, one JSON line per size.  Sizes whose population
    buffers exceed the 126 MB L2 measure the HBM-bound regime."""
    import lbl
    for spec in args.lbm.split(","):
        nx, m = (int(v) for v in spec.lower().split("x"))
        e = lbl.Ensemble(lbl.config_default("NATURE", nx, m, storage=STORAGE, lbm_variant=LBM_VARIANT))
        tuned = e.autotune()[0] if args.autotune else None  # between creation and init
        if PREFETCH is not None:
            e.set_launch_shape(PREFETCH, 0)
        e.init(0)
        if args.closure:
            e.set_closure(*closure_params())
        e.update(0, 2)
        e.profile_step(max(3, args.warmup))
        ms = e.profile_step(max(1, args.steps))
        bytes_launch = (36.0 if STORAGE else 72.0) * m * nx * nx
        peak, peak_kind = measured_peak()
        gbs = bytes_launch / (ms * 1e-3) / 1e9
        print(json.dumps({"lbm_stream_collide": {
            "nx": nx, "ny": nx, "members": m, "storage": "f16 deviations" if STORAGE else "f32",
            "closure": "mlp" if args.closure else "smagorinsky", "lbm_variant": args.lbm_variant,
            "launches": args.steps, "ms_per_launch": ms,
            "glups": m * nx * nx / (ms * 1e-3) / 1e9, "algorithmic_bytes_per_launch": bytes_launch,
            "population_buffer_mb": bytes_launch / 2 / 1e6, "achieved_gbs": gbs, "peak_gbs": peak,
            "frac": gbs / peak, "peak_kind": peak_kind, "autotuned": tuned is not None, "shape": e.launch_shape()}}), flush=True)
        e.close()


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["engine", "reference"], default="engine")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-side-legs", action="store_true",
                    help="skip the C2 (HBM roofline) and C4 (learned closure) legs of the default C1 line")
    ap.add_argument("--profile", action="store_true",
                    help="run warmup + steps cycles of the workload and exit (for ncu captures)")
    ap.add_argument("--workload", choices=sorted(WORKLOADS) + ["C3"], default="C1",
                    help="C1 (the headline, 256^2 x 16), C2 (512^2 x 64), C3 (8 concurrent experiments) or C4 "
                         "(C1 with the learned closure)")
    ap.add_argument("--storage", choices=["f32", "f16"], default="f32",
                    help="population storage: f32, or the precision form's f16 deviations f - w_q")
    ap.add_argument("--c3", choices=["batch", "contexts"], default="batch",
                    help="C3 as one batch with a batched persistent stream-collide, or as concurrent contexts")
    ap.add_argument("--gram", choices=["f32", "bf16", "tf32x3"], default="f32",
                    help="the analysis Gram: FP32 SIMT, the precision form's BF16 mma.sync (M > 32, i.e. C2), or "
                         "the tcgen05 tensor-core block Gram with FP32 accuracy (3 x TF32)")
    ap.add_argument("--lbm", default=None, metavar="NXxM[,NXxM...]",
                    help="time the stream-collide alone at these grids and exit")
    ap.add_argument("--closure", action="store_true",
                    help="with --lbm: the learned-closure stream-collide (trained parameters of the package)")
    ap.add_argument("--autotune", action="store_true",
                    help="with --lbm: time at the strip height lbl_autotune picks instead of the heuristic's")
    ap.add_argument("--shard", choices=["replicas", "slab"], default="replicas",
                    help="N GPUs: independent experiments (replicas, the default) or the workload's one experiment "
                         "split in y-bands, one per GPU (slab; C1 / C2 shapes)")
    ap.add_argument("--prefetch", type=int, default=None, choices=[0, 1],
                    help="the stream-collide's march (lbl_set_stream_collide_shape): 0 pulls each row when "
                         "needed, 1 holds the row after next in registers; default: the library's choice")
    ap.add_argument("--lbm-variant", choices=["auto", "direct", "tma", "vec", "vec2"], default="auto",
                    help="stream-collide kernel: the library's choice, one column per thread, TMA-fed rows, or "
                         "4 (vec, 128-bit) / 2 (vec2, 64-bit) columns per thread")
    ap.add_argument("--closure-refresh", type=int, default=20,
                    help="C4: run the closure's network every this many steps, holding each cell's multiplier between "
                         "(1: every step)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    global NX, M, WORKLOAD, STORAGE, CLOSURE, GRAM, CLOSURE_REFRESH, LBM_VARIANT, PREFETCH
    NX, M, WORKLOAD = WORKLOADS.get(args.workload, WORKLOADS["C1"])
    CLOSURE = args.workload == "C4"
    CLOSURE_REFRESH = args.closure_refresh
    if CLOSURE and CLOSURE_REFRESH > 1:
        WORKLOAD += f"; the network runs every {CLOSURE_REFRESH} steps, each cell's multiplier held between"
    STORAGE = 1 if args.storage == "f16" else 0
    GRAM = {"f32": 0, "bf16": 1, "tf32x3": 2}[args.gram]
    LBM_VARIANT = {"auto": 0, "direct": 1, "tma": 2, "vec": 3, "vec2": 4}[args.lbm_variant]
    PREFETCH = args.prefetch
    if GRAM == 1:
        WORKLOAD += "; Gram on BF16 tensor cores with FP32 sums"
    elif GRAM == 2:
        WORKLOAD += "; Gram on the tcgen05 tensor cores (TF32 split in two terms, FP32 sums)"
    if STORAGE:
        WORKLOAD = WORKLOAD.replace("FP32 storage", "FP16 deviation storage").replace(", FP32", ", FP16 deviation storage")
    if args.lbm:
        lbm_sweep(args)
        return
    if args.workload == "C3":
        print(json.dumps(run_batch_graph(args) if args.c3 == "batch" else run_batch(args)), flush=True)
        return
    if args.profile:
        profile_cycles(args)
        return
    if args.impl == "reference":
        # the CPU reference arm runs on rank 0 only; other ranks exit without work
        rank = int(os.environ.get("RANK", "0"))
        world = int(os.environ.get("WORLD_SIZE", "1"))
        line = run_reference(args, rank, world)
        if line is not None:
            print(json.dumps(line), flush=True)
        return
    dist, rank, world, device = init_dist()
    try:
        line = (run_slab if args.shard == "slab" else run_engine)(args, dist, rank, world, device)
        if rank == 0 and line is not None:
            print(json.dumps(line), flush=True)
    finally:
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
