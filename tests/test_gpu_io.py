"""Output path and run modes on the GPU: OBSERVE files bit-exact against the oracle
(io.cu:160-246), NATURE/DA_LETKF file layout and contents (io.cu:22-266), the
ensemble statistics, and the lbl_run driver replaying main.cu's loop end to end."""
import os
import subprocess

import numpy as np
import pytest

from conftest import PKG

import lbl
import oracle

pytestmark = pytest.mark.gpu


def read(path):
    return np.fromfile(path, np.float32)


def test_observe_files_bit_exact(tmp_path):
    cfg = lbl.config_default("OBSERVE", 64, 1, da_xyprune=4, ioprune=1)
    e = lbl.Ensemble(cfg)
    e.init(0)
    o = oracle.Oracle(cfg)  # its engine continues across outputs like the reference's static one
    pre = str(tmp_path / "io")
    for t in (0, cfg.iiter, 2 * cfg.iiter):
        if t:
            e.update(t - cfg.iiter, cfg.iiter)
        e.output(t, pre)
        r, u, v, w = e.get_fields(0)
        want = o.observe(r, u, v)
        step = f"{t // cfg.iiter:010d}"
        for var, a in zip(("rho", "u", "v", "vor"), want):
            got = read(f"{pre}/observed/ens0000/{var}_step{step}.dat")
            np.testing.assert_array_equal(got, a.reshape(-1))  # NaN positions and bits identical
        for var, a in zip(("rho", "u", "v", "vor"), (r, u, v, w)):
            np.testing.assert_array_equal(read(f"{pre}/nature/ens0000/{var}_step{step}.dat"), a.reshape(-1))
        assert not os.path.exists(f"{pre}/calc")  # OBSERVE writes no calc/ (io.cu:306-312)


def test_nature_files_and_vorticity(tmp_path):
    cfg = lbl.config_default("NATURE", 64, 2, ioprune=2)
    e = lbl.Ensemble(cfg)
    e.init(3)
    pre = str(tmp_path / "io")
    e.output(cfg.iiter, pre)  # off the IOPRUNE gate: nothing written
    assert not os.path.exists(pre)
    e.update(0, 2 * cfg.iiter)
    e.output(2 * cfg.iiter, pre)
    for k in range(2):
        r, u, v, w = e.get_fields(k)
        d = f"{pre}/calc/ens{k + 3:04d}"
        np.testing.assert_array_equal(read(f"{d}/u_step0000000002.dat"), u.reshape(-1))
        np.testing.assert_array_equal(read(f"{d}/vor_step0000000002.dat"), oracle.vorticity(cfg, u, v).reshape(-1))
    assert not os.path.exists(f"{pre}/nature")  # ensemble id 0 is not in this run (ofs = 3)


def test_da_output_with_ensemble_statistics(tmp_path):
    cfg = lbl.config_default("DA_LETKF", 64, 4, ioprune=1)
    e = lbl.Ensemble(cfg)
    e.init(0)
    e.update(0, 10)
    pre = str(tmp_path / "io")
    e.output(cfg.iiter, pre)
    us = np.stack([e.get_fields(k)[1] for k in range(4)])
    ws = np.stack([e.get_fields(k)[3] for k in range(4)])
    np.testing.assert_allclose(read(f"{pre}/calc/ens_mean_u_step0000000001.dat"), us.mean(0).reshape(-1), rtol=1e-5, atol=1e-9)
    np.testing.assert_allclose(read(f"{pre}/calc/ens_vor_mean_step0000000001.dat"), ws.mean(0).reshape(-1), rtol=1e-4, atol=1e-6)
    std = read(f"{pre}/calc/ens_vor_std_step0000000001.dat")
    ok = np.isfinite(std)
    np.testing.assert_allclose(std[ok], ws.std(0).reshape(-1)[ok], rtol=2e-2, atol=1e-3)
    for k in range(4):
        assert os.path.exists(f"{pre}/calc/ens{k:04d}/rho_step0000000001.dat")
    um, vm, wm, wsd = e.ens_stats()
    np.testing.assert_allclose(um, us.mean(0), rtol=1e-5, atol=1e-9)


def _stats_like_reference(us, vs, ws):
    """io.cu:88-139 in FP32, members summed in order, one rounding per operation."""
    M = len(us)
    iv = np.float32(1) / np.float32(M)
    um, vm, wm, w2 = (np.zeros_like(us[0]) for _ in range(4))
    for m in range(M):
        um = um + us[m]
        vm = vm + vs[m]
        wm = wm + ws[m]
        w2 = w2 + iv * (ws[m] * ws[m])
    um, vm, wm = um * iv, vm * iv, wm * iv
    with np.errstate(invalid="ignore"):
        sd = np.sqrt(w2 - wm * wm)
    return um, vm, wm, sd


def test_ensemble_statistics_bit_exact_and_async_output(tmp_path):
    """The device vorticity and statistics equal the reference's FP32 host loops bit
    for bit; the asynchronous output writes the same files as the synchronous one."""
    cfg = lbl.config_default("DA_LETKF", 64, 5, ioprune=1)
    e = lbl.Ensemble(cfg)
    e.init(0)
    e.update(0, 3 * cfg.iiter)
    a, b = str(tmp_path / "a"), str(tmp_path / "b")
    e.output(3 * cfg.iiter, a)
    e.output(3 * cfg.iiter, b, sync=False)
    e.sync()
    fields = [e.get_fields(k) for k in range(5)]
    us, vs = [f[1] for f in fields], [f[2] for f in fields]
    ws = [oracle.vorticity(cfg, f[1], f[2]) for f in fields]
    want = _stats_like_reference(us, vs, ws)
    step = "_step0000000003.dat"
    for name, w in zip(("ens_mean_u", "ens_mean_v", "ens_vor_mean", "ens_vor_std"), want):
        np.testing.assert_array_equal(read(f"{a}/calc/{name}{step}"), w.reshape(-1))
    for rel in [f"calc/{n}{step}" for n in ("ens_mean_u", "ens_mean_v", "ens_vor_mean", "ens_vor_std")] + \
               [f"calc/ens{k:04d}/{v}{step}" for k in range(5) for v in ("rho", "u", "v", "vor")]:
        assert open(f"{a}/{rel}", "rb").read() == open(f"{b}/{rel}", "rb").read(), rel


def test_async_output_reports_nan_at_the_next_wait(tmp_path):
    cfg = lbl.config_default("NATURE", 64, 1, ioprune=1)
    e = lbl.Ensemble(cfg)
    e.init(0)
    f = e.get_f(0)
    f[:, 10, 10] = np.nan
    e.set_f(0, f)
    e.output(0, str(tmp_path / "io"), sync=False)  # returns at once; the writer finds the NaN
    with pytest.raises(lbl.LblError) as ei:
        e.sync()
    assert ei.value.code == -5
    e.sync()  # the status was reported once


def test_driver_observe_then_letkf(tmp_path):
    """lbl_run replays main.cu: OBSERVE writes io/observed, DA_LETKF reads it."""
    exe = os.path.join(PKG, "lbl_run")
    pre = str(tmp_path / "io")
    common = ["--nx=64", "--SPINUP=0", "--ITER_MAIN=100", "--IOPRUNE=2", "--DA_XYPRUNE=4", f"--PREFIX={pre}"]
    subprocess.run([exe, "--mode=OBSERVE", *common], check=True, capture_output=True, timeout=300)
    assert os.path.exists(f"{pre}/observed/ens0000/u_step0000000020.dat")
    out = subprocess.run([exe, "--mode=DA_LETKF", "--n_ens=4", "--DAPRUNE=2", "--LETKF_RLOC_LEN=1",
                          "--LETKF_COVINF=1.1", *common], check=True, capture_output=True, text=True, timeout=300)
    assert "ensemble GLUPS" in out.stdout
    main_csv = open(f"{pre}/elapsed_time_rank0.csv").read()
    assert main_csv.startswith("#tag,sec\n")
    tags = [l.split(",")[0] for l in main_csv.strip().split("\n")[1:]]
    for tag in ("DA", "forecast", "output", "_sync.DA"):
        assert tag in tags
    letkf_csv = open(f"{pre}/letkf_elapsed_time_rank0.csv").read()
    assert "solve," in letkf_csv and "load_obs," in letkf_csv
    for k in range(4):
        assert os.path.exists(f"{pre}/calc/ens{k:04d}/vor_step0000000020.dat")
    assert os.path.exists(f"{pre}/calc/ens_vor_std_step0000000020.dat")


def test_async_rmse_equals_the_blocking_one():
    """lbl_rmse_uv_async enqueues what lbl_rmse_uv does and leaves the value in the
    caller's (pinned) double; it equals the blocking form (to the rounding of an FP64
    sum accumulated in no fixed order) after the stream has passed it.  lbl_get_stream hands out the
    context's stream, on which a caller's own work runs in submission order."""
    torch = pytest.importorskip("torch")
    e = lbl.Ensemble(lbl.config_default("NATURE", 128, 3))
    e.init(0)
    rng = np.random.default_rng(5)
    truth = [tuple(torch.from_numpy(rng.standard_normal((128, 128)).astype(np.float32) * 0.01).pin_memory().numpy()
                   for _ in range(2)) for _ in range(3)]
    out = torch.zeros(3, dtype=torch.float64).pin_memory().numpy()
    ref = []
    for k in range(3):
        e.update(k * 5, 5)
        ref.append(e.rmse_uv(*truth[k]))
    e2 = lbl.Ensemble(lbl.config_default("NATURE", 128, 3))
    e2.init(0)
    for k in range(3):
        e2.update(k * 5, 5)
        e2.rmse_uv_async(*truth[k], out, k)
    e2.sync()
    # the FP64 sum is accumulated with atomics, in no fixed order: equal to rounding
    np.testing.assert_allclose(out, np.array(ref), rtol=1e-12, atol=0)
    s = e2.stream()
    assert s != 0
    buf = torch.zeros(1 << 20, device="cuda:0")
    with torch.cuda.stream(torch.cuda.ExternalStream(s, device="cuda:0")):
        buf.fill_(2.0)
    e2.sync()
    assert float(buf.sum()) == 2.0 * (1 << 20)
    with pytest.raises(ValueError):
        e2.rmse_uv_async(truth[0][0].astype(np.float64), truth[0][1], out, 0)
    e.close()
    e2.close()
