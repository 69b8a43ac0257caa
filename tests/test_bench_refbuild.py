"""The host side of bench.py's reference-build timing (`reference_build` and the cycle rate of the
`--impl reference` line), on the CPU: a stand-in executable that speaks the `time`
protocol of oracle/ref_lbm_harness.cu (create the ready file, wait for the go file,
print `ref_lbm_time <id> <nsteps> <t0_ns> <t1_ns>`) replaces the reference build, so
the start barrier, the parsing and the aggregation are checked without a GPU."""
import os
import stat
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402

FAKE = """#!{py}
import os, sys, time
_, mode, ident, nsteps, warmup, ready, go = sys.argv
open(ready, "w").close()
t_end = time.time() + 30
while not os.path.exists(go):
    if time.time() > t_end:
        sys.exit(3)
    time.sleep(0.001)
t0 = time.time_ns()
time.sleep({step_s} * int(nsteps))
t1 = time.time_ns()
print("ref_lbm_time", ident, nsteps, t0, t1)
sys.exit({rc})
"""


def _fake(tmp_path, step_s=0.0002, rc=0):
    path = tmp_path / "fake_ref_lbm"
    path.write_text(FAKE.format(py=sys.executable, step_s=step_s, rc=rc))
    path.chmod(path.stat().st_mode | stat.S_IXUSR)
    return str(path)


def test_processes_start_together_and_rates_aggregate(tmp_path):
    exe = _fake(tmp_path)
    r = bench.reference_build_forecast(4, 100, exe=exe)
    assert "unavailable" not in r, r
    assert r["processes"] == 4 and r["steps_per_process"] == 100
    # 4 processes x 100 steps of >= 0.2 ms each, run side by side: the span covers one process at least
    assert r["seconds"] >= 0.02
    assert r["ms_per_100_steps"] == pytest.approx(1e3 * r["seconds"], rel=1e-9)
    assert r["forecast_glups"] == pytest.approx(4 * 256 * 256 * 100 / r["seconds"] * 1e-9, rel=1e-9)


def test_a_failing_process_makes_the_line_unavailable(tmp_path):
    r = bench.reference_build_forecast(2, 10, exe=_fake(tmp_path, rc=1))
    assert "unavailable" in r and "exited 1" in r["unavailable"]


def test_a_missing_build_is_reported(tmp_path):
    r = bench.reference_build_forecast(1, 10, exe=str(tmp_path / "nothing_here"))
    assert "unavailable" in r


def test_analysis_roofline_counts_the_per_point_flops():
    """analysis_roofline: Gram 2 n_obs M^2 + transform 2*9*M^2 + 4 M^3 + Jacobi 18 M M(M-1)/2
    per sweep, per grid point, over the phase time, against 148 x 128 x 2 x 1.965 GHz."""
    nx, m = bench.NX, bench.M
    try:
        bench.NX, bench.M = 256, 16
        r = bench.analysis_roofline({"mean_sweeps": 3.0}, 1.0)
        per_point = 2 * 75 * 256 + 2 * 9 * 256 + 4 * 4096 + 18 * 16 * 16 * 15 / 2 * 3.0
        assert r["flops_per_point"] == pytest.approx(per_point)
        assert r["achieved"] == pytest.approx(per_point * 256 * 256 / 1e-3 / 1e12)
        assert r["peak"] == pytest.approx(148 * 128 * 2 * 1.965e9 / 1e12)
        assert r["frac"] == pytest.approx(r["achieved"] / r["peak"])
    finally:
        bench.NX, bench.M = nx, m


FAKE_OSSE = """#!{py}
import sys
_, mode, m, cycles, steps, warmup = sys.argv
assert mode == "time"
print("ensemble 0: initial velocity with random_seed = 0")
print("ref_osse_time", m, cycles, steps, {sec})
sys.exit({rc})
"""


def _fake_osse(tmp_path, sec=0.5, rc=0):
    path = tmp_path / "fake_ref_osse"
    path.write_text(FAKE_OSSE.format(py=sys.executable, sec=sec, rc=rc))
    path.chmod(path.stat().st_mode | stat.S_IXUSR)
    return str(path)


def test_reference_cycle_rate_is_parsed(tmp_path):
    """reference_osse_cycle (the reference arm's value at 256^2 x 16): the `time` protocol of
    oracle/ref_osse_harness.cu, `ref_osse_time <M> <cycles> <steps> <seconds>`."""
    r = bench.reference_osse_cycle(cycles=5, warmup=2, exe=_fake_osse(tmp_path, sec=0.55))
    assert r["cycles_per_s"] == pytest.approx(5 / 0.55) and r["ms_per_cycle"] == pytest.approx(110.0)
    assert r["cycles"] == 5 and r["warmup"] == 2


def test_reference_cycle_failures_are_reported(tmp_path):
    assert "unavailable" in bench.reference_osse_cycle(exe=_fake_osse(tmp_path, rc=2))
    assert "unavailable" in bench.reference_osse_cycle(exe=str(tmp_path / "nothing_here"))
