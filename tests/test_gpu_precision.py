"""The precision form (the 512^2 x 64 workload's storage): populations stored as FP16 deviations
f - w_q with the collide, the forcing and the analysis in FP32.  Its error is
stated against the FP32 engine, which the other tests pin to the reference."""
import numpy as np
import pytest

import lbl

pytestmark = pytest.mark.gpu

W = np.array([1 / 36, 1 / 9, 1 / 36, 1 / 9, 4 / 9, 1 / 9, 1 / 36, 1 / 9, 1 / 36], np.float32)[:, None, None]


def storage_round(f):
    """What FP16 deviation storage keeps of FP32 populations [9][ny][nx]."""
    return W + (f - W).astype(np.float16).astype(np.float32)


def test_set_get_round_trip():
    e = lbl.Ensemble(lbl.config_default("NATURE", 64, 2, storage=lbl.STORAGE_F16))
    e.init(0)
    f = e.get_f(1)
    np.testing.assert_array_equal(f, storage_round(f))  # already representable
    rng = np.random.default_rng(0)
    g = (W * (1 + 0.1 * rng.standard_normal(f.shape))).astype(np.float32)
    e.set_f(1, g)
    np.testing.assert_array_equal(e.get_f(1), storage_round(g))


def test_initial_condition_is_the_rounded_fp32_one():
    a = lbl.Ensemble(lbl.config_default("NATURE", 128, 2))
    b = lbl.Ensemble(lbl.config_default("NATURE", 128, 2, storage=lbl.STORAGE_F16))
    for x in (a, b):
        x.init(0)
    for m in range(2):
        np.testing.assert_array_equal(b.get_f(m), storage_round(a.get_f(m)))


@pytest.mark.parametrize("nx", [128, 256])
def test_forecast_error_against_fp32(nx):
    """100 steps: the FP16 storage error stays small against the FP32 run (stated bound)."""
    a = lbl.Ensemble(lbl.config_default("NATURE", nx, 2))
    b = lbl.Ensemble(lbl.config_default("NATURE", nx, 2, storage=lbl.STORAGE_F16))
    for x in (a, b):
        x.init(0)
        x.update(0, 100)
    for m in range(2):
        fa, fb = a.get_f(m).astype(np.float64), b.get_f(m).astype(np.float64)
        norm = np.linalg.norm(fb - fa) / np.linalg.norm(fa)
        elem = np.max(np.abs(fb - fa) / np.abs(fa))
        ua, ub = a.get_fields(m)[1].astype(np.float64), b.get_fields(m)[1].astype(np.float64)
        uerr = np.max(np.abs(ub - ua)) / np.max(np.abs(ua))
        print(f"nx={nx} member {m}: populations normwise {norm:.2e}, elementwise {elem:.2e}; u {uerr:.2e} of max")
        assert norm < 1e-4 and elem < 2e-3 and uerr < 2e-2


def test_analysis_is_the_fp32_analysis_rounded():
    """The analysis runs in FP32 on the expanded forecast; only its result is rounded."""
    kw = dict(da_xyprune=4, letkf_rloc_len=1, letkf_covinf=1.1, obs_error_u=0.002, obs_error_rho=1e-4, daprune=1)
    h = lbl.Ensemble(lbl.config_default("DA_LETKF", 64, 8, storage=lbl.STORAGE_F16, **kw))
    s = lbl.Ensemble(lbl.config_default("DA_LETKF", 64, 8, **kw))
    h.init(0)
    h.update(0, 20)
    s.init(0)
    for m in range(8):
        s.set_f(m, h.get_f(m))  # the same forecast, FP32 storage
    rng = np.random.default_rng(2)
    obs = []
    for sig, base in ((1e-4, 1.0), (2e-3, 0.0), (2e-3, 0.0)):
        o = np.full((64, 64), np.nan, np.float32)
        o[::4, ::4] = base + sig * rng.standard_normal((16, 16))
        obs.append(o)
    h.assimilate(h.cfg.iiter, *obs)
    s.assimilate(s.cfg.iiter, *obs)
    for m in range(8):
        np.testing.assert_array_equal(h.get_f(m), storage_round(s.get_f(m)))


def test_nudging_with_fp16_storage():
    kw = dict(da_xyprune=4, daprune=1)
    h = lbl.Ensemble(lbl.config_default("DA_NUDGING", 64, 2, storage=lbl.STORAGE_F16, **kw))
    s = lbl.Ensemble(lbl.config_default("DA_NUDGING", 64, 2, **kw))
    h.init(0)
    h.update(0, 10)
    s.init(0)
    for m in range(2):
        s.set_f(m, h.get_f(m))
    rng = np.random.default_rng(5)
    obs = []
    for sig, base in ((1e-2, 1.0), (5e-2, 0.0), (5e-2, 0.0)):
        o = np.full((64, 64), np.nan, np.float32)
        o[::4, ::4] = base + sig * rng.standard_normal((16, 16))
        obs.append(o)
    h.assimilate(h.cfg.iiter, *obs)
    s.assimilate(s.cfg.iiter, *obs)
    for m in range(2):
        # the two kernel instantiations may contract alpha f_obs + (1 - alpha) f into different
        # FMAs: the FP32 values then differ in the last bit, and a few FP16 roundings by one ulp
        got, want = h.get_f(m), storage_round(s.get_f(m))
        ulp = np.spacing(np.abs(want - W).astype(np.float16)).astype(np.float32)
        assert np.all(np.abs(got - want) <= ulp)
        assert np.mean(got != want) < 0.01


def test_fp16_storage_rejects_the_tma_kernel():
    with pytest.raises(lbl.LblError) as ei:
        lbl.Ensemble(lbl.config_default("NATURE", 256, 1, storage=lbl.STORAGE_F16, lbm_variant=lbl.LBM_TMA))
    assert ei.value.code == -8
