"""DA_NUDGING (nudging.cu:40-143) and DA_DUMMY (config.h:71-74, main.cu:94) on the GPU,
through the C ABI, against the FP64 oracle on the same forecast state and observations."""
import numpy as np
import pytest

import lbl
import oracle
from test_oracle_nudging import observations

pytestmark = pytest.mark.gpu


def nudging_case(nx, M, p, quadra, ruv, steps=20):
    cfg = lbl.config_default("DA_NUDGING", nx, M, da_xyprune=p, da_quadra=quadra, da_obs_ruv=ruv,
                             daprune=1, da_nud_rate=0.1)
    e = lbl.Ensemble(cfg)
    e.init(0)
    e.update(0, steps)
    return cfg, e


@pytest.mark.parametrize("nx,M,p,quadra,ruv", [(64, 3, 1, 0, 1), (64, 2, 4, 0, 1), (128, 2, 4, 3, 0),
                                               (64, 2, 2, 1, 1), (64, 2, 8, 2, 0)])
def test_nudging_matches_oracle(nx, M, p, quadra, ruv):
    cfg, e = nudging_case(nx, M, p, quadra, ruv)
    o = oracle.Oracle(cfg)
    F = [e.get_f(m) for m in range(M)]
    mac = [e.get_fields(m) for m in range(M)]
    for m in range(M):
        o.set_f(m, F[m])
    ro, uo, vo = observations(nx, p, 11)
    # DA_OBS_UV takes rho from the model's current macros: give the oracle the same
    if not ruv:
        for m in range(M):
            o.set_macros(m, r=mac[m][0])
    e.assimilate(cfg.iiter, ro, uo, vo)
    o.nudge(ro, uo, vo)
    for m in range(M):
        got, want = e.get_f(m).astype(np.float64), o.get_f(m)
        assert np.max(np.abs(got - want) / np.abs(want)) < 1e-6, m
        # the macros are not refreshed by the nudging (nudging.cu has no lbm2euler)
        for a, b in zip(e.get_fields(m)[:3], mac[m][:3]):
            np.testing.assert_array_equal(a, b)
    changed = np.any(e.get_f(0) != F[0], axis=0)
    if quadra % 2 == 1:
        assert not changed[:, nx // 2:].any()
    if quadra >= 2:
        assert not changed[nx // 2:, :].any()
    assert changed.any()


def test_nudging_gate_and_cycle_graph():
    cfg, a = nudging_case(64, 2, 4, 0, 1)
    cfg.daprune = 2
    a.close()
    a, b = lbl.Ensemble(cfg), lbl.Ensemble(cfg)
    for x in (a, b):
        x.init(0)
        x.update(0, 20)
    ro, uo, vo = observations(64, 4, 5)
    f0 = a.get_f(1)
    a.assimilate(cfg.iiter, ro, uo, vo)  # (t/iiter) % daprune = 1: skipped (nudging.cu:43-44)
    np.testing.assert_array_equal(a.get_f(1), f0)
    t = 2 * cfg.iiter
    a.assimilate(t, ro, uo, vo)
    a.update(t, 15)
    b.cycle_async(t, ro, uo, vo, 15)  # one graph: nudging + forcing + 15 steps
    b.sync()
    for m in range(2):
        np.testing.assert_array_equal(a.get_f(m), b.get_f(m))


@pytest.mark.parametrize("mode", ["DA_LETKF", "DA_NUDGING"])
def test_da_dummy_runs_the_ensemble_without_analyses(mode):
    """DA_DUMMY: the DA run's ensemble (seeds +334) with no assimilation (main.cu:94)."""
    kw = dict(daprune=1, da_xyprune=4, letkf_rloc_len=1)
    d = lbl.Ensemble(lbl.config_default(mode, 64, 4, da_dummy=1, **kw))
    r = lbl.Ensemble(lbl.config_default(mode, 64, 4, **kw))
    for x in (d, r):
        x.init(0)
        x.update(0, 10)
    for m in range(4):
        np.testing.assert_array_equal(d.get_f(m), r.get_f(m))  # same members as the DA run
    ro, uo, vo = observations(64, 4, 3)
    f0 = [d.get_f(m) for m in range(4)]
    d.assimilate(d.cfg.iiter, ro, uo, vo)
    for m in range(4):
        np.testing.assert_array_equal(d.get_f(m), f0[m])
    free = lbl.Ensemble(lbl.config_default(mode, 64, 4, da_dummy=1, **kw))
    free.init(0)
    free.update(0, 10)
    d.cycle_async(2 * d.cfg.iiter, ro, uo, vo, 12)  # no analysis inside the graph either
    d.sync()
    free.update(10, 12)
    for m in range(4):
        np.testing.assert_array_equal(d.get_f(m), free.get_f(m))


def test_da_dummy_needs_a_da_mode():
    with pytest.raises(lbl.LblError) as ei:
        lbl.Ensemble(lbl.config_default("NATURE", 64, 1, da_dummy=1))
    assert ei.value.code == -1
