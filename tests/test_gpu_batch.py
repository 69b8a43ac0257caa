"""Batches on the GPU: several experiments of uneven grid and ensemble size cycled
together (one graph per cycle, one batched persistent stream-collide launch per step)
give bit for bit the populations of the same experiments cycled one by one."""
import numpy as np
import pytest

import lbl

pytestmark = pytest.mark.gpu

# (mode, nx, M): whole 128-column rows, chunked rows (2, 4 chunks), the wide
# analysis (M = 40) and an experiment without analysis
EXPERIMENTS = [("DA_LETKF", 128, 4), ("DA_LETKF", 256, 8), ("NATURE", 256, 2), ("DA_LETKF", 512, 2),
               ("DA_LETKF", 128, 40)]


def _cfg(mode, nx, M):
    return lbl.config_default(mode, nx, M, da_xyprune=4, letkf_rloc_len=1, letkf_covinf=1.1, obs_error_u=0.1,
                              obs_error_rho=0.01, iiter=20, daprune=5, ic_kind=lbl.IC_K4EXP, ic_amp=1.0,
                              ens_init=lbl.ENS_PERTURBED, ens_perturb=0.1)


def _observations(nx, seed):
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:nx, 0:nx] * (2 * np.pi / nx)
    u = (np.sin(4 * y + seed) + 0.1 * rng.standard_normal((nx, nx))).astype(np.float32)
    v = (np.cos(4 * x) + 0.1 * rng.standard_normal((nx, nx))).astype(np.float32)
    r = (1 + 0.01 * rng.standard_normal((nx, nx))).astype(np.float32)
    off = np.ones((nx, nx), bool)
    off[::4, ::4] = False
    for a in (r, u, v):
        a[off] = np.nan
    return r, u, v


@pytest.mark.parametrize("strip_rows", [0, 7])
def test_batch_equals_separate_contexts(strip_rows):
    solo = [lbl.Ensemble(_cfg(*ex)) for ex in EXPERIMENTS]
    mine = [lbl.Ensemble(_cfg(*ex)) for ex in EXPERIMENTS]
    for e in solo + mine:
        e.init(0)
    batch = lbl.Batch(mine, strip_rows)
    T = 100
    for c in range(3):
        t = c * T
        obs = [_observations(nx, 10 * c + i) if mode != "NATURE" else None
               for i, (mode, nx, M) in enumerate(EXPERIMENTS)]
        for e, o in zip(solo, obs):
            e.cycle_async(t, *(o if o is not None else (None, None, None)), T)
        batch.cycle_async(t, obs, T)
    for e in solo:
        e.sync()
    batch.sync()
    for (mode, nx, M), a, b in zip(EXPERIMENTS, solo, mine):
        for m in range(M):
            np.testing.assert_array_equal(a.get_f(m), b.get_f(m), err_msg=f"{mode} {nx} member {m}")
        np.testing.assert_array_equal(a.get_fields(M - 1)[1], b.get_fields(M - 1)[1])
    assert all(b.letkf_stats()["nan"] == 0 for b, (mode, _, _) in zip(mine, EXPERIMENTS) if mode == "DA_LETKF")
    batch.close()


def test_batch_rejects_what_it_does_not_batch():
    a = lbl.Ensemble(lbl.config_default("NATURE", 64, 1))
    a.init(0)
    with pytest.raises(lbl.LblError) as ei:  # 64 columns: not a multiple of the 128-column chunk
        lbl.Batch([a])
    assert ei.value.code == -8
    b = lbl.Ensemble(lbl.config_default("NATURE", 128, 1))
    with pytest.raises(lbl.LblError) as ei:  # not initialised
        lbl.Batch([b])
    assert ei.value.code == -6
    b.init(0)
    with pytest.raises(lbl.LblError) as ei:  # the same context twice
        lbl.Batch([b, b])
    assert ei.value.code == -1
