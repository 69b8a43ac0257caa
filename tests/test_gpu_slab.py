"""The y-slab split on the GPU, through the C ABI (lbl_slab_set, lbl_slab_pack,
lbl_slab_unpack) and lbl.slab.SlabExperiment.

All bands of one experiment run in this process on one GPU and read each other's packed
halos in place (the transfer between GPUs is NCCL's, covered on the CPU by
tests/test_slab_split.py).  Every band runs the same kernels as a whole-grid context over
its own rows plus halos, so its own rows must equal the whole-grid run bit for bit: the
forecast, the analysis, FP32 and FP16 storage, 1 to 4 bands, even and uneven."""
import numpy as np
import pytest

import lbl
from lbl import slab

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _whole(cfg):
    e = lbl.Ensemble(cfg)
    e.init(0)
    return e


def _assert_own_rows_equal(whole, exp, what):
    for m in range(whole.M):
        f = whole.get_f(m)
        for rank, fo in exp.own_f(m).items():
            row0, own = exp.bands[rank]
            d = np.abs(fo - f[:, row0:row0 + own])
            assert d.max() == 0.0, (what, m, rank, float(d.max()), np.argwhere(d > 0)[:3].tolist())


def test_pack_and_unpack_move_the_planned_rows():
    cfg = lbl.config_default("NATURE", 64, 3)
    with slab.SlabExperiment(cfg, world=2, halo=4) as exp:
        exp.init(0)
        b = exp.local[0]
        nyl = b.own + 2 * b.halo
        rng = np.random.default_rng(3)
        fs = [rng.random((9, nyl, 64), dtype=np.float32) for _ in range(3)]
        for m, f in enumerate(fs):
            b.ens.set_f(m, f)
        for rows in (1, 3, 4):
            plan = slab.halo_rows(nyl, b.halo, rows)
            b.ens.slab_pack(rows, b.ptr("send_prev"), b.ptr("send_next"))
            b.ens.sync()
            nb = b.ens.slab_halo_bytes(rows)
            assert nb == 3 * 9 * rows * 64 * 4
            for key, buf in (("to_prev", "send_prev"), ("to_next", "send_next")):
                got = b.buf[buf][:nb].cpu().view(torch.float32).numpy().reshape(3, 9, rows, 64)
                want = np.stack([f[:, slice(*plan[key])] for f in fs])
                assert np.array_equal(got, want), (rows, key)
            # unpack two marked buffers into the halos and leave every other row alone
            src_p = torch.full((nb // 4,), 7.0, device="cuda")
            src_n = torch.full((nb // 4,), -7.0, device="cuda")
            b.ens.slab_unpack(rows, src_p.data_ptr(), src_n.data_ptr())
            b.ens.sync()
            for m, f in enumerate(fs):
                g = b.ens.get_f(m)
                assert (g[:, :rows] == 7.0).all() and (g[:, nyl - rows:] == -7.0).all()
                assert np.array_equal(g[:, rows:nyl - rows], f[:, rows:nyl - rows])
                b.ens.set_f(m, f)


@pytest.mark.parametrize("storage", [lbl.STORAGE_F32, lbl.STORAGE_F16])
@pytest.mark.parametrize("nx,world,halo,bands", [
    (128, 1, 2, None), (128, 2, 2, None), (128, 3, 2, [(0, 40), (40, 40), (80, 48)]), (128, 4, 8, None),
    (128, 2, 6, [(0, 72), (72, 56)]),
    (256, 2, 8, None), (512, 2, 8, None),  # the bands' kernels specialised on 256 and 512 columns
])
def test_forecast_bands_equal_the_whole_grid(storage, nx, world, halo, bands):
    cfg = lbl.config_default("NATURE", nx, 4, storage=storage)
    whole = _whole(cfg)
    with slab.SlabExperiment(cfg, world=world, halo=halo, bands=bands) as exp:
        exp.init(0)
        _assert_own_rows_equal(whole, exp, "initial condition")
        whole.update(0, 37)
        exp.update(0, 37)
        exp.sync()
        _assert_own_rows_equal(whole, exp, f"37 steps, halo {halo}")
    whole.close()


def _observations(nx, steps):
    nat = lbl.Ensemble(lbl.config_default("NATURE", nx, 1))
    nat.init(0)
    nat.update(0, steps)
    r, u, v, _ = nat.get_fields(0)
    nat.close()
    rng = np.random.default_rng(5)
    return ((r + rng.normal(0, 0.01, r.shape)).astype(np.float32), (u + rng.normal(0, 0.1, u.shape) * 0.05)
            .astype(np.float32), (v + rng.normal(0, 0.1, v.shape) * 0.05).astype(np.float32), u, v)


@pytest.mark.parametrize("nx,m,storage,world,bands", [
    (128, 16, lbl.STORAGE_F32, 2, None),
    (128, 16, lbl.STORAGE_F32, 3, [(0, 48), (48, 40), (88, 40)]),
    (128, 16, lbl.STORAGE_F16, 4, None),
    (64, 40, lbl.STORAGE_F32, 2, None),       # the M > 32 analysis kernel (8-row tiles)
    (128, 16, lbl.STORAGE_F32, 1, None),      # one band, its own neighbour
])
def test_da_cycle_bands_equal_the_whole_grid(nx, m, storage, world, bands):
    cfg = lbl.config_default("DA_LETKF", nx, m, storage=storage, da_xyprune=4, letkf_rloc_len=1,
                             obs_error_u=0.1, obs_error_rho=0.01, iiter=10, daprune=5)  # t = 50 is due
    ro, uo, vo, ut, vt = _observations(nx, 50)
    whole = _whole(cfg)
    with slab.SlabExperiment(cfg, world=world, bands=bands) as exp:
        assert exp.halo == 8
        exp.init(0)
        whole.update(0, 50)
        exp.update(0, 50)
        whole.assimilate(50, ro, uo, vo)
        exp.assimilate(50, ro, uo, vo)
        exp.sync()
        _assert_own_rows_equal(whole, exp, "analysis")
        assert exp.rmse_uv(ut, vt) == pytest.approx(whole.rmse_uv(ut, vt), rel=1e-12)
        st = exp.letkf_stats()
        assert st["nan"] == 0 and st["max_sweeps"] > 0 and whole.letkf_stats()["max_sweeps"] > 0
        whole.update(50, 23)
        exp.update(50, 23)
        exp.sync()
        _assert_own_rows_equal(whole, exp, "forecast after the analysis")
    whole.close()


def test_slab_conditions_are_checked():
    def fresh(mode="DA_LETKF", ny=None, **kw):
        c = lbl.config_default(mode, 64, 4, da_xyprune=4, letkf_rloc_len=1, **kw)
        if ny:
            c.ny = ny
        return lbl.Ensemble(c)

    e = fresh(ny=48)
    with pytest.raises(lbl.LblError, match="halo must cover"):
        fresh(ny=40).slab_set(64, 0, 4)
    with pytest.raises(lbl.LblError, match="multiples"):
        e.slab_set(64, 4, 8)
    with pytest.raises(lbl.LblError, match="at least 2"):
        fresh("NATURE", ny=40).slab_set(64, 0, 1)
    with pytest.raises(lbl.LblError, match="own at least"):
        fresh("NATURE", ny=20).slab_set(64, 0, 8)
    with pytest.raises(lbl.LblError, match="NATURE or DA_LETKF"):
        fresh("OBSERVE", ny=48).slab_set(64, 0, 8)
    with pytest.raises(lbl.LblError, match="not a y-slab"):
        fresh(ny=48).slab_pack(2, 0, 0)
    e.slab_set(64, 0, 8)
    with pytest.raises(lbl.LblError, match="before lbl_init"):
        e.slab_pack(2, 0, 0)
    e.init(0)
    with pytest.raises(lbl.LblError, match="after lbl_init"):
        e.slab_set(64, 0, 8)
    buf = torch.empty(e.slab_halo_bytes(8) + 16, dtype=torch.uint8, device="cuda")
    with pytest.raises(lbl.LblError, match=r"\[1, halo\]"):
        e.slab_pack(9, buf.data_ptr(), buf.data_ptr())
    with pytest.raises(lbl.LblError, match="16-byte"):
        e.slab_pack(2, buf.data_ptr() + 4, buf.data_ptr())
    with pytest.raises(lbl.LblError, match="cycle graph"):
        e.cycle_async(0, None, None, None, 10)
    with pytest.raises(lbl.LblError, match="no files"):
        e.output(0, "/nonexistent")
    with pytest.raises(lbl.LblError, match="Smagorinsky"):
        e.set_closure(np.zeros(lbl.CLOSURE_PARAMS, np.float32), 1e-4, 0.1)
    # the chunked forecast: begun steps only, at most halo / 2 per chunk, nothing else until done
    with pytest.raises(lbl.LblError, match="no chunked forecast"):
        e.slab_forecast_chunk(2)
    with pytest.raises(lbl.LblError, match=r"\[1, lbl_slab_forecast_steps\]"):
        e.slab_forecast_begin(0, e.slab_forecast_steps() + 1)
    e.slab_forecast_begin(0, 6)
    with pytest.raises(lbl.LblError, match="has steps left"):
        e.update(0, 1)
    with pytest.raises(lbl.LblError, match="has steps left"):
        e.slab_forecast_begin(0, 6)
    with pytest.raises(lbl.LblError, match=r"halo / 2"):
        e.slab_forecast_chunk(5)
    e.slab_forecast_chunk(4)
    with pytest.raises(lbl.LblError, match=r"steps left\)"):
        e.slab_forecast_chunk(3)
    e.slab_forecast_chunk(2)
    e.update(6, 1)
    e.sync()
    e.close()


@pytest.mark.parametrize("world", [2, 4])
def test_c1_workload_in_bands_equals_the_whole_grid(world):
    """The 256^2 x 16 DA workload's own settings (Cs 0.1, tau 0.51: nu from the global dt; the
    k^4 exp initial condition rescaled by the whole grid's energy; members = the nature IC plus
    10 % perturbations) through three whole cycles (100 steps, then an analysis) in 2 and 4
    bands: bit for bit, and the same RMSE."""
    cfg = lbl.config_default("DA_LETKF", 256, 16, da_xyprune=4, letkf_rloc_len=1, letkf_covinf=1.1, obs_error_u=0.1,
                             obs_error_rho=0.01, iiter=20, daprune=5, cs=0.1, tau=0.51, ic_kind=lbl.IC_K4EXP,
                             ic_amp=1.0, ens_init=lbl.ENS_PERTURBED, ens_perturb=0.1)
    obs = [_observations(256, 100 * c) for c in (1, 2, 3)]
    whole = _whole(cfg)
    with slab.SlabExperiment(cfg, world=world) as exp:
        exp.init(0)
        _assert_own_rows_equal(whole, exp, "initial condition")
        for c, (ro, uo, vo, ut, vt) in enumerate(obs):
            t = 100 * c
            whole.update(t, 100)
            exp.update(t, 100)
            whole.assimilate(t + 100, ro, uo, vo)
            exp.assimilate(t + 100, ro, uo, vo)
            exp.sync()
            assert whole.letkf_stats()["max_sweeps"] > 0
            _assert_own_rows_equal(whole, exp, f"cycle {c + 1}")
            assert exp.rmse_uv(ut, vt) == pytest.approx(whole.rmse_uv(ut, vt), rel=1e-12)
    whole.close()
