"""LETKF analysis on the GPU, through the C ABI, against the FP64 oracle on
identical forecast ensembles and observations, for the reference's window
geometries (p = 1 pointwise, p > 1 R-localised, LETKF_RLOC_LEN), ensemble sizes
and inflation; plus the stale-v quirk, the DA gate, NaN reporting and the
one-graph cycle."""
import numpy as np
import pytest

import lbl
import oracle

pytestmark = pytest.mark.gpu


def make_case(nx, M, p, L, beta, steps=30, sig_u=0.002, sig_r=1e-4, **kw):
    cfg = lbl.config_default("DA_LETKF", nx, M, da_xyprune=p, letkf_rloc_len=L, letkf_covinf=beta,
                             obs_error_u=sig_u, obs_error_rho=sig_r, daprune=1, **kw)
    e = lbl.Ensemble(cfg)
    e.init(0)
    e.update(0, steps)
    nat = lbl.Ensemble(lbl.config_default("NATURE", nx, 1))
    nat.init(0)
    nat.update(0, steps)
    r, u, v, _ = nat.get_fields(0)
    rng = np.random.default_rng(nx + M + p)
    ro = (r + sig_r * rng.standard_normal(r.shape)).astype(np.float32)
    uo = (u + sig_u * rng.standard_normal(u.shape)).astype(np.float32)
    vo = (v + sig_u * rng.standard_normal(v.shape)).astype(np.float32)
    off = np.ones_like(ro, bool)
    off[::p, ::p] = False
    for a in (ro, uo, vo):
        a[off] = np.nan  # like io/observed files: NaN off the observation lattice
    return cfg, e, (ro, uo, vo), u, v


CASES = [  # nx, M, p, L, beta
    (64, 4, 1, 0, 1.0),
    (64, 8, 2, 0, 1.1),
    (64, 16, 4, 1, 1.1),
    (64, 6, 4, 1, 1.05),
    (64, 32, 4, 1, 1.1),
    (128, 16, 4, 2, 1.2),
    (256, 16, 4, 1, 1.1),
    (96, 12, 4, 1, 1.1),
    (64, 64, 4, 1, 1.1),   # 32 < M <= 64: the 64-thread analysis kernel (the 512^2 workload's ensemble size)
    (64, 48, 4, 1, 1.1),
    (64, 40, 2, 0, 1.05),
    (64, 33, 4, 1, 1.1),   # 31 zero padding columns in the quad-owned Jacobi
    (96, 64, 4, 1, 1.1),   # 24 x 12 tiles of 4 x 8 points
]


@pytest.mark.parametrize("nx,M,p,L,beta", CASES)
def test_analysis_matches_oracle(nx, M, p, L, beta):
    cfg, e, obs, _, _ = make_case(nx, M, p, L, beta)
    F = [e.get_f(m) for m in range(M)]
    o = oracle.Oracle(cfg)
    for m in range(M):
        o.set_f(m, F[m])
    t = cfg.iiter
    e.assimilate(t, *obs)
    o.assimilate(*obs)
    st = e.letkf_stats()
    assert st["nan"] == 0 and st["n_noconv"] == 0 and 1 <= st["max_sweeps"] <= 30, st
    inc_e = np.stack([e.get_f(m).astype(np.float64) - F[m] for m in range(M)])
    inc_o = np.stack([o.get_f(m) - F[m] for m in range(M)])
    scale = np.max(np.abs(inc_o))
    print(f"nx={nx} M={M} p={p} L={L}: sweeps max {st['max_sweeps']} mean {st['mean_sweeps']:.2f}, "
          f"increment error {np.max(np.abs(inc_e - inc_o)) / scale:.2e} of the largest increment")
    assert scale > 1e-6  # the analysis does something
    # analysis increments within 1e-3 of their largest magnitude (FP32 Gram/Jacobi vs FP64)
    assert np.max(np.abs(inc_e - inc_o)) / scale < 1e-3
    # populations themselves within 1e-5 relative
    fa = np.stack([o.get_f(m) for m in range(M)])
    assert np.max(np.abs(np.stack([e.get_f(m) for m in range(M)]) - fa) / np.abs(fa)) < 1e-5


# The bench workloads at their own observation errors (sigma_u 0.1, sigma_rho 0.01):
# 256^2 x 16 and 512^2 x 64 (the wide analysis kernel), the benchmark workloads' shapes, analysed
# on a band of rows by the FP64 oracle.  Measured: 1.0e-5 and 2.8e-5 of the largest
# increment (the reference's own FP32 cuBLAS/cuSOLVER path sits 3e-6..2.5e-5 from FP64).
WORKLOAD_TOL = 1e-4


@pytest.mark.parametrize("nx,M,rows", [(256, 16, (0, 16)), (512, 64, (0, 8)), (1024, 64, (1020, 1024))])
def test_workload_analysis_matches_oracle(nx, M, rows):
    """(1024^2 x 64 is the largest DA configuration: its last rows, whose windows wrap
    around the periodic edge.)"""
    cfg = lbl.config_default("DA_LETKF", nx, M, da_xyprune=4, letkf_rloc_len=1, letkf_covinf=1.1, obs_error_u=0.1,
                             obs_error_rho=0.01, daprune=1, iiter=20, cs=0.1, tau=0.51, ic_kind=lbl.IC_K4EXP,
                             ic_amp=1.0, ens_init=lbl.ENS_PERTURBED, ens_perturb=0.1)
    e = lbl.Ensemble(cfg)
    e.init(0)
    e.update(0, 100)
    ncfg = lbl.config_default("NATURE", nx, 1, cs=0.1, tau=0.51, ic_kind=lbl.IC_K4EXP, ic_amp=1.0)
    nat = lbl.Ensemble(ncfg)
    nat.init(0)
    nat.update(0, 100)
    r, u, v, _ = nat.get_fields(0)
    nat.close()
    rng = np.random.default_rng(nx + M)
    obs = []
    for a, sg in ((r, 0.01), (u, 0.1), (v, 0.1)):
        o_ = (a + sg * rng.standard_normal(a.shape)).astype(np.float32)
        off = np.ones_like(o_, bool)
        off[::4, ::4] = False
        o_[off] = np.nan
        obs.append(o_)
    F = np.stack([e.get_f(m) for m in range(M)])
    o = oracle.Oracle(cfg)
    for m in range(M):
        o.set_f(m, F[m])
    j0, j1 = rows
    o.assimilate_rows(*obs, j0, j1)
    inc_o = np.stack([o.get_f(m)[:, j0:j1] for m in range(M)]) - F[:, :, j0:j1]
    o.close()
    e.assimilate(cfg.iiter, *obs)
    st = e.letkf_stats()
    inc_e = np.stack([e.get_f(m)[:, j0:j1] for m in range(M)]).astype(np.float64) - F[:, :, j0:j1]
    e.close()
    assert st["nan"] == 0 and st["n_noconv"] == 0, st
    scale = np.max(np.abs(inc_o))
    err = np.max(np.abs(inc_e - inc_o)) / scale
    print(f"{nx}^2 x {M}: increment error {err:.2e} of the largest increment, mean sweeps {st['mean_sweeps']:.2f}")
    assert scale > 1e-6 and err < WORKLOAD_TOL


@pytest.mark.parametrize("M,p,L", [(64, 4, 1), (48, 2, 0), (40, 4, 2)])
def test_bf16_gram_precision_form(M, p, L):
    """The precision form's Gram (BF16 operands on the tensor cores, FP32 sums) against
    the FP64 oracle: the analysis increments move by the BF16 rounding of the weighted
    window (2^-9 relative), so the bound is 1e-2 of the largest increment instead of 1e-3;
    and it is a different computation from the FP32 Gram."""
    cfg, e, obs, _, _ = make_case(64, M, p, L, 1.1, gram=lbl.GRAM_BF16)
    F = [e.get_f(m) for m in range(M)]
    o = oracle.Oracle(cfg)
    for m in range(M):
        o.set_f(m, F[m])
    e.assimilate(cfg.iiter, *obs)
    o.assimilate(*obs)
    st = e.letkf_stats()
    assert st["nan"] == 0 and st["n_noconv"] == 0, st
    inc_e = np.stack([e.get_f(m).astype(np.float64) - F[m] for m in range(M)])
    inc_o = np.stack([o.get_f(m) - F[m] for m in range(M)])
    scale = np.max(np.abs(inc_o))
    err = np.max(np.abs(inc_e - inc_o)) / scale
    print(f"BF16 Gram M={M} p={p} L={L}: increment error {err:.2e} of the largest increment")
    assert scale > 1e-6 and err < 1e-2
    cfg32, e32, _, _, _ = make_case(64, M, p, L, 1.1)
    e32.assimilate(cfg32.iiter, *obs)
    inc_32 = np.stack([e32.get_f(m).astype(np.float64) - F[m] for m in range(M)])
    assert np.max(np.abs(inc_e - inc_32)) > 0


@pytest.mark.parametrize("nx,M,p,L", [(64, 16, 4, 1), (64, 6, 4, 1), (64, 32, 4, 1), (64, 64, 4, 1), (64, 40, 4, 1),
                                      (64, 12, 4, 0), (128, 16, 4, 1), (96, 64, 4, 1)])
def test_tensor_core_gram_matches_oracle(nx, M, p, L):
    """The Gram on the tcgen05 tensor cores (LBL_GRAM_TF32X3: every operand split into two
    TF32 terms, three MMAs, FP32 sums) against the FP64 oracle, with the FP32 analysis's
    bound, and against the SIMT FP32 Gram of the same forecast."""
    cfg, e, obs, _, _ = make_case(nx, M, p, L, 1.1, gram=lbl.GRAM_TF32X3)
    F = [e.get_f(m) for m in range(M)]
    o = oracle.Oracle(cfg)
    for m in range(M):
        o.set_f(m, F[m])
    e.assimilate(cfg.iiter, *obs)
    o.assimilate(*obs)
    st = e.letkf_stats()
    assert st["nan"] == 0 and st["n_noconv"] == 0, st
    inc_e = np.stack([e.get_f(m).astype(np.float64) - F[m] for m in range(M)])
    inc_o = np.stack([o.get_f(m) - F[m] for m in range(M)])
    scale = np.max(np.abs(inc_o))
    err = np.max(np.abs(inc_e - inc_o)) / scale
    cfg32, e32, _, _, _ = make_case(nx, M, p, L, 1.1)
    e32.assimilate(cfg32.iiter, *obs)
    inc_32 = np.stack([e32.get_f(m).astype(np.float64) - F[m] for m in range(M)])
    err32 = np.max(np.abs(inc_e - inc_32)) / scale
    print(f"tcgen05 Gram nx={nx} M={M} p={p} L={L}: increment error {err:.2e} of the largest (vs SIMT Gram {err32:.2e})")
    assert scale > 1e-6 and err < 1e-3


def test_tensor_core_gram_limits():
    # p^2 not a multiple of the points per tile; not a DA run; a 243-slot window (LETKF_RLOC_LEN = 2)
    # whose operands do not fit in shared memory
    for kw in (dict(mode="DA_LETKF", M=16, p=2, L=0), dict(mode="DA_LETKF", M=16, p=1, L=0),
               dict(mode="NATURE", M=16, p=4, L=1), dict(mode="DA_LETKF", M=16, p=4, L=2)):
        with pytest.raises(lbl.LblError) as ei:
            lbl.Ensemble(lbl.config_default(kw["mode"], 64, kw["M"], da_xyprune=kw["p"], letkf_rloc_len=kw["L"],
                                            gram=lbl.GRAM_TF32X3))
        assert ei.value.code == -8


def test_bf16_gram_limits():
    for kw in (dict(mode="DA_LETKF", M=16), dict(mode="NATURE", M=64)):
        with pytest.raises(lbl.LblError) as ei:
            lbl.Ensemble(lbl.config_default(kw["mode"], 64, kw["M"], gram=lbl.GRAM_BF16))
        assert ei.value.code == -8


def moments(f):
    ex = np.array([(q % 3) - 1 for q in range(9)], float)
    ey = np.array([(q // 3) - 1 for q in range(9)], float)
    f = f.astype(np.float64)
    r = f.sum(0)
    return np.tensordot(ex * 20, f, axes=(0, 0)) / r, np.tensordot(ey * 20, f, axes=(0, 0)) / r, r


def test_analysis_reduces_error():
    """With observations consistent with the observation operator the filter pulls
    the ensemble mean toward the truth.  (The reference's H(x) takes moments of the
    post-collision populations, letkf.cu:172-180, while its observation files hold the
    post-stream macros; the forcing impulse between the two biases young flows.)"""
    cfg = lbl.config_default("DA_LETKF", 64, 16, da_xyprune=2, letkf_covinf=1.1, obs_error_u=0.002,
                             obs_error_rho=1e-4, daprune=1, compat_stale_v=0)
    e = lbl.Ensemble(cfg)
    e.init(0)
    e.update(0, 30)
    nat = lbl.Ensemble(lbl.config_default("NATURE", 64, 1))
    nat.init(0)
    nat.update(0, 30)
    ut, vt, rt = moments(nat.get_f(0))
    rng = np.random.default_rng(3)
    obs = [(a + s * rng.standard_normal(a.shape)).astype(np.float32) for a, s in ((rt, 1e-4), (ut, 2e-3), (vt, 2e-3))]

    def rmse():
        us, vs = zip(*[moments(e.get_f(m))[:2] for m in range(16)])
        return float(np.sqrt(np.mean((np.mean(us, 0) - ut) ** 2 + (np.mean(vs, 0) - vt) ** 2)))

    before = rmse()
    e.assimilate(cfg.iiter, *obs)
    after = rmse()
    assert after < 0.8 * before, (before, after)


def test_stale_v_after_analysis():
    for stale in (1, 0):
        cfg, e, obs, _, _ = make_case(64, 4, 2, 0, 1.0, compat_stale_v=stale)
        e.assimilate(cfg.iiter, *obs)
        f = e.get_f(1).astype(np.float64)
        r, u, v, _ = e.get_fields(1)
        ey = np.array([(q // 3) - 1 for q in range(9)], float)
        ex = np.array([(q % 3) - 1 for q in range(9)], float)
        v_mom = np.tensordot(ey * 20, f, axes=(0, 0)) / f.sum(0)
        u_mom = np.tensordot(ex * 20, f, axes=(0, 0)) / f.sum(0)
        np.testing.assert_allclose(u, u_mom, rtol=1e-4, atol=1e-6)
        if stale:
            assert np.max(np.abs(v - v_mom)) > 1e-6  # letkf.cu:340-355 leaves v untouched
        else:
            np.testing.assert_allclose(v, v_mom, rtol=1e-4, atol=1e-6)


def test_gate_skips_off_cycle():
    cfg, e, obs, _, _ = make_case(64, 4, 2, 0, 1.0)
    e2 = lbl.Ensemble(lbl.config_default("DA_LETKF", 64, 4, da_xyprune=2, daprune=5))
    e2.init(0)
    g0 = e2.get_f(0)
    e2.assimilate(e2.cfg.iiter * 3, *obs)  # step 3 is not a multiple of DAPRUNE=5
    np.testing.assert_array_equal(e2.get_f(0), g0)


def test_nan_observation_is_reported():
    cfg, e, (ro, uo, vo), _, _ = make_case(64, 4, 2, 0, 1.0)
    uo = uo.copy()
    uo[0, 0] = np.nan  # an observed site
    with pytest.raises(lbl.LblError) as ei:
        e.assimilate(cfg.iiter, ro, uo, vo)
    assert ei.value.code == -5


def test_cycle_graph_equals_separate_calls():
    cfg, a, obs, _, _ = make_case(64, 8, 4, 1, 1.1)
    b = lbl.Ensemble(cfg)
    b.init(0)
    b.update(0, 30)
    t = cfg.iiter
    a.cycle_async(t, *obs, 20)
    a.sync()
    b.assimilate(t, *obs)
    b.update(t, 20)
    for m in range(cfg.n_ens):
        np.testing.assert_array_equal(a.get_f(m), b.get_f(m))
    # NULL observation pointers reuse the observations already on the device
    c = lbl.Ensemble(cfg)
    c.init(0)
    d = lbl.Ensemble(cfg)
    d.init(0)
    for x in (c, d):
        x.update(0, 30)
        x.cycle_async(t, *obs, 5)
    c.cycle_async(2 * t, None, None, None, 5)
    d.cycle_async(2 * t, *obs, 5)
    c.sync()
    d.sync()
    for m in range(cfg.n_ens):
        np.testing.assert_array_equal(c.get_f(m), d.get_f(m))


def test_letkf_timer_tags():
    cfg, e, obs, _, _ = make_case(64, 4, 2, 0, 1.0)
    e.assimilate(cfg.iiter, *obs)
    csv = e.timer_csv(lbl.TIMER_LETKF)
    assert csv.startswith("#tag,sec\n")
    tags = [line.split(",")[0] for line in csv.strip().split("\n")[1:]]
    for tag in ("pack_xk", "pack_yk", "mpi_yk", "load_obs", "set_yo", "mpi_xk", "solve_comm_ovlp",
                "mpi_barrier", "solve", "mpi_xsol", "update_xk", "lbm2euler"):
        assert tag in tags
    assert tags == sorted(tags)  # std::map order (util/timer.hpp:66-72)


def test_cycle_phase_events():
    cfg, e, obs, _, _ = make_case(64, 8, 4, 1, 1.1)
    t = cfg.iiter
    e.cycle_async(t, *obs, 20)
    ana, fc = e.cycle_phases()
    assert ana > 0 and fc > 0
    e.update(2 * t, 10)  # a forecast-only graph has no analysis phase
    ana, fc = e.cycle_phases()
    assert ana == 0 and fc > 0
    fresh = lbl.Ensemble(cfg)
    with pytest.raises(lbl.LblError):
        fresh.cycle_phases()  # nothing launched yet


def test_cycle_longer_than_one_forcing_buffer():
    """At 1024^2 one graph holds 32 steps of forcing: a 45-step cycle is split over graphs
    and still equals the analysis followed by 45 separate steps."""
    kw = dict(da_xyprune=8, letkf_rloc_len=0, letkf_covinf=1.1, obs_error_u=0.002, obs_error_rho=1e-4, daprune=1)
    cfg = lbl.config_default("DA_LETKF", 1024, 2, **kw)
    a, b = lbl.Ensemble(cfg), lbl.Ensemble(cfg)
    rng = np.random.default_rng(3)
    obs = []
    for s_ in (1e-4, 2e-3, 2e-3):
        o_ = np.full((1024, 1024), np.nan, np.float32)
        o_[::8, ::8] = (1.0 if s_ == 1e-4 else 0.0) + s_ * rng.standard_normal((128, 128))
        obs.append(o_)
    for x in (a, b):
        x.init(0)
        x.update(0, 3)
    t = cfg.iiter
    a.cycle_async(t, *obs, 45)
    a.sync()
    b.assimilate(t, *obs)
    b.update(t, 45)
    for m in range(2):
        np.testing.assert_array_equal(a.get_f(m), b.get_f(m))
