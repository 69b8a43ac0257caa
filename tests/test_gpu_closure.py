"""Learned closure on the GPU, through the C ABI, against the closure oracle: the
tensor-core and per-thread inference, the fused forward/backward training kernel,
the training-data generator, the closure inside the stream-collide (against the
FP64 stepping oracle), and training that beats the plain Smagorinsky multiplier."""
import numpy as np
import pytest

import closure_oracle as co
import lbl
import oracle

pytestmark = pytest.mark.gpu


def _params(seed, scale=0.3):
    rng = np.random.default_rng(seed)
    return (co.init_params(seed) + rng.normal(0, scale, co.N_PARAMS)).astype(np.float32)


def _features(n, seed):
    """Rows spread like the generator's: log rates, ratios in [-1, 1], scale, asinh."""
    rng = np.random.default_rng(seed)
    x = np.empty((n, 6), np.float32)
    x[:, 0] = rng.uniform(0, 6, n)
    x[:, 1] = rng.uniform(0, 6, n)
    x[:, 2] = rng.uniform(-1, 1, n)
    x[:, 3] = rng.normal(0, 0.05, n)
    x[:, 4] = rng.choice([0.5, 1.0, 2.0], n)
    x[:, 5] = rng.normal(0, 4, n)
    return x


@pytest.mark.parametrize("path", [0, 1])
def test_inference_matches_oracle(path):
    p = _params(11)
    x = _features(5000, 12)
    want = co.forward(p, x)[0]
    got = lbl.closure_infer(p, x, path=path).astype(np.float64)
    err = np.abs(got - want) / (1 + np.abs(want))
    # path 1: FP32 sums and tanhf; path 0: tensor cores and the MUFU tanh (2^-11),
    # whose result flips some BF16 roundings of the first-layer activations
    # (both: an FP16 rounding of a first-layer activation may flip against FP64)
    tol_max, tol_mean = (2e-3, 1e-5) if path == 1 else (2e-2, 2e-3)
    assert err.max() < tol_max and err.mean() < tol_mean, (err.max(), err.mean())


def test_inference_ragged_count():
    """n not a multiple of the warp: the padded lanes leave the real rows alone."""
    p = _params(13)
    x = _features(37, 14)
    np.testing.assert_allclose(lbl.closure_infer(p, x, 0), lbl.closure_infer(p, np.vstack([x, x[:27]]), 0)[:37],
                               rtol=0, atol=0)


def test_gradient_matches_oracle():
    p = _params(21)
    x = _features(3000, 22)
    t = np.random.default_rng(23).uniform(0, 4, 3000).astype(np.float32)
    loss, g = lbl.closure_grad(p, x, t)
    want_loss, want_g = co.loss_and_grad(p, x, t, contract=True)
    assert loss == pytest.approx(want_loss, rel=1e-5)
    assert np.linalg.norm(g - want_g) < 1e-3 * np.linalg.norm(want_g)


def _fine_cfg(nx=128, M=2):
    return lbl.config_default("NATURE", nx, M, ic_kind=lbl.IC_K4EXP, ic_amp=1.0, cs=0.1, tau=0.55)


def _nu(cfg):
    """The run's molecular viscosity as the engine derives it (FP32 constants)."""
    c = np.float32(cfg.u_ref) / np.float32(cfg.cfl)
    dt = (np.float32(cfg.h_ref) / np.float32(cfg.ny - 1)) / c
    return float(np.float32((cfg.tau - 0.5) * float(c) * float(c) * float(dt) / 3.0 if cfg.tau > 0 else cfg.nu))


def test_generator_matches_oracle_filter_and_targets():
    cfg = _fine_cfg()
    F, spin, snaps, spacing = 4, 20, 2, 10
    feat, tgt = lbl.closure_generate(cfg, F, spin, snaps, spacing)
    nc = (cfg.nx // F) * (cfg.ny // F)
    assert feat.shape == (nc * cfg.n_ens * snaps, 6)
    e = lbl.Ensemble(cfg)
    e.init(0)
    e.update(0, spin)
    t = spin
    dx_c = cfg.h_ref / (cfg.ny // F - 1)  # the coarse grid's own spacing scales the features
    h = F * float(np.float32(cfg.h_ref) / np.float32(cfg.ny - 1))  # filtered cells lie F fine cells apart
    for s in range(snaps):
        e.update(t, spacing)
        t += spacing
        for m in range(cfg.n_ens):
            _, u, v, _ = e.get_fields(m)
            k = (s * cfg.n_ens + m) * nc
            got_x, got_t = feat[k:k + nc].astype(np.float64), tgt[k:k + nc].astype(np.float64)
            x_o, t_o = co.samples(u, v, F, h, cfg.cs, dx_c, _nu(cfg), cfg.h_ref / 255)
            for j, (rtol, atol) in enumerate([(1e-4, 1e-6), (1e-4, 1e-6), (0, 2e-4), (0, 2e-3), (1e-6, 0),
                                              (1e-4, 1e-6)]):
                np.testing.assert_allclose(got_x[:, j], x_o[:, j], rtol=rtol, atol=atol, err_msg=f"feature {j}")
            dm = np.abs(got_t - t_o)
            assert np.mean(dm < 0.02) > 0.99 and np.median(dm) < 1e-3, (np.mean(dm < 0.02), np.median(dm))


def _lbm_pair(cfg, params, steps):
    """Engine with the closure vs the FP64 oracle with the same network, the engine's
    forcing injected every step; returns (max relative error, the error of the plain
    Smagorinsky oracle)."""
    e = lbl.Ensemble(cfg)
    e.init(0)
    e.set_closure(params)
    orc, plain = oracle.Oracle(cfg), oracle.Oracle(cfg)
    orc.set_closure(params)
    for m in range(cfg.n_ens):
        orc.set_f(m, e.get_f(m))
        plain.set_f(m, e.get_f(m))
    for t in range(steps):
        e.update(t, 1)
        fx, fy = e.force()
        for o in (orc, plain):
            o.set_force(fx, fy)
            o.step_noforce()
    err = max(float(np.max(np.abs(e.get_f(m) - orc.get_f(m)) / np.abs(orc.get_f(m)))) for m in range(cfg.n_ens))
    off = max(float(np.max(np.abs(e.get_f(m) - plain.get_f(m)) / np.abs(plain.get_f(m)))) for m in range(cfg.n_ens))
    return err, off


# cs and the output bias large enough that nu_t is comparable to nu on each grid, so
# that the network moves the populations well above the FP32-vs-FP64 difference
@pytest.mark.parametrize("nx,M,cs,b3", [(64, 2, 0.5, 0.0), (256, 1, 4.0, 2.0)])
def test_closure_stream_collide_matches_oracle(nx, M, cs, b3):
    cfg = lbl.config_default("NATURE", nx, M, cs=cs)
    p = _params(31)
    p[co.B3] += b3
    err, off = _lbm_pair(cfg, p, 10)
    assert err < 1e-5, err
    assert off > 20 * err, (off, err)  # the check sees the network, not just Smagorinsky


def test_closure_off_restores_smagorinsky_bitwise():
    cfg = lbl.config_default("NATURE", 64, 2, cs=0.5)
    a, b = lbl.Ensemble(cfg), lbl.Ensemble(cfg)
    a.init(0)
    b.init(0)
    a.set_closure(_params(41))
    a.update(0, 3)
    a.set_closure(None)
    b.set_closure(_params(41))
    b.update(0, 3)
    b.set_closure(None)
    a.update(3, 5)
    b.update(3, 5)
    np.testing.assert_array_equal(a.get_f(0), b.get_f(0))
    c = lbl.Ensemble(cfg)
    c.init(0)
    c.update(0, 8)
    assert np.max(np.abs(a.get_f(0) - c.get_f(0))) > 0  # the 3 closure steps left their mark


def test_closure_rejects_the_tma_stream_collide():
    e = lbl.Ensemble(lbl.config_default("NATURE", 64, 1, lbm_variant=lbl.LBM_TMA))
    with pytest.raises(lbl.LblError):
        e.set_closure(_params(1))
    bad = _params(1)
    bad[5] = np.nan
    f = lbl.Ensemble(lbl.config_default("NATURE", 64, 1))
    with pytest.raises(lbl.LblError):
        f.set_closure(bad)


def test_training_lowers_the_loss_below_smagorinsky():
    cfg = _fine_cfg(256, 4)
    feat, tgt = lbl.closure_generate(cfg, 4, 200, 4, 50)
    n = len(tgt)
    rng = np.random.default_rng(0)
    idx = rng.permutation(n)
    tr, te = idx[: n * 3 // 4], idx[n * 3 // 4:]
    w, curve = lbl.closure_train(feat[tr], tgt[tr], iters=600, batch=4096, lr=3e-3, seed=5)
    assert np.all(np.isfinite(curve)) and curve[-50:].mean() < curve[:10].mean()
    m_test = lbl.closure_infer(w, feat[te])
    mse_mlp = float(np.mean((m_test - tgt[te]) ** 2))
    mse_smag = float(np.mean((1.0 - tgt[te]) ** 2))
    mse_const = float(np.var(tgt[te]))
    assert mse_mlp < mse_smag and mse_mlp < mse_const, (mse_mlp, mse_smag, mse_const)


def test_held_multiplier_equals_evaluation_for_a_constant_network():
    """lbl_set_closure_refresh: between two evaluations of the network each cell keeps its
    multiplier.  A network whose output does not depend on its inputs (every weight zero,
    m = softplus(b3)) gives the same multiplier either way, so a run that evaluates it
    every 5 steps must equal, bit for bit, a run that evaluates it every step: the held
    path recomputes |S| exactly as the evaluating path does."""
    w = np.zeros(lbl.CLOSURE_PARAMS, np.float32)
    w[-1] = 0.7  # b3
    out = []
    for k in (1, 5):
        e = lbl.Ensemble(lbl.config_default("NATURE", 64, 2, cs=0.1, tau=0.51))
        e.init(0)
        e.set_closure(w)
        e.set_closure_refresh(k)
        e.update(0, 23)
        out.append([e.get_f(m) for m in range(2)])
        e.close()
    for m in range(2):
        np.testing.assert_array_equal(out[0][m], out[1][m])


@pytest.mark.parametrize("storage", [0, 1])
def test_held_steps_vector_kernel_is_bit_identical(storage):
    """The held-multiplier steps run the two-column vector-load kernel when the context's
    plain steps do (LBL_LBM_AUTO at 256 columns) and lbm_step_kernel's CLH form under
    LBL_LBM_DIRECT: same populations bit for bit, FP32 and FP16 storage."""
    from lbl import closure
    w, meta = closure.load_params()
    out = {}
    for v in (lbl.LBM_DIRECT, lbl.LBM_AUTO):
        e = lbl.Ensemble(lbl.config_default("NATURE", 256, 2, cs=0.1, tau=0.51, ic_kind=lbl.IC_K4EXP, ic_amp=1.0,
                                            lbm_variant=v, storage=storage))
        e.init(0)
        e.set_closure(w, meta["nu_ref"], meta["dx_ref"])
        e.set_closure_refresh(10)
        e.update(0, 47)
        out[v] = [e.get_f(m) for m in range(2)] + [a for m in range(2) for a in e.get_fields(m)[:3]]
        e.close()
    for a, b in zip(out[lbl.LBM_DIRECT], out[lbl.LBM_AUTO]):
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("refresh", [10, 20])
def test_held_multiplier_follows_the_network(refresh):
    """With the trained network, holding the multipliers for 10 or 20 steps stays close
    to evaluating every step (populations within 1e-4 relative after 100 steps; they
    differ, since m changes from step to step)."""
    from lbl import closure
    w, meta = closure.load_params()
    out = []
    for k in (1, refresh):
        e = lbl.Ensemble(lbl.config_default("NATURE", 256, 2, cs=0.1, tau=0.51, ic_kind=lbl.IC_K4EXP, ic_amp=1.0))
        e.init(0)
        e.set_closure(w, meta["nu_ref"], meta["dx_ref"])
        e.set_closure_refresh(k)
        e.update(0, 100)
        out.append(np.stack([e.get_f(m) for m in range(2)]).astype(np.float64))
        e.close()
    rel = np.max(np.abs(out[1] - out[0]) / np.abs(out[0]))
    print(f"refresh {refresh} against 1 after 100 steps: {rel:.2e}")
    assert np.all(np.isfinite(out[1])) and 0 < rel < 1e-4
    with pytest.raises(lbl.LblError):
        lbl.Ensemble(lbl.config_default("NATURE", 64, 1)).set_closure_refresh(0)
