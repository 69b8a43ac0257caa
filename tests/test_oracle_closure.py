"""CPU checks of the closure oracle (oracle/closure_oracle.py and the C++ stepping
oracle's closure): gradient against finite differences, BF16 rounding against
torch, known-answer features and targets, and the two oracles against each other."""
import numpy as np
import pytest

import closure_oracle as co
import oracle


def _params(seed, scale=0.3):
    rng = np.random.default_rng(seed)
    return (co.init_params(seed) + rng.normal(0, scale, co.N_PARAMS)).astype(np.float32)


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = _params(3).astype(np.float64)
    x = rng.normal(0, 1, (48, 6))
    t = rng.uniform(0, 3, 48)
    _, g = co.loss_and_grad(p, x, t, contract=False)
    eps = 1e-6
    fd = np.empty_like(p)
    for k in range(p.size):
        e = np.zeros_like(p)
        e[k] = eps
        fd[k] = (co.loss_and_grad(p + e, x, t, False)[0] - co.loss_and_grad(p - e, x, t, False)[0]) / (2 * eps)
    assert np.max(np.abs(fd - g)) <= 1e-7 * np.max(np.abs(g))


def test_bf16_rounding_matches_torch():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(1)
    x = np.concatenate([rng.normal(0, 10, 10000), rng.uniform(-1, 1, 10000),
                        # exact ties between two BF16 values: both rounding directions
                        (np.arange(1, 200) * 2.0 ** -8 + 2.0 ** -9) * 3.0]).astype(np.float32)
    ref = torch.from_numpy(x).to(torch.bfloat16).to(torch.float64).numpy()
    np.testing.assert_array_equal(co.bf16(x), ref)


def test_features_known_values():
    a = 0.3
    # solid rotation u = -a y, v = a x: no strain
    x, smag = co.features(0.0, -a, a, 0.0, dx=0.1, nu_ref=1e-3, dx_ref=0.1)
    assert smag[0] == 0 and x[0, 0] == 0 and x[0, 2] == pytest.approx(1.0) and x[0, 4] == 1.0
    assert x[0, 5] == pytest.approx(np.arcsinh(0.1 * 0.1 / 1e-3 * 2 * a))
    # pure strain u = a x, v = -a y: no rotation, no divergence
    x, smag = co.features(a, 0.0, 0.0, -a, dx=0.1, nu_ref=1e-3, dx_ref=0.2)
    assert smag[0] == pytest.approx(2 * a) and x[0, 1] == 0 and x[0, 2] == pytest.approx(-1.0)
    assert x[0, 3] == pytest.approx(0.0) and x[0, 4] == 0.5 and x[0, 5] == 0


def test_targets_known_answers():
    n, f = 64, 4
    y = np.arange(n)[:, None] * np.ones((1, n))
    # parallel shear u(y): the deviatoric subgrid stress has no component along S
    u = np.sin(2 * np.pi * y / n)
    x, m = co.samples(u, np.zeros_like(u), f, h=0.4, cs=0.1, dx=0.4, nu_ref=1e-3, dx_ref=0.4)
    strained = x[:, 0] > 1e-6
    assert strained.sum() > 100 and np.all(m[strained] == 0)
    # uniform flow: no strain, the target keeps Smagorinsky
    _, m = co.samples(np.full((n, n), 0.05), np.full((n, n), -0.02), f, 0.4, 0.1, 0.4, 1e-3, 0.4)
    assert np.all(m == 1.0)


def test_cpp_and_numpy_oracles_agree():
    rng = np.random.default_rng(2)
    p = _params(5)
    x = rng.normal(0, 2, (400, 6))
    np.testing.assert_allclose(oracle.closure_forward(p, x), co.forward(p, x)[0], rtol=1e-12, atol=1e-12)


def test_stepping_oracle_with_constant_multiplier_is_rescaled_smagorinsky():
    """W3 = 0 makes the multiplier the constant softplus(b3): the closure run equals
    a plain run whose Smagorinsky constant is scaled by sqrt(m)."""
    import lbl  # the config mirror (no GPU call)

    p = _params(7)
    p[co.W3:co.B3] = 0
    p[co.B3] = 1.3
    m = float(co.forward(p, np.zeros((1, 6)))[0][0])
    cfg = lbl.config_default("NATURE", 32, 1, cs=0.5, ic_amp=0.05)
    a, b = oracle.Oracle(cfg), None
    cfg2 = cfg.copy()
    cfg2.cs = cfg.cs * np.sqrt(m)
    b = oracle.Oracle(cfg2)
    a.init(0)
    b.init(0)
    a.set_closure(p)
    for _ in range(5):
        a.step_noforce()
        b.step_noforce()
    np.testing.assert_allclose(a.get_f(0), b.get_f(0), rtol=1e-13, atol=0)
    # the closure changes the run: not the plain Smagorinsky constant
    c = oracle.Oracle(cfg)
    c.init(0)
    for _ in range(5):
        c.step_noforce()
    assert np.max(np.abs(a.get_f(0) - c.get_f(0))) > 1e-9
