"""Pin the CPU oracle against the reference itself.

The fixtures in tests/golden/ref_lbm_id*.npz were produced by running the
reference's own src/lbm.cu + src/data.cu (oracle/_ref/ref_lbm) on a B200
(tests/golden/make_golden.py).  The oracle, given the same cuRAND normals,
must reproduce the reference's initial condition, forcing table, forcing field,
cursor arithmetic and 1/10/100-step populations.
"""
import numpy as np
import pytest

from conftest import checksums, golden, rel_err

import lbl
import oracle

N_MODES = 29


@pytest.fixture(scope="module")
def g0():
    return golden("ref_lbm_id0.npz")


@pytest.fixture(scope="module")
def cfg():
    return lbl.config_default("NATURE", 256, 1)


def normals_of_call(g, call):
    n4 = 4 * N_MODES
    return g["normals_head"][call * n4:(call + 1) * n4]


def test_force_mode_table_bit_exact(g0, cfg):
    kx, ky, amp = oracle.force_modes(cfg)
    assert kx.size == N_MODES
    np.testing.assert_array_equal(kx, g0["kx"])
    np.testing.assert_array_equal(ky, g0["ky"])
    np.testing.assert_array_equal(amp, g0["amp"])


@pytest.mark.parametrize("name,seed", [("ref_lbm_id0.npz", 0), ("ref_lbm_id334.npz", 334)])
def test_initial_condition(name, seed, cfg):
    g = golden(name)
    rows = g["rows"]
    r, u, v, f = oracle.ic_fields(cfg, seed)
    # FP64 cos of glibc vs CUDA may differ in the last ulp of single terms: allow 2 float ulps
    for var, a in (("r", r), ("u", u), ("v", v)):
        np.testing.assert_array_max_ulp(a[rows], g[f"s0_rows_{var}"], maxulp=2)
    np.testing.assert_array_max_ulp(f[:, rows, :], g["s0_rows_f"], maxulp=2)
    for var, a in (("f", f), ("u", u), ("v", v)):
        np.testing.assert_allclose(checksums(a), g[f"s0_sums_{var}"], rtol=1e-6)


def test_forcing_cursor(g0):
    # two update_forces calls at init, then one per step (data.cu:240-247)
    for s in g0["steps"]:
        assert int(g0[f"s{s}_cursor"][0]) == (s + 1) * 4 * N_MODES


def test_forcing_field(g0, cfg):
    o = oracle.Oracle(cfg)
    for s in g0["steps"]:
        fx, fy = o.force(normals_of_call(g0, s + 1))
        rows = g0["rows"]
        # the reference uses fast-math __sinf/__cosf (|err| ~ 1e-6 at |theta| <= 20)
        assert rel_err(fx[rows], g0[f"s{s}_rows_fx"]) < 2e-5
        assert rel_err(fy[rows], g0[f"s{s}_rows_fy"]) < 2e-5
        w = np.random.default_rng(12345).random(fx.size).reshape(fx.shape)
        scale = np.array([(fx * fx).sum(), np.abs(fx * w).sum()])
        assert np.all(np.abs(checksums(fx)[1:] - g0[f"s{s}_sums_fx"][1:]) < 2e-5 * scale)


def test_lbm_steps_against_reference(g0, cfg):
    """FP64 oracle vs the reference's FP32 populations after 1, 10 and 100 steps.

    The reference's own FP32 rounding (f stored in float, omega ~ 2 so rounding
    errors are not damped) separates it from FP64 by 6e-7, 3e-6 and 1.2e-5 after
    1, 10 and 100 steps; the bound is 2e-5 (the FP32 engine vs the FP32 reference
    is held to 1e-5 in tests/test_gpu_lbm.py)."""
    o = oracle.Oracle(cfg)
    o.init(0)
    rows = g0["rows"]
    done = 0
    for s in sorted(int(x) for x in g0["steps"]):
        while done < s:
            o.step(1, normals_of_call(g0, done + 2))
            done += 1
        f = o.get_f(0)
        ref = g0[f"s{s}_rows_f"].astype(np.float64)
        err = np.max(np.abs(f[:, rows, :] - ref) / np.abs(ref))
        assert err < 2e-5, (s, err)
        # the reference's FP32 total mass drifts by 1.5e-6 relative in 100 steps
        np.testing.assert_allclose(checksums(f), g0[f"s{s}_sums_f"], rtol=1e-5)
        if s > 0:
            r, u, v = o.macros(0)
            assert rel_err(u[rows], g0[f"s{s}_rows_u"]) < 1e-3
            assert rel_err(v[rows], g0[f"s{s}_rows_v"]) < 1e-3
            assert rel_err(r[rows], g0[f"s{s}_rows_r"]) < 1e-5
