"""The oracle's OBSERVE restatement (io.cu:160-246) against an independent Python
restatement: std::mt19937(334) raw words (numpy's legacy MT19937 seeding is the
same init_genrand), libstdc++'s polar normal_distribution<float>, the rho,u,v
draw order per cell, observed vorticity before NaN pruning, and the NaN lattice."""
import numpy as np
import pytest

import lbl
import oracle


class PolarNormal:
    """libstdc++ normal_distribution<float> (bits/random.tcc, polar method) on mt19937."""

    def __init__(self, seed):
        self.rs = np.random.RandomState(seed)
        self.saved = None

    def _u(self):
        w = np.float32(self.rs.randint(0, 2**32, dtype=np.uint64))
        r = np.float32(w / np.float32(4294967296.0))
        return r if r < 1 else np.nextafter(np.float32(1), np.float32(0))

    def __call__(self):
        if self.saved is not None:
            s, self.saved = self.saved, None
            return s
        while True:
            x = np.float32(np.float64(np.float32(2.0) * self._u()) - 1.0)
            y = np.float32(np.float64(np.float32(2.0) * self._u()) - 1.0)
            r2 = np.float32(x * x + y * y)
            if not (r2 > 1.0 or r2 == 0.0):
                break
        mult = np.sqrt(np.float32(np.float32(-2) * np.log(r2) / r2))
        self.saved = np.float32(x * mult)
        return np.float32(y * mult)


def test_observation_noise_and_pruning():
    cfg = lbl.config_default("OBSERVE", 64, 1, da_xyprune=4, obs_error_rho=0.01, obs_error_u=0.1)
    o = oracle.Oracle(cfg)
    rng = np.random.default_rng(1)
    r = (1 + 0.001 * rng.standard_normal((64, 64))).astype(np.float32)
    u = rng.standard_normal((64, 64)).astype(np.float32)
    v = rng.standard_normal((64, 64)).astype(np.float32)
    ro, uo, vo, wo = o.observe(r, u, v)
    # noise restated in Python for the whole field (draw order rho, u, v per cell)
    pn = PolarNormal(334)
    rr, uu, vv = (np.empty(64 * 64, np.float32) for _ in range(3))
    for ij in range(64 * 64):
        rr[ij] = np.float32(r.flat[ij] + np.float32(0.01) * pn())
        uu[ij] = np.float32(u.flat[ij] + np.float32(0.1) * pn())
        vv[ij] = np.float32(v.flat[ij] + np.float32(0.1) * pn())
    keep = np.zeros((64, 64), bool)
    keep[::4, ::4] = True
    for got, want in ((ro, rr), (uo, uu), (vo, vv)):
        assert np.all(np.isnan(got[~keep]))
        np.testing.assert_allclose(got[keep], want.reshape(64, 64)[keep], rtol=2e-7, atol=2e-7)
    # observed vorticity is taken from the noisy fields before pruning (io.cu:355-376)
    w = oracle.vorticity(cfg, uu, vv)
    assert np.all(np.isnan(wo[~keep]))
    np.testing.assert_allclose(wo[keep], w[keep], rtol=1e-5, atol=1e-4)


def test_engine_persists_between_outputs():
    cfg = lbl.config_default("OBSERVE", 32, 1, da_xyprune=1)
    o = oracle.Oracle(cfg)
    z = np.zeros((32, 32), np.float32)
    a = o.observe(z + 1, z, z)
    b = o.observe(z + 1, z, z)
    assert not np.array_equal(a[1], b[1])  # the static engine keeps running (io.cu:321)
    o2 = oracle.Oracle(cfg)
    np.testing.assert_array_equal(o2.observe(z + 1, z, z)[1], a[1])


def test_vorticity_central_differences():
    cfg = lbl.config_default("NATURE", 64, 1)
    x = np.arange(64) * cfg.h_ref / 63
    u = np.tile(np.sin(x)[:, None], (1, 64)).astype(np.float32)  # u(y)
    v = np.tile(np.cos(x)[None, :], (64, 1)).astype(np.float32)  # v(x)
    w = oracle.vorticity(cfg, u, v)
    dx = np.float32(cfg.h_ref / 63)
    vx = (np.roll(v, -1, 1) - np.roll(v, 1, 1)) / (2 * dx)
    uy = (np.roll(u, -1, 0) - np.roll(u, 1, 0)) / (2 * dx)
    np.testing.assert_allclose(w, vx - uy, rtol=1e-6, atol=1e-6)
