"""The oracle's DA_NUDGING (nudging.cu:40-143) against an independent numpy
statement of the same update: bilinear interpolation of the p-lattice
observations (periodic corners), DA_QUADRA masks, DA_OBS_RUV / DA_OBS_UV, and
f <- alpha feq(rho_o, u_o, v_o) + (1 - alpha) f."""
import numpy as np
import pytest

import lbl
import oracle

EX = np.array([(q % 3) - 1 for q in range(9)], float)
EY = np.array([(q // 3) - 1 for q in range(9)], float)
W = np.array([1 / 36, 1 / 9, 1 / 36, 1 / 9, 4 / 9, 1 / 9, 1 / 36, 1 / 9, 1 / 36])


def feq(r, u, v, c):
    uc = (u[None] * EX[:, None, None] + v[None] * EY[:, None, None]) / c
    uu = (u * u + v * v)[None] / (c * c)
    return r[None] * W[:, None, None] * (1 + 3 * uc + 4.5 * uc * uc - 1.5 * uu)


def interp(a, p):
    """Bilinear interpolation of the p-lattice values of a (periodic)."""
    ny, nx = a.shape
    j, i = np.mgrid[0:ny, 0:nx]
    iw, js = (i // p) * p, (j // p) * p
    ir, jr = (i - iw) / p, (j - js) / p
    g = lambda ii, jj: a[jj % ny, ii % nx].astype(np.float64)
    return ((1 - ir) * (1 - jr) * g(iw, js) + ir * (1 - jr) * g(iw + p, js) + (1 - ir) * jr * g(iw, js + p)
            + ir * jr * g(iw + p, js + p))


def observations(nx, p, seed):
    rng = np.random.default_rng(seed)
    ro = np.full((nx, nx), np.nan, np.float32)
    uo, vo = ro.copy(), ro.copy()
    ro[::p, ::p] = 1 + 0.01 * rng.standard_normal((nx // p, nx // p))
    uo[::p, ::p] = 0.05 * rng.standard_normal((nx // p, nx // p))
    vo[::p, ::p] = 0.05 * rng.standard_normal((nx // p, nx // p))
    return ro, uo, vo


@pytest.mark.parametrize("p,quadra,ruv", [(1, 0, 1), (4, 0, 1), (4, 3, 0), (2, 1, 1), (4, 2, 0)])
def test_oracle_nudging_matches_numpy(p, quadra, ruv):
    nx, M, alpha = 32, 2, 0.1
    cfg = lbl.config_default("DA_NUDGING", nx, M, da_xyprune=p, da_quadra=quadra, da_obs_ruv=ruv,
                             da_nud_rate=alpha)
    o = oracle.Oracle(cfg)
    o.init(0)
    o.step(3)
    f0 = [o.get_f(m) for m in range(M)]
    rm = [o.macros(m)[0] for m in range(M)]
    ro, uo, vo = observations(nx, p, 7)
    o.nudge(ro, uo, vo)
    a = float(np.float32(alpha))
    c = float(np.float32(cfg.u_ref) / np.float32(cfg.cfl))
    mask = np.ones((nx, nx), bool)
    if quadra % 2 == 1:
        mask[:, nx // 2:] = False
    if quadra >= 2:
        mask[nx // 2:, :] = False
    for m in range(M):
        r = interp(ro, p) if ruv else rm[m]
        want = a * feq(r, interp(uo, p), interp(vo, p), c) + (1 - a) * f0[m]
        want = np.where(mask[None], want, f0[m])
        np.testing.assert_allclose(o.get_f(m), want, rtol=1e-12, atol=0)
    o.close()
