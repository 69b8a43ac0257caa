"""The oracle's LETKF analysis (letkf.cu / letkf_solver.h restated) against an
independent formulation: the Kalman-gain form of the ensemble update with the
localised R, and the symmetric square root of the analysis covariance from
numpy's eigh.  Also: window geometry and Gaspari-Cohn weights, and the limits
(no information -> analysis == forecast)."""
import math

import numpy as np
import pytest

import lbl
import oracle

C = 20.0  # u_ref / cfl


def gc(d):
    if d <= 0:
        return 1.0
    if d <= 1:
        return -d**5 / 4 + d**4 / 2 + 5 * d**3 / 8 - 5 * d**2 / 3 + 1
    if d <= 2:
        return d**5 / 12 - d**4 / 2 + 5 * d**3 / 8 + 5 * d**2 / 3 - 5 * d + 4 - 2 / (3 * d)
    return 0.0


def geometry(p, L):
    if L <= 0:
        return (p - 1, 0 if p == 1 else 2, 0 if p == 1 else 1, 1 if p == 1 else 4)
    return (L * p, 2 * L, 0, 4 * L + 1)


def window(cfg, i, j):
    p, L = cfg.da_xyprune, cfg.letkf_rloc_len
    dloc, nl, off, nox = geometry(p, L)
    out = []
    for b in range(nox):
        for a in range(nox):
            io = (i // p + a - (nl - off)) * p
            jo = (j // p + b - (nl - off)) * p
            di, dj = i - io, j - jo
            valid = not (abs(di) > nl * p or abs(dj) > nl * p)
            g = gc(math.sqrt(di * di + dj * dj) / (dloc + 1e-6)) if p > 1 else 1.0
            out.append(((io + cfg.nx) % cfg.nx, (jo + cfg.ny) % cfg.ny, valid, g))
    return out


def moments(f):
    rho = f.sum(axis=0)
    ex = np.array([(q % 3) - 1 for q in range(9)], float)
    ey = np.array([(q // 3) - 1 for q in range(9)], float)
    u = np.tensordot(ex * C, f, axes=(0, 0)) / rho
    v = np.tensordot(ey * C, f, axes=(0, 0)) / rho
    return u, v, rho


def kalman_point(cfg, F, obs, i, j):
    """ETKF at one point written as the Kalman-gain update + symmetric square root."""
    M = cfg.n_ens
    beta = cfg.letkf_covinf
    H = [moments(F[m]) for m in range(M)]  # (u, v, rho) per member
    rows, yo, w = [], [], []
    for (io, jo, valid, g) in window(cfg, i, j):
        if not valid:
            continue
        for var, sig in ((0, cfg.obs_error_u), (1, cfg.obs_error_u), (2, cfg.obs_error_rho)):
            wt = g / sig**2
            if wt <= 0:
                continue
            rows.append([H[m][var][jo, io] for m in range(M)])
            yo.append(obs[var][jo, io])
            w.append(wt)
    Y = np.array(rows)
    yo = np.array(yo)
    R = np.diag(1.0 / np.array(w))
    X = F[:, :, j, i].T  # 9 x M
    xbar, ybar = X.mean(1), Y.mean(1)
    dX, dY = X - xbar[:, None], Y - ybar[:, None]
    K = dX @ dY.T @ np.linalg.inv(dY @ dY.T + (M - 1) / beta * R)
    xa = xbar + K @ (yo - ybar)
    Pt = np.linalg.inv((M - 1) / beta * np.eye(M) + dY.T @ np.diag(w) @ dY)
    lam, V = np.linalg.eigh(Pt)
    W = math.sqrt(M - 1) * (V * np.sqrt(lam)) @ V.T
    return xa[:, None] + dX @ W  # 9 x M


@pytest.fixture(scope="module")
def setup():
    cfg = lbl.config_default("DA_LETKF", 32, 8, da_xyprune=4, letkf_rloc_len=1, letkf_covinf=1.1,
                             obs_error_u=0.003, obs_error_rho=1e-5)
    o = oracle.Oracle(cfg)
    o.init(0)
    rng = np.random.default_rng(7)
    o.step(5, rng.normal(0, 0.84, 4 * 29 * 5).astype(np.float32))
    F = np.stack([o.get_f(m) for m in range(cfg.n_ens)])
    nat = oracle.Oracle(lbl.config_default("NATURE", 32, 1))
    nat.init(0)
    fn = nat.get_f(0)
    un, vn, rn = moments(fn)
    obs = (un + 0.003 * rng.standard_normal(un.shape), vn + 0.003 * rng.standard_normal(un.shape),
           rn + 1e-5 * rng.standard_normal(un.shape))
    return cfg, o, F, obs


def test_window_weights_match_geometry(setup):
    cfg, o, _, _ = setup
    for (i, j) in ((0, 0), (5, 3), (31, 30), (17, 8)):
        for b in range(5):
            for a in range(5):
                w, valid = o.obs_weight(i, j, a, b, 0)
                io, jo, v2, g = window(cfg, i, j)[a + 5 * b]
                assert valid == v2
                assert math.isclose(w, g / cfg.obs_error_u**2, rel_tol=1e-9, abs_tol=1e-9)  # GC cancels near d=2


def test_analysis_matches_kalman_gain_form(setup):
    cfg, o, F, obs = setup
    o2 = oracle.Oracle(cfg)
    for m in range(cfg.n_ens):
        o2.set_f(m, F[m].astype(np.float32))
    F32 = np.stack([o2.get_f(m) for m in range(cfg.n_ens)])
    u_o, v_o, r_o = (np.asarray(a, np.float32) for a in obs)
    sweeps = o2.assimilate(r_o, u_o, v_o)
    assert 1 <= sweeps < 100
    Fa = np.stack([o2.get_f(m) for m in range(cfg.n_ens)])
    obs32 = tuple(np.asarray(a, np.float64) for a in (u_o, v_o, r_o))
    for (i, j) in ((0, 0), (3, 7), (16, 16), (31, 1), (10, 29)):
        want = kalman_point(cfg, F32, obs32, i, j)
        got = Fa[:, :, j, i].T
        np.testing.assert_allclose(got, want, rtol=1e-9, atol=1e-12)
        # the analysis increment is not trivially zero
        assert np.max(np.abs(got - F32[:, :, j, i].T)) > 1e-7


def test_no_information_leaves_forecast(setup):
    cfg, _, F, obs = setup
    c2 = cfg.copy()
    c2.obs_error_u = 1e9
    c2.obs_error_rho = 1e9
    c2.letkf_covinf = 1.0
    o = oracle.Oracle(c2)
    for m in range(c2.n_ens):
        o.set_f(m, F[m].astype(np.float32))
    F0 = np.stack([o.get_f(m) for m in range(c2.n_ens)])
    o.assimilate(*(np.asarray(a, np.float32) for a in (obs[2], obs[0], obs[1])))
    Fa = np.stack([o.get_f(m) for m in range(c2.n_ens)])
    np.testing.assert_allclose(Fa, F0, rtol=1e-9)


def test_pointwise_geometry_p1():
    cfg = lbl.config_default("DA_LETKF", 32, 4)
    o = oracle.Oracle(cfg)
    w, valid = o.obs_weight(7, 9, 0, 0, 2)
    assert valid and math.isclose(w, 1 / cfg.obs_error_rho**2)
