"""The pair ordering of the wide analysis's Jacobi (analysis_wide_kernel, step 5 in
csrc/letkf_kernels.cu), restated on the CPU.

64 columns, 32 thread quads; at level L = 0..5 the columns form blocks of 2H
(H = 32 >> L) with a fixed and a shifting half.  Quad s = (block b, index i) holds
fixed column 2Hb + i and, in round j, shifting column 2Hb + H + ((i + j) mod H); between
rounds the shifting column a quad takes is the one the quad above it held.  The kernel
relies on three properties, checked here: every pair of columns meets exactly once per
sweep, every column has exactly one owner in every round, and a quad's next shifting
column was some quad's shifting column in the round before (so it is in its home slot,
written by its previous owner before the barrier).  The GPU parity of the kernel itself
is in test_gpu_letkf.py."""
import numpy as np
import pytest

N = 64
QUADS = N // 2


def pairs_of_round(level, j):
    H = QUADS >> level
    out = []
    for s in range(QUADS):
        b, i = s >> (5 - level), s & (H - 1)
        out.append((2 * H * b + i, 2 * H * b + H + ((i + j) & (H - 1))))
    return out


def test_every_pair_once_per_sweep():
    seen = set()
    rounds = 0
    for level in range(6):
        for j in range(QUADS >> level):
            rounds += 1
            for ca, cb in pairs_of_round(level, j):
                pair = (min(ca, cb), max(ca, cb))
                assert pair not in seen, pair
                seen.add(pair)
    assert rounds == N - 1
    assert len(seen) == N * (N - 1) // 2


@pytest.mark.parametrize("level", range(6))
def test_one_owner_per_column_and_handoffs(level):
    prev = None
    for j in range(QUADS >> level):
        cur = pairs_of_round(level, j)
        owned = sorted(c for pair in cur for c in pair)
        assert owned == list(range(N))
        if prev is not None:
            shifting_before = {cb for _, cb in prev}
            for (ca, cb), (ca0, _) in zip(cur, prev):
                assert ca == ca0                  # the fixed column stays with its quad
                assert cb in shifting_before      # the new shifting column was handed on
        prev = cur


def quad_jacobi(A, tol=1e-6, max_sweeps=20):
    """The wide kernel's Jacobi in numpy (float64): one-sided rotations of the columns of
    A in the recursive block ordering, lazily scaled columns (column c = sc[c] * X[:, c]),
    squared thresholds (rotate when g^2 > tol^2 a_lo a_hi; a sweep in which no rotated pair
    reached g^2 >= tol a_lo a_hi ends the iteration), t = sign(de)|e| / (|d| + sqrt(d^2 + e^2))."""
    X = A.copy()
    n = X.shape[1]
    sc = np.ones(n)
    sweeps = 0
    for _ in range(max_sweeps):
        sweeps += 1
        X *= sc
        sc[:] = 1.0
        a = np.einsum("ij,ij->j", X, X)
        big = False
        for level in range(6):
            for j in range(QUADS >> level):
                for ca, cb in pairs_of_round(level, j):
                    g = (X[:, ca] @ X[:, cb]) * sc[ca] * sc[cb]
                    lo, hi = (ca, cb) if ca < cb else (cb, ca)
                    p2 = a[lo] * a[hi]
                    if not g * g > tol * tol * p2:
                        continue
                    big |= g * g >= tol * p2
                    d, e = a[hi] - a[lo], 2 * g
                    t = np.copysign(abs(e), d * e) / (abs(d) + np.sqrt(d * d + e * e))
                    cs = 1 / np.sqrt(1 + t * t)
                    xl, xh = X[:, lo].copy(), X[:, hi].copy()
                    X[:, lo] = xl - t * (sc[hi] / sc[lo]) * xh
                    X[:, hi] = xh + t * (sc[lo] / sc[hi]) * xl
                    sc[lo] *= cs
                    sc[hi] *= cs
                    a[lo] -= t * g
                    a[hi] += t * g
        if not big:
            break
    return X * sc, sweeps


def test_quad_jacobi_diagonalises_an_spd_matrix():
    """A = Q with orthogonal columns at the end is V Lambda: lambda_k = |a_k|, v_k = a_k / |a_k|.
    The last sweep leaves relative off-diagonals of about tol (1e-6, the reference's syevj
    tolerance), so V is orthogonal to a few tol; the eigenvalues are second order in it."""
    rng = np.random.default_rng(7)
    C = rng.standard_normal((75, N)) * 0.3
    Q = (N - 1) / 1.1 * np.eye(N) + C.T @ C
    A, sweeps = quad_jacobi(Q)
    lam = np.linalg.norm(A, axis=0)
    V = A / lam
    assert sweeps <= 8
    np.testing.assert_allclose(V.T @ V, np.eye(N), atol=1e-5)
    np.testing.assert_allclose(Q @ V, V * lam, atol=1e-5 * lam.max())
    np.testing.assert_allclose(np.sort(lam), np.linalg.eigvalsh(Q), rtol=1e-9)


def test_quad_jacobi_warm_start_needs_fewer_sweeps():
    """The kernel starts each point from the previous point's eigenvectors (A = Q V_prev):
    for a nearby matrix that leaves little to rotate."""
    rng = np.random.default_rng(8)
    C = rng.standard_normal((75, N)) * 0.3
    Q1 = (N - 1) / 1.1 * np.eye(N) + C.T @ C
    C2 = C + 0.02 * rng.standard_normal(C.shape)
    Q2 = (N - 1) / 1.1 * np.eye(N) + C2.T @ C2
    A1, cold = quad_jacobi(Q1)
    V1 = A1 / np.linalg.norm(A1, axis=0)
    A2, warm = quad_jacobi(Q2 @ V1)
    assert warm < cold
    # V_prev is orthogonal to about tol, so the eigenvalues of Q V_prev's columns are too
    lam2 = np.linalg.norm(A2, axis=0)
    np.testing.assert_allclose(np.sort(lam2), np.linalg.eigvalsh(Q2), rtol=1e-5)
