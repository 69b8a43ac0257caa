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
