"""The FP64 oracle's LETKF against the reference's own solver (CPU, no GPU).

tests/golden/ref_letkf_<case>.npz hold the analysis that the reference's letkf.cu glue
and letkf_solver.h cuBLAS / cuSOLVER sequence (oracle/_ref/ref_letkf_*, made by
tests/golden/make_letkf_golden.py on a GPU) computed for inputs the oracle regenerates
bit for bit (tests/letkf_ref_cases.py).  The reference works in FP32 with a Jacobi
tolerance of 1e-6; the oracle in FP64 to convergence.  Increments agree within
REF_TOL of the largest increment, eigenvalues within LAMBDA_TOL relative, and the
whole-field checksums of the increment within CHECKSUM_TOL relative.
"""
import json

import numpy as np
import pytest

from conftest import golden

import letkf_ref_cases as lc
import oracle

REF_TOL = 1e-4        # increments: FP32 cuBLAS/cuSOLVER (tol 1e-6) against FP64 (measured 3e-6..2.5e-5)
LAMBDA_TOL = 1e-4     # eigenvalues of Q, relative
CHECKSUM_TOL = 1e-3   # sum, sum of squares and weighted sum of the whole increment field, relative


def oracle_analysis(case):
    f, obs = lc.inputs(case)
    z = golden(f"ref_letkf_{case}.npz")
    meta = json.loads(str(z["meta"]))
    assert lc.digest(f, obs) == meta["digest"], "regenerated inputs differ from the ones the reference analysed"
    cfg = lc.config(oracle, case)
    o = oracle.Oracle(cfg)
    for m in range(cfg.n_ens):
        o.set_f(m, f[m])
    _, lam = o.assimilate(*obs, want_lambda=True)
    inc = np.stack([o.get_f(m) for m in range(cfg.n_ens)]) - f.astype(np.float64)
    o.close()
    return z, inc, lam


@pytest.mark.parametrize("case", list(lc.CASES))
def test_oracle_matches_reference_solver(case):
    z, inc, lam = oracle_analysis(case)
    rows = list(z["rows"])
    ref = z["inc_rows"].astype(np.float64)
    scale = float(np.max(np.abs(ref)))
    assert scale > 0
    err = float(np.max(np.abs(inc[:, :, rows, :] - ref))) / scale
    assert err < REF_TOL, f"{case}: increment error {err:.3e} of the largest increment"
    lam_ref = z["lambda_rows"].astype(np.float64)
    lerr = float(np.max(np.abs(lam[rows] - lam_ref) / np.abs(lam_ref)))
    assert lerr < LAMBDA_TOL, f"{case}: eigenvalue error {lerr:.3e}"
    sums = lc.checksums(inc)
    ref_sums = z["inc_sums"]
    cerr = np.abs(sums - ref_sums) / np.maximum(np.abs(ref_sums), 1e-300)
    # the plain sum can cancel to near zero; compare it with the sum of |increments| instead
    cerr[0] = abs(sums[0] - ref_sums[0]) / float(np.sum(np.abs(inc)))
    assert np.all(cerr < CHECKSUM_TOL), f"{case}: checksum errors {cerr}"
