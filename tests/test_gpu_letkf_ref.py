"""The engine's LETKF analysis, through the C ABI, against the reference's own solver.

tests/golden/ref_letkf_<case>.npz hold the analysis that the reference's letkf.cu glue
and letkf_solver.h cuBLAS / cuSOLVER sequence (oracle/_ref/ref_letkf_*) computed for
inputs regenerated here bit for bit (tests/letkf_ref_cases.py): the 256^2 x 16 workload's localisation and
observation errors at M = 16 and 32, the pointwise p = 1 analysis, and p = 4 without
LETKF_RLOC_LEN at small observation errors.  Both sides work in FP32 (the engine: FP32
Gram and its own Jacobi; the reference: cuBLAS and syevjBatched at tolerance 1e-6).
"""
import json

import numpy as np
import pytest

from conftest import golden

import lbl
import letkf_ref_cases as lc

pytestmark = pytest.mark.gpu

REF_TOL = 1e-4       # increments, as a fraction of the largest increment (measured 7e-6..3e-5)
CHECKSUM_TOL = 1e-3  # whole-field increment checksums, relative


@pytest.mark.parametrize("case,gram", [(c, 0) for c in lc.CASES] +
                         [(c, 2) for c in lc.CASES if lc.CASES[c]["p"] == 4])
def test_engine_matches_reference_solver(case, gram):
    z = golden(f"ref_letkf_{case}.npz")
    meta = json.loads(str(z["meta"]))
    f, obs = lc.inputs(case)
    assert lc.digest(f, obs) == meta["digest"]
    cfg = lc.config(lbl, case)
    cfg.gram = gram  # 0: the SIMT FP32 Gram; 2: the tcgen05 tensor-core Gram (LBL_GRAM_TF32X3)
    e = lbl.Ensemble(cfg)
    e.init(0)
    for m in range(cfg.n_ens):
        e.set_f(m, f[m])
    e.assimilate(cfg.iiter, *obs)
    st = e.letkf_stats()
    inc = np.stack([e.get_f(m) for m in range(cfg.n_ens)]).astype(np.float64) - f.astype(np.float64)
    e.close()
    assert st["nan"] == 0 and st["n_noconv"] == 0, st
    rows = list(z["rows"])
    ref = z["inc_rows"].astype(np.float64)
    err = float(np.max(np.abs(inc[:, :, rows, :] - ref))) / float(np.max(np.abs(ref)))
    assert err < REF_TOL, f"{case}: increment error {err:.3e} of the largest increment"
    sums = lc.checksums(inc)
    ref_sums = z["inc_sums"]
    cerr = np.abs(sums - ref_sums) / np.maximum(np.abs(ref_sums), 1e-300)
    cerr[0] = abs(sums[0] - ref_sums[0]) / float(np.sum(np.abs(inc)))
    assert np.all(cerr < CHECKSUM_TOL), f"{case}: checksum errors {cerr}"
