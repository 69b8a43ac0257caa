"""Generate the fixtures that pin the LETKF analysis to the reference's own solver.

For every case of tests/letkf_ref_cases.py, builds the inputs (a forecast ensemble
and observations the FP64 oracle regenerates bit for bit), runs
oracle/_ref/ref_letkf_<harness> on them -- the reference's letkf.cu glue and its
letkf_solver.h cuBLAS / cuSOLVER call sequence (oracle/ref_letkf_harness.cu) --
and condenses the analysis into tests/golden/ref_letkf_<case>.npz:

  meta           JSON: the case, the harness, the eigensolver used, input digest
  rows           the stored grid rows
  inc_rows       analysis minus forecast populations at those rows, [M][9][rows][nx] float32
  lambda_rows    eigenvalues of Q at those rows, ascending, [rows][nx][M] float32
  inc_sums       FP64 checksums (sum, sum of squares, weighted sum) of the whole increment field
  inc_max        max |increment| over the whole field

Needs a CUDA GPU and the harnesses (`make -C oracle ref REF_SRC=<reference src/>`).
Usage:  python tests/golden/make_letkf_golden.py [--out tests/golden] [case ...]
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import letkf_ref_cases as lc  # noqa: E402


def run_case(name, out_dir):
    c = lc.CASES[name]
    f, obs = lc.inputs(name)
    M, nx = c["M"], c["nx"]
    ny = nx
    exe = os.path.join(ROOT, "oracle", "_ref", f"ref_letkf_{c['harness']}")
    with tempfile.TemporaryDirectory() as tmp:
        src, dst = os.path.join(tmp, "in.bin"), os.path.join(tmp, "out.bin")
        with open(src, "wb") as fp:
            np.array([nx, ny, M, 0, ny], np.int32).tofile(fp)
            f.tofile(fp)
            for a in obs:
                a.tofile(fp)
        subprocess.run([exe, src, dst], check=True)
        raw = np.fromfile(dst, np.uint8)
    hdr = raw[:24].view(np.int32)
    assert list(hdr[:5]) == [nx, ny, M, 0, ny], hdr
    evd = int(hdr[5])
    body = raw[24:].view(np.float32)
    fa = body[: M * 9 * nx * ny].reshape(M, 9, ny, nx)
    lam = body[M * 9 * nx * ny:].reshape(ny, nx, M)
    inc = fa.astype(np.float64) - f.astype(np.float64)
    rows = list(c["rows"])
    out = {
        "meta": json.dumps({"case": name, **{k: v for k, v in c.items() if k != "rows"}, "beta": lc.BETA,
                            "evd": "cusolverDnSsyevj per matrix (EigenG-Batched stand-in)" if evd else
                                   "cusolverDnSsyevjBatched, tol 1e-6, max 100 sweeps, unsorted",
                            "digest": lc.digest(f, obs)}),
        "rows": np.array(rows, np.int32),
        "inc_rows": inc[:, :, rows, :].astype(np.float32),
        "lambda_rows": np.sort(lam[rows], axis=-1).astype(np.float32),
        "inc_sums": lc.checksums(inc),
        "inc_max": np.array(np.max(np.abs(inc))),
    }
    path = os.path.join(out_dir, f"ref_letkf_{name}.npz")
    np.savez_compressed(path, **out)
    print(f"{path}: max|inc| {out['inc_max']:.4e}, evd {evd}, {os.path.getsize(path)} bytes")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=HERE)
    ap.add_argument("cases", nargs="*")
    args = ap.parse_args()
    for name in args.cases or list(lc.CASES):
        run_case(name, args.out)


if __name__ == "__main__":
    main()
