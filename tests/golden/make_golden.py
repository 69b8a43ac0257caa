"""Generate the golden fixtures that pin the oracle and the engine to the reference.

Runs oracle/_ref/ref_lbm -- the reference's own src/lbm.cu + src/data.cu, compiled
unmodified by oracle/Makefile and driven by oracle/ref_lbm_harness.cu -- on a GPU,
and condenses its dumps into small .npz files:

  ref_lbm_id<N>.npz   ensemble id N (seed N in NATURE mode; id 334 is DA member 0)
    kx, ky, amp           forcing mode table (data.cu:161-237)
    normals_head          first 4*n*(2+nsteps) cuRAND MTGP32 normals (data.cu:240-247)
    s<k>_rows_<var>       rows ROWS of f (9 planes), r, u, v, fx, fy after k steps
    s<k>_sums_<var>       FP64 checksums of the whole field: sum, sum of squares,
                          sum weighted by weights(shape) (see below)
    s<k>_cursor           the reference's i_rand_outdated after k steps

Needs a CUDA GPU.  Usage:
  python tests/golden/make_golden.py --out tests/golden [--ref oracle/_ref/ref_lbm]
"""
import argparse
import os
import subprocess
import sys
import tempfile

import numpy as np

NX = NY = 256
ROWS = (0, 1, NY // 2, NY - 1)
STEPS = (0, 1, 10, 100)


def weights(shape):
    """Fixed pseudo-random FP64 weights for the third checksum."""
    return np.random.default_rng(12345).random(int(np.prod(shape))).reshape(shape)


def checksums(a):
    a = np.asarray(a, np.float64)
    return np.array([a.sum(), (a * a).sum(), (a * weights(a.shape)).sum()])


def run(ref, ens_id, nsteps, dumps, outdir):
    os.makedirs(outdir, exist_ok=True)
    subprocess.run([ref, outdir, str(ens_id), str(nsteps), ",".join(map(str, dumps))], check=True)


def load(path, dtype=np.float32):
    return np.fromfile(path, dtype=dtype)


def condense(tmp, dumps, nsteps):
    out = {}
    kx = load(f"{tmp}/modes_kx.f32")
    out["kx"], out["ky"], out["amp"] = kx, load(f"{tmp}/modes_ky.f32"), load(f"{tmp}/modes_amp.f32")
    n = kx.size
    out["normals_head"] = load(f"{tmp}/normals.f32")[: 4 * n * (2 + nsteps)]
    for s in dumps:
        pre = f"{tmp}/s{s}_"
        f = load(pre + "f.f32").reshape(9, NY, NX)
        out[f"s{s}_rows_f"] = f[:, list(ROWS), :]
        out[f"s{s}_sums_f"] = checksums(f)
        for var in ("r", "u", "v", "fx", "fy"):
            a = load(pre + var + ".f32").reshape(NY, NX)
            out[f"s{s}_rows_{var}"] = a[list(ROWS), :]
            out[f"s{s}_sums_{var}"] = checksums(a)
        out[f"s{s}_cursor"] = load(pre + "cursor.i32", np.int32)
    return out


def main():
    ap = argparse.ArgumentParser()
    root = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    ap.add_argument("--ref", default=os.path.join(root, "oracle", "_ref", "ref_lbm"))
    ap.add_argument("--out", default=os.path.dirname(os.path.abspath(__file__)))
    a = ap.parse_args()
    if not os.path.exists(a.ref):
        sys.exit(f"missing {a.ref}: build it with `make -C oracle ref` where the reference is mounted")
    os.makedirs(a.out, exist_ok=True)
    for ens_id, nsteps, dumps in ((0, 100, STEPS), (334, 1, (0, 1))):
        with tempfile.TemporaryDirectory() as tmp:
            run(a.ref, ens_id, nsteps, dumps, tmp)
            data = condense(tmp, dumps, nsteps)
        path = os.path.join(a.out, f"ref_lbm_id{ens_id}.npz")
        np.savez_compressed(path, rows=np.array(ROWS), steps=np.array(dumps), **data)
        print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
