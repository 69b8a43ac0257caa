"""Generate the long-run fixture: the reference's own LBM (oracle/_ref/ref_lbm, its
src/lbm.cu + src/data.cu compiled unmodified) run for 10,000 steps of the NATURE case
at its defaults (256x256, ensemble id 0), condensed into the statistics that a
chaotic run can be compared on:

  ref_longrun_id0.npz      the reference's defaults (Cs 0.2, nu 1e-4)
  ref_longrun_c0_id0.npz   --ref oracle/_ref/ref_lbm_c0 --name ref_longrun_c0_id0.npz: the same
                           build with Cs 0.1 and tau 0.51 (oracle/make_ref_c0.sh)
    steps        the sampled steps (every 500 from 2000 to 10000)
    spectra      [len(steps)][129] energy spectrum E(k) of (u, v) at each sample, the
                 shell sum of postprocess/fourier.ipynb cell 2 (numpy FFT here)
    energy       [len(steps)] domain mean of (u^2 + v^2) / 2
    enstrophy    [len(steps)] domain mean of omega^2 / 2, omega by central differences

Needs a CUDA GPU and the built reference binary.  Usage:
  python tests/golden/make_longrun.py --out tests/golden [--ref oracle/_ref/ref_lbm]
"""
import argparse
import os
import subprocess
import sys
import tempfile

import numpy as np

NX = NY = 256
NSTEPS = 10000
STEPS = tuple(range(2000, NSTEPS + 1, 500))


def spectrum(u, v):
    """E(k), k = 0..nx/2: |(F(u)^2 + F(v)^2) / 2| summed over shells of the
    non-negative wavenumbers, F = fft2 / (nx ny) (fourier.ipynb cell 2)."""
    ny, nx = u.shape
    fu = np.fft.fft2(np.asarray(u, np.float64)) / (nx * ny)
    fv = np.fft.fft2(np.asarray(v, np.float64)) / (nx * ny)
    kmax = nx // 2
    i = np.arange(min(kmax, ny - 1) + 1)[:, None]
    j = np.arange(kmax + 1)[None, :]
    k = np.floor(np.sqrt(i * i + j * j) + 0.5).astype(int)
    e = np.abs(0.5 * (fu[: i.shape[0], : kmax + 1] ** 2 + fv[: i.shape[0], : kmax + 1] ** 2))
    out = np.zeros(kmax + 1)
    sel = k <= kmax
    np.add.at(out, k[sel], e[sel])
    return out


def stats(u, v, dx):
    u = np.asarray(u, np.float64)
    v = np.asarray(v, np.float64)
    w = (np.roll(v, -1, 1) - np.roll(v, 1, 1)) / (2 * dx) - (np.roll(u, -1, 0) - np.roll(u, 1, 0)) / (2 * dx)
    return spectrum(u, v), float(np.mean(0.5 * (u * u + v * v))), float(np.mean(0.5 * w * w))


def main():
    ap = argparse.ArgumentParser()
    root = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    ap.add_argument("--ref", default=os.path.join(root, "oracle", "_ref", "ref_lbm"))
    ap.add_argument("--out", default=os.path.dirname(os.path.abspath(__file__)))
    ap.add_argument("--name", default="ref_longrun_id0.npz")
    a = ap.parse_args()
    if not os.path.exists(a.ref):
        sys.exit(f"missing {a.ref}: build it with `make -C oracle ref` where the reference is mounted")
    dx = float(np.float32(2 * np.pi) / np.float32(NY - 1))
    spectra, energy, enstrophy = [], [], []
    with tempfile.TemporaryDirectory() as tmp:
        subprocess.run([a.ref, tmp, "0", str(NSTEPS), ",".join(map(str, STEPS))], check=True)
        for s in STEPS:
            u = np.fromfile(f"{tmp}/s{s}_u.f32", np.float32).reshape(NY, NX)
            v = np.fromfile(f"{tmp}/s{s}_v.f32", np.float32).reshape(NY, NX)
            e, en, z = stats(u, v, dx)
            spectra.append(e)
            energy.append(en)
            enstrophy.append(z)
    path = os.path.join(a.out, a.name)
    np.savez_compressed(path, steps=np.array(STEPS), spectra=np.array(spectra), energy=np.array(energy),
                        enstrophy=np.array(enstrophy))
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
