"""The evaluation measures (bindiff, ensemble_stat, the energy spectrum of
fourier.ipynb) against independent numpy statements, on files written the way
lbl_output writes them.  Host only: no GPU."""
import os
import subprocess

import numpy as np

import lbl

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "lbm2d-letkf_b200")


def write(d, var, step, a):
    os.makedirs(d, exist_ok=True)
    np.asarray(a, np.float32).tofile(os.path.join(d, f"{var}_step{step:010d}.dat"))


def make_run(tmp, nx=24, M=3, steps=(0, 10, 20), seed=0):
    rng = np.random.default_rng(seed)
    nat, ens = {}, {}
    for t in steps:
        for var in ("u", "v", "rho"):
            base = (1.0 if var == "rho" else 0.0) + 0.05 * rng.standard_normal((nx, nx))
            nat[t, var] = base.astype(np.float32)
            write(f"{tmp}/nature/ens0000", var, t, nat[t, var])
            for m in range(M):
                a = (base + 0.01 * rng.standard_normal((nx, nx))).astype(np.float32)
                ens[t, var, m] = a
                write(f"{tmp}/calc/ens{m:04d}", var, t, a)
    return nat, ens


def test_ensemble_stat_matches_numpy(tmp_path):
    M = 3
    nat, ens = make_run(str(tmp_path), M=M)
    got = lbl.ensemble_stat(f"{tmp_path}/nature", f"{tmp_path}/calc", M, 10)
    L = np.longdouble
    mean, sd = {}, {}
    for var in ("u", "v", "rho"):
        x = np.stack([ens[10, var, m] for m in range(M)]).astype(L)
        mu = x.sum(0) / M
        var_ = (x * x).sum(0) / M - mu * mu
        mean[var] = mu.astype(np.float32).astype(L)
        sd[var] = np.sqrt(np.maximum(var_, 0)).astype(np.float32).astype(L)
    e_uv = np.concatenate([(mean[v] - nat[10, v].astype(L)).ravel() for v in ("u", "v")])
    s_uv = np.concatenate([sd[v].ravel() for v in ("u", "v")])
    np.testing.assert_allclose(got["rmse"], float(np.sqrt((e_uv ** 2).mean())), rtol=1e-12)
    np.testing.assert_allclose(got["spread"], float(np.sqrt((s_uv ** 2).mean())), rtol=1e-12)
    np.testing.assert_allclose(got["rho_rmse"], float(np.sqrt(((mean["rho"] - nat[10, "rho"]) ** 2).mean())),
                               rtol=1e-12)
    np.testing.assert_allclose(got["rho_spread"], float(np.sqrt((sd["rho"] ** 2).mean())), rtol=1e-12)
    np.testing.assert_allclose(got["max"], float(max(0, mean["u"].max(), mean["v"].max())), rtol=1e-12)


def test_bindiff_matches_numpy(tmp_path):
    make_run(str(tmp_path), M=2)
    a, b = f"{tmp_path}/nature/ens0000", f"{tmp_path}/calc/ens0001"
    rmse, n = lbl.bindiff(a, b, 20)
    d = [np.fromfile(f"{a}/{v}_step{20:010d}.dat", np.float32) - np.fromfile(f"{b}/{v}_step{20:010d}.dat", np.float32)
         for v in ("u", "v")]
    d = np.concatenate(d)
    assert n == d.size
    # the difference and its square are float (bindiff/main.cpp:57-59), the sum long double
    np.testing.assert_allclose(rmse, float(np.sqrt((d * d).astype(np.longdouble).mean())), rtol=1e-12)


def notebook_spectrum(u, v):
    """fourier.ipynb cell 2, with numpy's FFT in place of scipy.fftpack.fftn."""
    nx = u.shape[1]
    kmax = nx // 2
    fu = np.fft.fftn(u.astype(np.float64)) / nx / u.shape[0]
    fv = np.fft.fftn(v.astype(np.float64)) / nx / u.shape[0]
    f = (fu ** 2 + fv ** 2) / 2
    ek = np.zeros(kmax + 1)
    for i in range(kmax + 1):
        for j in range(kmax + 1):
            k = int(np.sqrt(i ** 2 + j ** 2) + 0.5)
            if k <= kmax:
                ek[k] += np.abs(f[i, j])
    return ek


def test_energy_spectrum_matches_notebook():
    rng = np.random.default_rng(4)
    for nx in (16, 32):
        y, x = np.mgrid[0:nx, 0:nx] * (2 * np.pi / nx)
        u = (np.sin(3 * x + 1) * np.cos(2 * y) + 0.1 * rng.standard_normal((nx, nx))).astype(np.float32)
        v = (np.cos(5 * y) + 0.1 * rng.standard_normal((nx, nx))).astype(np.float32)
        np.testing.assert_allclose(lbl.energy_spectrum(u, v), notebook_spectrum(u, v), rtol=1e-9, atol=1e-14)


def test_longrun_fixture_measure_is_the_notebook_spectrum():
    """The statistics in tests/golden/ref_longrun_id0.npz use this spectrum."""
    import os
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    import make_longrun as ml
    rng = np.random.default_rng(7)
    u, v = rng.standard_normal((2, 32, 32)).astype(np.float32)
    np.testing.assert_allclose(ml.spectrum(u, v), notebook_spectrum(u, v), rtol=1e-12, atol=1e-15)
    from conftest import golden
    g = golden("ref_longrun_id0.npz")
    assert g["spectra"].shape == (len(g["steps"]), 129) and np.all(g["energy"] > 0) and np.all(g["enstrophy"] > 0)


def test_cli_tools_keep_the_reference_formats(tmp_path):
    make_run(str(tmp_path), M=3, steps=(0, 10))
    out = subprocess.run([os.path.join(PKG, "lbl_ensemble_stat"), f"{tmp_path}/nature", f"{tmp_path}/calc", "10"],
                         capture_output=True, text=True, check=True)
    lines = out.stdout.strip().split("\n")
    assert lines[0].startswith("dirinfo: nature=")
    assert lines[1].startswith("t_step, spread, rmse, rho_spread, rho_rmse, max(debug) = 0, ")
    assert len(lines) == 3  # steps 0 and 10 (t % 10 == 0)
    out = subprocess.run([os.path.join(PKG, "lbl_bindiff"), f"{tmp_path}/nature/ens0000",
                          f"{tmp_path}/calc/ens0000", "10"], capture_output=True, text=True, check=True)
    rows = [r.split(",") for r in out.stdout.strip().split("\n")]
    assert [r[0] for r in rows] == ["0", "10"] and float(rows[1][1]) > 0
    write(f"{tmp_path}/spec", "u", 0, np.ones((16, 16)))
    write(f"{tmp_path}/spec", "v", 0, np.zeros((16, 16)))
    out = subprocess.run([os.path.join(PKG, "lbl_spectrum"), f"{tmp_path}/spec", "--t0=0", "--t1=0"],
                         capture_output=True, text=True, check=True)
    ek = [float(r.split(",")[1]) for r in out.stdout.strip().split("\n")]
    assert len(ek) == 9 and abs(ek[0] - 0.5) < 1e-12 and sum(ek[1:]) < 1e-12  # uniform u = 1: E(0) = 1/2


def test_h5_writer_round_trip(tmp_path):
    """The matrix-dump HDF5 writer against a reader written from the format specification."""
    import ctypes
    from h5_parse import read_datasets
    lib = lbl.load_library()
    rng = np.random.default_rng(1)
    for dtype, is_double in ((np.float32, 0), (np.float64, 1)):
        a = rng.standard_normal((3, 5, 7)).astype(dtype)
        path = str(tmp_path / f"_Q.float_3_5_7.{is_double}.h5")
        rc = lib.lbl_h5_write_dataset(path.encode(), 3, 5, 7, a.ctypes.data_as(ctypes.c_void_p), is_double)
        assert rc == 0
        ds = read_datasets(path)
        assert list(ds) == ["data"]
        assert ds["data"].dtype == dtype and ds["data"].shape == (3, 5, 7)
        np.testing.assert_array_equal(ds["data"], a)
