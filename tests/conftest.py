"""Shared test setup: import paths, the `gpu` marker, builds, fixture loaders."""
import ctypes
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "lbm2d-letkf_b200")
ORACLE = os.path.join(ROOT, "oracle")
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (PKG, ORACLE, ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs the engine through its C ABI)")


def _ensure_built():
    if not os.path.exists(os.path.join(PKG, "liblbl.so")):
        subprocess.run(["make", "-C", PKG, "-j8"], check=True, stdout=subprocess.DEVNULL)
    if not os.path.exists(os.path.join(ORACLE, "liboracle.so")):
        subprocess.run(["make", "-C", ORACLE, "liboracle.so"], check=True, stdout=subprocess.DEVNULL)


_ensure_built()


def gpu_count() -> int:
    try:
        cuda = ctypes.CDLL("libcuda.so.1")
    except OSError:
        return 0
    if cuda.cuInit(0) != 0:
        return 0
    n = ctypes.c_int()
    return n.value if cuda.cuDeviceGetCount(ctypes.byref(n)) == 0 else 0


def golden(name):
    path = os.path.join(GOLDEN, name)
    if not os.path.exists(path):
        pytest.skip(f"golden fixture {name} not generated (tests/golden/make_golden.py)")
    return np.load(path)


def weights(shape):
    """Same FP64 weights as tests/golden/make_golden.py uses for its checksums."""
    return np.random.default_rng(12345).random(int(np.prod(shape))).reshape(shape)


def checksums(a):
    a = np.asarray(a, np.float64)
    return np.array([a.sum(), (a * a).sum(), (a * weights(a.shape)).sum()])


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))
