"""Inputs of the reference-LETKF fixtures (tests/golden/ref_letkf_<case>.npz).

Each case is a forecast ensemble and a set of observations that the FP64 oracle
regenerates bit for bit wherever liboracle.so runs: members are the reference's
DA ensemble (independent random-phase initial conditions, ensemble id 334 + k,
src/data.cu:31-35) advanced a few steps by the oracle with seeded forcing normals,
and the observations are a NATURE run (id 0) advanced the same way plus seeded
Gaussian noise, NaN off the observation lattice like io/observed files.  The
fixture stores a hash of both, so a test knows it feeds the exact inputs the
reference analysed.

The reference side is oracle/_ref/ref_letkf_<harness> (oracle/ref_letkf_harness.cu):
the reference's letkf.cu glue and letkf_solver.h cuBLAS / cuSOLVER call sequence,
built with one set of the reference's compile-time knobs per harness.
"""
import hashlib

import numpy as np

import oracle

# name: harness binary (its compile-time knobs), members, grid, DA_XYPRUNE,
# LETKF_RLOC_LEN, OBS_ERROR_U, OBS_ERROR_RHO, initial-condition kind and amplitude,
# oracle steps, noise seed, stored rows
CASES = {
    # the 256^2 x 16 workload's localisation and observation errors (sigma_u 0.1, sigma_rho 0.01), the
    # bench's initial spectrum (rms 1.0 physical)
    "p4r1_m16": dict(harness="p4r1", M=16, nx=64, p=4, L=1, su=0.1, sr=0.01, ic="k4exp", amp=1.0, steps=10,
                     seed=11, rows=(0, 1, 2, 3, 33, 63)),
    "p4r1_m32": dict(harness="p4r1", M=32, nx=64, p=4, L=1, su=0.1, sr=0.01, ic="k4exp", amp=1.0, steps=10,
                     seed=12, rows=(0, 1, 2, 63)),
    # pointwise analysis (the reference's default DA_XYPRUNE = 1): 3 observations per point
    "p1_m16": dict(harness="p1", M=16, nx=64, p=1, L=0, su=0.1, sr=0.01, ic="k4exp", amp=1.0, steps=10,
                   seed=13, rows=(0, 1, 31, 63)),
    # p = 4 without LETKF_RLOC_LEN (48 observations), small errors against the
    # reference's own initial condition: a Q with a large condition number
    "p4_m8_small": dict(harness="p4small", M=8, nx=64, p=4, L=0, su=0.002, sr=1e-4, ic="reference", amp=0.01,
                        steps=10, seed=14, rows=(0, 1, 2, 3, 62, 63)),
}
BETA = 1.1


def config(lib, case, mode="DA_LETKF", n_ens=None):
    """lbl_config of a case from `lib` (the oracle module or the product package)."""
    c = CASES[case]
    return lib.config_default(mode, c["nx"], c["M"] if n_ens is None else n_ens, da_xyprune=c["p"],
                              letkf_rloc_len=c["L"], letkf_covinf=BETA, obs_error_u=c["su"], obs_error_rho=c["sr"],
                              daprune=1, ic_kind=1 if c["ic"] == "k4exp" else 0, ic_amp=c["amp"])


def _step(o, cfg, steps, seed):
    n_modes = oracle.force_modes(cfg)[0].size
    rng = np.random.default_rng(seed)
    o.step(steps, rng.standard_normal(4 * n_modes * steps).astype(np.float32))


def inputs(case):
    """(f [M][9][ny][nx] float32, (ro, uo, vo) float32 with NaN off the lattice)."""
    c = CASES[case]
    cfg = config(oracle, case)
    o = oracle.Oracle(cfg)
    o.init(0)
    _step(o, cfg, c["steps"], 1000 + c["seed"])
    f = np.stack([o.get_f(m).astype(np.float32) for m in range(c["M"])])
    o.close()
    nat_cfg = config(oracle, case, "NATURE", 1)
    n = oracle.Oracle(nat_cfg)
    n.init(0)
    _step(n, nat_cfg, c["steps"], 1000 + c["seed"])
    r, u, v = (a.astype(np.float32) for a in n.macros(0))
    n.close()
    rng = np.random.default_rng(c["seed"])
    ro = (r + c["sr"] * rng.standard_normal(r.shape)).astype(np.float32)
    uo = (u + c["su"] * rng.standard_normal(u.shape)).astype(np.float32)
    vo = (v + c["su"] * rng.standard_normal(v.shape)).astype(np.float32)
    off = np.ones(r.shape, bool)
    off[::c["p"], ::c["p"]] = False
    for a in (ro, uo, vo):
        a[off] = np.nan
    return f, (ro, uo, vo)


def digest(f, obs):
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(f).tobytes())
    for a in obs:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def weights(shape):
    """Fixed pseudo-random FP64 weights for the third checksum."""
    return np.random.default_rng(12345).random(int(np.prod(shape))).reshape(shape)


def checksums(a):
    """FP64 sum, sum of squares and weighted sum of a whole field."""
    a = np.asarray(a, np.float64)
    return np.array([a.sum(), (a * a).sum(), (a * weights(a.shape)).sum()])
