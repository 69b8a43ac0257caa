"""ORACLE (test infrastructure only): ctypes wrapper of liboracle.so, the FP64 CPU
restatement of the reference's forecast-and-assimilate path (oracle.cpp).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module, and only as the checker or the timed CPU baseline; the product path
(liblbl.so) never calls it.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_LBM = os.path.join(HERE, "_ref", "ref_lbm")
Q = 9

_lib = None

MODES = {"NATURE": 0, "OBSERVE": 1, "DA_LETKF": 2, "DA_NUDGING": 3}
IC_K4EXP = 1
ENS_PERTURBED = 1


class Config(ctypes.Structure):
    """lbl_config of include/lbl.h (the C struct the oracle reads), so that callers of the
    oracle need nothing from the product package."""

    _fields_ = [
        ("abi_version", ctypes.c_int32), ("mode", ctypes.c_int32), ("nx", ctypes.c_int32),
        ("ny", ctypes.c_int32), ("n_ens", ctypes.c_int32), ("iiter", ctypes.c_int32),
        ("ioprune", ctypes.c_int32), ("daprune", ctypes.c_int32), ("da_xyprune", ctypes.c_int32),
        ("letkf_rloc_len", ctypes.c_int32), ("iter_main", ctypes.c_int32), ("spinup", ctypes.c_int32),
        ("ic_kind", ctypes.c_int32), ("ens_init", ctypes.c_int32), ("compat_stale_v", ctypes.c_int32),
        ("jacobi_max_sweeps", ctypes.c_int32), ("write_mat", ctypes.c_int32), ("lbm_variant", ctypes.c_int32),
        ("letkf_covinf", ctypes.c_double), ("obs_error_rho", ctypes.c_double), ("obs_error_u", ctypes.c_double),
        ("cs", ctypes.c_double), ("nu", ctypes.c_double), ("tau", ctypes.c_double), ("cfl", ctypes.c_double),
        ("rho_ref", ctypes.c_double), ("u_ref", ctypes.c_double), ("h_ref", ctypes.c_double),
        ("kf", ctypes.c_double), ("fkf", ctypes.c_double), ("friction_rate", ctypes.c_double),
        ("ic_amp", ctypes.c_double), ("ens_perturb", ctypes.c_double), ("jacobi_tol", ctypes.c_double),
        ("force_seed", ctypes.c_uint64), ("obs_seed", ctypes.c_uint64),
        ("da_dummy", ctypes.c_int32), ("da_quadra", ctypes.c_int32), ("da_obs_ruv", ctypes.c_int32),
        ("gram", ctypes.c_int32), ("da_nud_rate", ctypes.c_double),
        ("storage", ctypes.c_int32), ("reserved1", ctypes.c_int32),
    ]

    def copy(self) -> "Config":
        c = Config()
        ctypes.pointer(c)[0] = self
        return c

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


def config_default(mode="NATURE", nx: int = 256, n_ens: int = 1, **overrides) -> Config:
    """The reference's config.h defaults (orc_config_default) with lbl_config overrides."""
    c = Config()
    m = MODES[mode] if isinstance(mode, str) else int(mode)
    if load().orc_config_default(ctypes.byref(c), m, nx, n_ens) != 0:
        raise ValueError("orc_config_default")
    for k, v in overrides.items():
        if not hasattr(c, k):
            raise KeyError(f"unknown config field {k}")
        setattr(c, k, v)
    return c


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"oracle not built: {LIB_PATH} (run `make -C oracle liboracle.so`)")
    lib = ctypes.CDLL(LIB_PATH)
    P, I = ctypes.c_void_p, ctypes.c_int
    F = ctypes.POINTER(ctypes.c_float)
    D = ctypes.POINTER(ctypes.c_double)
    IP = ctypes.POINTER(ctypes.c_int)
    sig = {
        "orc_set_threads": (I, [I]),
        "orc_config_default": (I, [P, I, I, I]),
        "orc_create": (P, [P]),
        "orc_destroy": (None, [P]),
        "orc_ic_fields": (I, [P, I, F, F, F, F]),
        "orc_init": (I, [P, I]),
        "orc_force_modes": (I, [P, F, F, F, I]),
        "orc_force": (I, [P, F, D, D]),
        "orc_set_force": (I, [P, F, F]),
        "orc_set_f": (I, [P, I, F]),
        "orc_get_f": (I, [P, I, D]),
        "orc_get_macros": (I, [P, I, D, D, D]),
        "orc_set_macros": (I, [P, I, F, F, F]),
        "orc_step_noforce": (I, [P]),
        "orc_step": (I, [P, I, F]),
        "orc_vorticity_f32": (I, [P, F, F, F]),
        "orc_observe": (I, [P, F, F, F, F, F, F, F]),
        "orc_obs_weight": (I, [P, I, I, I, I, I, D, IP]),
        "orc_assimilate": (I, [P, F, F, F, D]),
        "orc_assimilate_rows": (I, [P, F, F, F, D, I, I]),
        "orc_max_sweeps": (I, [P]),
        "orc_nudge": (I, [P, F, F, F]),
        "orc_set_closure": (I, [P, F, ctypes.c_double, ctypes.c_double]),
        "orc_closure_forward": (I, [F, D, I, D]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _f(a):
    return None if a is None else a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def _d(a):
    return None if a is None else a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32).reshape(-1)


def set_threads(n: int) -> int:
    return load().orc_set_threads(n)


def ic_fields(cfg, seed: int):
    """(r, u, v, f) of ensemble id `seed` exactly as stdata::init_lbm makes them (FP32)."""
    lib = load()
    nxy = cfg.nx * cfg.ny
    r, u, v = (np.empty(nxy, np.float32) for _ in range(3))
    f = np.empty(Q * nxy, np.float32)
    lib.orc_ic_fields(ctypes.byref(cfg), seed, _f(r), _f(u), _f(v), _f(f))
    sh = (cfg.ny, cfg.nx)
    return r.reshape(sh), u.reshape(sh), v.reshape(sh), f.reshape((Q,) + sh)


def force_modes(cfg):
    lib = load()
    kx, ky, amp = (np.empty(128, np.float32) for _ in range(3))
    n = lib.orc_force_modes(ctypes.byref(cfg), _f(kx), _f(ky), _f(amp), 128)
    return kx[:n].copy(), ky[:n].copy(), amp[:n].copy()


def closure_forward(params, x):
    """The C++ oracle's closure multiplier for feature rows x [n][6]."""
    lib = load()
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.empty(x.shape[0], np.float64)
    lib.orc_closure_forward(_f(_f32(params)), _d(x), x.shape[0], _d(out))
    return out


def vorticity(cfg, u, v):
    out = np.empty(cfg.nx * cfg.ny, np.float32)
    load().orc_vorticity_f32(ctypes.byref(cfg), _f(_f32(u)), _f(_f32(v)), _f(out))
    return out.reshape(cfg.ny, cfg.nx)


class Oracle:
    """FP64 CPU state of a whole ensemble (the oracle's counterpart of lbl.Ensemble)."""

    def __init__(self, cfg):
        self.lib = load()
        self.cfg = cfg.copy()
        self.nx, self.ny, self.M = cfg.nx, cfg.ny, cfg.n_ens
        self.nxy = cfg.nx * cfg.ny
        self.h = self.lib.orc_create(ctypes.byref(self.cfg))
        if not self.h:
            raise ValueError("orc_create rejected the configuration")

    def close(self):
        if self.h:
            self.lib.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def init(self, ens_offset: int = 0):
        self.lib.orc_init(self.h, ens_offset)

    def set_f(self, m: int, f):
        self.lib.orc_set_f(self.h, m, _f(_f32(f)))

    def get_f(self, m: int) -> np.ndarray:
        out = np.empty(Q * self.nxy, np.float64)
        self.lib.orc_get_f(self.h, m, _d(out))
        return out.reshape(Q, self.ny, self.nx)

    def macros(self, m: int):
        r, u, v = (np.empty(self.nxy, np.float64) for _ in range(3))
        self.lib.orc_get_macros(self.h, m, _d(r), _d(u), _d(v))
        return tuple(a.reshape(self.ny, self.nx) for a in (r, u, v))

    def set_macros(self, m: int, r=None, u=None, v=None):
        """Overwrite member m's current macros (any of r, u, v; None keeps it)."""
        a = [None if x is None else _f32(x) for x in (r, u, v)]
        self.lib.orc_set_macros(self.h, m, *(_f(x) for x in a))

    def force(self, randoms):
        fx, fy = np.empty(self.nxy, np.float64), np.empty(self.nxy, np.float64)
        self.lib.orc_force(self.h, _f(_f32(randoms)), _d(fx), _d(fy))
        return fx.reshape(self.ny, self.nx), fy.reshape(self.ny, self.nx)

    def set_force(self, fx, fy):
        self.lib.orc_set_force(self.h, _f(_f32(fx)), _f(_f32(fy)))

    def step_noforce(self):
        self.lib.orc_step_noforce(self.h)

    def step(self, nsteps: int, randoms=None):
        r = None if randoms is None else _f32(randoms)
        self.lib.orc_step(self.h, nsteps, _f(r))

    def observe(self, r, u, v):
        ro, uo, vo, wo = (np.empty(self.nxy, np.float32) for _ in range(4))
        self.lib.orc_observe(self.h, _f(_f32(r)), _f(_f32(u)), _f(_f32(v)), _f(ro), _f(uo), _f(vo), _f(wo))
        return tuple(a.reshape(self.ny, self.nx) for a in (ro, uo, vo, wo))

    def obs_weight(self, i, j, a, b, var):
        w = ctypes.c_double()
        valid = ctypes.c_int()
        self.lib.orc_obs_weight(ctypes.byref(self.cfg), i, j, a, b, var, ctypes.byref(w), ctypes.byref(valid))
        return w.value, bool(valid.value)

    def assimilate_rows(self, rho_o, u_o, v_o, j0: int, j1: int):
        return self.lib.orc_assimilate_rows(self.h, _f(_f32(rho_o)), _f(_f32(u_o)), _f(_f32(v_o)), None, j0, j1)

    def set_closure(self, params=None, nu_ref: float = 0.0, dx_ref: float = 0.0):
        """Learned eddy-viscosity multiplier in the steps (1313 parameters; None = plain
        Smagorinsky), FP64 under the engine's BF16 operand contract."""
        w = None if params is None else _f32(params)
        return self.lib.orc_set_closure(self.h, None if w is None else _f(w), float(nu_ref), float(dx_ref))

    def nudge(self, rho_o, u_o, v_o):
        """DA_NUDGING (nudging.cu:40-143) of every member, FP64."""
        return self.lib.orc_nudge(self.h, _f(_f32(rho_o)), _f(_f32(u_o)), _f(_f32(v_o)))

    def assimilate(self, rho_o, u_o, v_o, want_lambda: bool = False):
        lam = np.empty(self.nxy * self.M, np.float64) if want_lambda else None
        sweeps = self.lib.orc_assimilate(self.h, _f(_f32(rho_o)), _f(_f32(u_o)), _f(_f32(v_o)), _d(lam))
        return (sweeps, lam.reshape(self.ny, self.nx, self.M)) if want_lambda else sweeps
