"""Python bindings of liblbl, the B200 forecast-and-assimilate engine.

The engine holds all M ensemble members of an LBM2D-LETKF experiment on one GPU.
This module is a thin ctypes layer over the C ABI declared in include/lbl.h, plus
functions named after the reference's host interface so that calling code reads
like the reference's main loop (src/main.cu:80-116):

    update(dat, t)                         -> src/lbm.h:16-29
    DataAssimilator(dat).assimilate(dat,t) -> src/assimilate.h:54-68, src/letkf.cu:120-360
    output(dat, t)                         -> src/io.cu:22-266

The shared library is loaded from the package directory (built in-tree by
``make -C lbm2d-letkf_b200``).  There is no fallback: if liblbl.so is missing or a
call fails, an exception is raised.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Tuple

import numpy as np

_PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(_PKG_DIR, "liblbl.so")

ABI_VERSION = 2
MODE_NATURE, MODE_OBSERVE, MODE_DA_LETKF, MODE_DA_NUDGING = 0, 1, 2, 3
MODES = {"NATURE": MODE_NATURE, "OBSERVE": MODE_OBSERVE, "DA_LETKF": MODE_DA_LETKF, "DA_NUDGING": MODE_DA_NUDGING}
IC_REFERENCE, IC_K4EXP = 0, 1
ENS_INDEPENDENT, ENS_PERTURBED = 0, 1
TIMER_MAIN, TIMER_LETKF = 0, 1
Q = 9

ERRORS = {
    -1: "LBL_ERR_ARG", -2: "LBL_ERR_CUDA", -3: "LBL_ERR_CURAND", -4: "LBL_ERR_IO",
    -5: "LBL_ERR_NAN", -6: "LBL_ERR_STATE", -7: "LBL_ERR_NOMEM", -8: "LBL_ERR_UNSUPPORTED",
    -9: "LBL_ERR_NOCONV", -10: "LBL_ERR_TIMEOUT",
}
LBM_AUTO, LBM_DIRECT, LBM_TMA, LBM_VEC, LBM_VEC2 = 0, 1, 2, 3, 4
STORAGE_F32, STORAGE_F16 = 0, 1
GRAM_F32, GRAM_BF16, GRAM_TF32X3 = 0, 1, 2

# names of the exported C functions (must match include/lbl.h)
EXPORTS = (
    "lbl_config_default", "lbl_create", "lbl_destroy", "lbl_last_error", "lbl_version", "lbl_init",
    "lbl_update", "lbl_update_async", "lbl_assimilate", "lbl_assimilate_async", "lbl_assimilate_files",
    "lbl_cycle_async", "lbl_sync", "lbl_output", "lbl_output_async", "lbl_get_f", "lbl_set_f", "lbl_get_fields",
    "lbl_get_ens_stats", "lbl_get_force", "lbl_get_force_state", "lbl_get_observed",
    "lbl_get_letkf_stats", "lbl_get_diagnostics", "lbl_rmse_uv", "lbl_rmse_uv_async", "lbl_get_stream", "lbl_timer_csv", "lbl_timer_clear",
    "lbl_timer_transit", "lbl_profile_step", "lbl_get_cycle_phases", "lbl_event_record", "lbl_event_elapsed",
    "lbl_letkf_analysis_noalloc", "lbl_bindiff", "lbl_ensemble_stat", "lbl_energy_spectrum",
    "lbl_set_io_prefix", "lbl_h5_write_dataset", "lbl_autotune", "lbl_stream_collide_shape", "lbl_set_stream_collide_shape", "lbl_set_closure", "lbl_closure_generate",
    "lbl_closure_grad", "lbl_closure_train", "lbl_closure_infer", "lbl_batch_create", "lbl_batch_last_error",
    "lbl_batch_cycle_async", "lbl_batch_sync", "lbl_batch_destroy", "lbl_inject", "lbl_set_closure_refresh",
    "lbl_slab_set", "lbl_slab_halo_bytes", "lbl_slab_pack", "lbl_slab_unpack", "lbl_slab_forecast_steps",
    "lbl_slab_forecast_begin", "lbl_slab_forecast_chunk",
)
INJECT_NONE, INJECT_TMA_STALL = 0, 1
CLOSURE_PARAMS, CLOSURE_FEATURES = 1313, 6


class LblError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class Config(ctypes.Structure):
    """Mirror of lbl_config (include/lbl.h): the reference's config.h constants and -D knobs."""

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


_lib = None


def load_library() -> ctypes.CDLL:
    """Load liblbl.so from the package directory; raises if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"liblbl.so not built: {LIB_PATH} (run `make -C lbm2d-letkf_b200`)")
    lib = ctypes.CDLL(LIB_PATH)
    P, I, F, D, U = ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_double), ctypes.c_size_t
    IP = ctypes.POINTER(ctypes.c_int)
    CP = ctypes.POINTER(Config)
    sig = {
        "lbl_config_default": (I, [CP, I, I, I]),
        "lbl_create": (I, [CP, I, ctypes.POINTER(P)]),
        "lbl_destroy": (I, [P]),
        "lbl_last_error": (ctypes.c_char_p, [P]),
        "lbl_version": (ctypes.c_char_p, []),
        "lbl_init": (I, [P, I]),
        "lbl_update": (I, [P, I, I]),
        "lbl_update_async": (I, [P, I, I]),
        "lbl_assimilate": (I, [P, I, F, F, F]),
        "lbl_assimilate_async": (I, [P, I, F, F, F]),
        "lbl_assimilate_files": (I, [P, I, ctypes.c_char_p]),
        "lbl_cycle_async": (I, [P, I, F, F, F, I]),
        "lbl_sync": (I, [P]),
        "lbl_output": (I, [P, I, ctypes.c_char_p]),
        "lbl_output_async": (I, [P, I, ctypes.c_char_p]),
        "lbl_get_f": (I, [P, I, F]),
        "lbl_set_f": (I, [P, I, F]),
        "lbl_get_fields": (I, [P, I, F, F, F, F]),
        "lbl_get_ens_stats": (I, [P, F, F, F, F]),
        "lbl_get_force": (I, [P, F, F]),
        "lbl_get_force_state": (I, [P, F, F, F, F, IP, IP]),
        "lbl_get_observed": (I, [P, F, F, F, F]),
        "lbl_get_letkf_stats": (I, [P, IP, IP, IP, IP]),
        "lbl_get_diagnostics": (I, [P, I, D, D, D]),
        "lbl_rmse_uv": (I, [P, F, F, D]),
        "lbl_rmse_uv_async": (I, [P, F, F, D]),
        "lbl_get_stream": (P, [P]),
        "lbl_set_closure": (I, [P, F, ctypes.c_double, ctypes.c_double]),
        "lbl_closure_generate": (I, [CP, I, I, I, I, I, F, F, U, ctypes.POINTER(U), ctypes.c_char_p, U]),
        "lbl_closure_grad": (I, [F, F, F, U, I, F, F]),
        "lbl_closure_train": (I, [F, F, U, I, I, ctypes.c_float, ctypes.c_uint64, I, F, F, F]),
        "lbl_closure_infer": (I, [F, F, U, I, I, F]),
        "lbl_batch_create": (I, [ctypes.POINTER(P), I, I, ctypes.POINTER(P)]),
        "lbl_batch_last_error": (ctypes.c_char_p, [P]),
        "lbl_batch_cycle_async": (I, [P, I, ctypes.POINTER(F), ctypes.POINTER(F), ctypes.POINTER(F), I]),
        "lbl_batch_sync": (I, [P]),
        "lbl_batch_destroy": (I, [P]),
        "lbl_timer_csv": (I, [P, I, ctypes.c_char_p, U]),
        "lbl_timer_clear": (I, [P, I]),
        "lbl_timer_transit": (I, [P, I, ctypes.c_char_p]),
        "lbl_profile_step": (I, [P, I, D]),
        "lbl_get_cycle_phases": (I, [P, D, D]),
        "lbl_event_record": (I, [P, I]),
        "lbl_event_elapsed": (I, [P, I, I, D]),
        "lbl_letkf_analysis_noalloc": (I, [CP, P, P, P, P, P, IP, ctypes.c_char_p, U]),
        "lbl_bindiff": (I, [ctypes.c_char_p, ctypes.c_char_p, I, D, ctypes.POINTER(ctypes.c_longlong),
                            ctypes.c_char_p, U]),
        "lbl_ensemble_stat": (I, [ctypes.c_char_p, ctypes.c_char_p, I, I, D, ctypes.c_char_p, U]),
        "lbl_energy_spectrum": (I, [F, F, I, I, D]),
        "lbl_set_io_prefix": (I, [P, ctypes.c_char_p]),
        "lbl_autotune": (I, [P, IP, D]),
        "lbl_stream_collide_shape": (I, [P, IP, IP, IP]),
        "lbl_set_stream_collide_shape": (I, [P, I, I]),
        "lbl_inject": (I, [P, I, I]),
        "lbl_set_closure_refresh": (I, [P, I]),
        "lbl_slab_set": (I, [P, I, I, I]),
        "lbl_slab_halo_bytes": (I, [P, I, ctypes.POINTER(U)]),
        "lbl_slab_pack": (I, [P, I, P, P]),
        "lbl_slab_unpack": (I, [P, I, P, P]),
        "lbl_slab_forecast_steps": (I, [P, ctypes.POINTER(I)]),
        "lbl_slab_forecast_begin": (I, [P, I, I]),
        "lbl_slab_forecast_chunk": (I, [P, I]),
        "lbl_h5_write_dataset": (I, [ctypes.c_char_p, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, P, I]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _fp(a: Optional[np.ndarray]):
    if a is None:
        return None
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def _f32(a, n: int) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.float32).reshape(-1)
    if a.size != n:
        raise ValueError(f"expected {n} values, got {a.size}")
    return a


def config_default(mode="NATURE", nx: int = 256, n_ens: int = 1, **overrides) -> Config:
    """The reference's defaults for a run mode at grid nx (= 64*SCALER), with overrides.

    Override names are lbl_config fields (daprune, da_xyprune, letkf_rloc_len, letkf_covinf,
    obs_error_u, cs, tau, ...)."""
    lib = load_library()
    m = MODES[mode] if isinstance(mode, str) else int(mode)
    c = Config()
    rc = lib.lbl_config_default(ctypes.byref(c), m, nx, n_ens)
    if rc != 0:
        raise LblError(rc, "lbl_config_default")
    for k, v in overrides.items():
        if not hasattr(c, k):
            raise KeyError(f"unknown config field {k}")
        setattr(c, k, v)
    return c


class Ensemble:
    """All M members of one experiment on one GPU (the reference's `data` per rank x M,
    plus its DataAssimilator)."""

    def __init__(self, cfg: Config, device: int = 0):
        self.lib = load_library()
        self.cfg = cfg.copy()
        self.nx, self.ny, self.M = cfg.nx, cfg.ny, cfg.n_ens
        self.nxy = cfg.nx * cfg.ny
        h = ctypes.c_void_p()
        rc = self.lib.lbl_create(ctypes.byref(self.cfg), device, ctypes.byref(h))
        self._h = h
        if rc != 0:
            msg = self.lib.lbl_last_error(h).decode() if h.value else "lbl_create"
            if h.value:
                self.lib.lbl_destroy(h)
            self._h = ctypes.c_void_p()
            raise LblError(rc, msg)

    # -- plumbing ---------------------------------------------------------------
    def _check(self, rc: int, what: str):
        if rc != 0:
            raise LblError(rc, f"{what}: {self.lib.lbl_last_error(self._h).decode()}")

    def close(self):
        if self._h and self._h.value:
            self.lib.lbl_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- the path ---------------------------------------------------------------
    def init(self, ens_offset: int = 0):
        self._check(self.lib.lbl_init(self._h, ens_offset), "lbl_init")

    def update(self, t0: int = 0, nsteps: int = 1, sync: bool = True):
        fn = self.lib.lbl_update if sync else self.lib.lbl_update_async
        self._check(fn(self._h, t0, nsteps), "lbl_update")

    def assimilate(self, t: int, rho_o, u_o, v_o, sync: bool = True):
        ro, uo, vo = (_f32(a, self.nxy) for a in (rho_o, u_o, v_o))
        fn = self.lib.lbl_assimilate if sync else self.lib.lbl_assimilate_async
        self._check(fn(self._h, t, _fp(ro), _fp(uo), _fp(vo)), "lbl_assimilate")

    def assimilate_files(self, t: int, io_prefix: str = "io"):
        self._check(self.lib.lbl_assimilate_files(self._h, t, io_prefix.encode()), "lbl_assimilate_files")

    def cycle_async(self, t: int, rho_o, u_o, v_o, n_fc: int):
        if rho_o is None:
            self._check(self.lib.lbl_cycle_async(self._h, t, None, None, None, n_fc), "lbl_cycle_async")
            return
        ro, uo, vo = (_f32(a, self.nxy) for a in (rho_o, u_o, v_o))
        self._check(self.lib.lbl_cycle_async(self._h, t, _fp(ro), _fp(uo), _fp(vo), n_fc), "lbl_cycle_async")

    def sync(self):
        self._check(self.lib.lbl_sync(self._h), "lbl_sync")

    def output(self, t: int, io_prefix: str = "io", sync: bool = True):
        """The reference's output files; sync=False leaves the file writing to a host
        thread (lbl_output_async) that the next output or sync() waits for."""
        fn = self.lib.lbl_output if sync else self.lib.lbl_output_async
        self._check(fn(self._h, t, io_prefix.encode()), "lbl_output")

    # -- accessors --------------------------------------------------------------
    def get_f(self, member: int) -> np.ndarray:
        out = np.empty(Q * self.nxy, np.float32)
        self._check(self.lib.lbl_get_f(self._h, member, _fp(out)), "lbl_get_f")
        return out.reshape(Q, self.ny, self.nx)

    def set_f(self, member: int, f):
        a = _f32(f, Q * self.nxy)
        self._check(self.lib.lbl_set_f(self._h, member, _fp(a)), "lbl_set_f")

    def get_fields(self, member: int) -> Tuple[np.ndarray, ...]:
        r, u, v, w = (np.empty(self.nxy, np.float32) for _ in range(4))
        self._check(self.lib.lbl_get_fields(self._h, member, _fp(r), _fp(u), _fp(v), _fp(w)), "lbl_get_fields")
        return tuple(a.reshape(self.ny, self.nx) for a in (r, u, v, w))

    def ens_stats(self) -> Tuple[np.ndarray, ...]:
        a = [np.empty(self.nxy, np.float32) for _ in range(4)]
        self._check(self.lib.lbl_get_ens_stats(self._h, *(_fp(x) for x in a)), "lbl_get_ens_stats")
        return tuple(x.reshape(self.ny, self.nx) for x in a)

    def force(self) -> Tuple[np.ndarray, np.ndarray]:
        fx, fy = np.empty(self.nxy, np.float32), np.empty(self.nxy, np.float32)
        self._check(self.lib.lbl_get_force(self._h, _fp(fx), _fp(fy)), "lbl_get_force")
        return fx.reshape(self.ny, self.nx), fy.reshape(self.ny, self.nx)

    def force_state(self) -> dict:
        n = ctypes.c_int()
        cur = ctypes.c_int()
        self._check(self.lib.lbl_get_force_state(self._h, None, None, None, None, ctypes.byref(n), None),
                    "lbl_get_force_state")
        r, kx, ky, amp = (np.empty(4 * n.value, np.float32), np.empty(n.value, np.float32),
                          np.empty(n.value, np.float32), np.empty(n.value, np.float32))
        self._check(self.lib.lbl_get_force_state(self._h, _fp(r), _fp(kx), _fp(ky), _fp(amp), ctypes.byref(n),
                                                 ctypes.byref(cur)), "lbl_get_force_state")
        return {"randoms": r, "kx": kx, "ky": ky, "amp": amp, "n_modes": n.value, "cursor": cur.value}

    def observed(self) -> Tuple[np.ndarray, ...]:
        a = [np.empty(self.nxy, np.float32) for _ in range(4)]
        self._check(self.lib.lbl_get_observed(self._h, *(_fp(x) for x in a)), "lbl_get_observed")
        return tuple(x.reshape(self.ny, self.nx) for x in a)

    def letkf_stats(self) -> dict:
        a, b, c, d = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self._check(self.lib.lbl_get_letkf_stats(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c),
                                                 ctypes.byref(d)), "lbl_get_letkf_stats")
        return {"max_sweeps": a.value, "n_noconv": b.value, "nan": c.value,
                "mean_sweeps": d.value / float(self.nxy)}

    def diagnostics(self, member: int = -1) -> dict:
        e, z, m = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.lbl_get_diagnostics(self._h, member, ctypes.byref(e), ctypes.byref(z), ctypes.byref(m)),
                    "lbl_get_diagnostics")
        return {"energy": e.value, "enstrophy": z.value, "mass": m.value}

    def rmse_uv(self, u_true, v_true) -> float:
        ut, vt = _f32(u_true, self.nxy), _f32(v_true, self.nxy)
        r = ctypes.c_double()
        self._check(self.lib.lbl_rmse_uv(self._h, _fp(ut), _fp(vt), ctypes.byref(r)), "lbl_rmse_uv")
        return r.value

    def rmse_uv_async(self, u_true: np.ndarray, v_true: np.ndarray, out: np.ndarray, index: int = 0):
        """lbl_rmse_uv_async: enqueue the RMSE of the ensemble mean (u, v) against the true
        fields; out[index] (a float64 array, pinned for an asynchronous copy) holds it once
        the context's stream has passed this point (sync(), or event_elapsed on a later
        event).  u_true and v_true must be contiguous float32 arrays of nx*ny values that
        stay alive and unchanged until then."""
        for a in (u_true, v_true):
            if a.dtype != np.float32 or not a.flags["C_CONTIGUOUS"] or a.size != self.nxy:
                raise ValueError("rmse_uv_async needs contiguous float32 arrays of nx*ny values")
        if out.dtype != np.float64 or not 0 <= index < out.size:
            raise ValueError("out must be a float64 array with a slot at index")
        ptr = ctypes.cast(out.ctypes.data + 8 * index, ctypes.POINTER(ctypes.c_double))
        self._check(self.lib.lbl_rmse_uv_async(self._h, _fp(u_true), _fp(v_true), ptr), "lbl_rmse_uv_async")

    def stream(self) -> int:
        """The context's cudaStream_t as an integer (lbl_get_stream), e.g. for
        torch.cuda.ExternalStream."""
        return int(self.lib.lbl_get_stream(self._h) or 0)

    def timer_csv(self, which: int = TIMER_MAIN) -> str:
        n = self.lib.lbl_timer_csv(self._h, which, None, 0)
        if n < 0:
            raise LblError(n, "lbl_timer_csv")
        buf = ctypes.create_string_buffer(n + 1)
        self.lib.lbl_timer_csv(self._h, which, buf, n + 1)
        return buf.value.decode()

    def profile_step(self, n: int) -> float:
        """Average milliseconds per launch of the fused stream-collide kernel (CUDA events)."""
        ms = ctypes.c_double()
        self._check(self.lib.lbl_profile_step(self._h, n, ctypes.byref(ms)), "lbl_profile_step")
        return ms.value

    def autotune(self) -> Tuple[int, float]:
        """Pick the stream-collide strip height for this grid and ensemble (before init)."""
        ty, ms = ctypes.c_int(), ctypes.c_double()
        self._check(self.lib.lbl_autotune(self._h, ctypes.byref(ty), ctypes.byref(ms)), "lbl_autotune")
        return ty.value, ms.value

    def launch_shape(self) -> dict:
        """The stream-collide launch shape (lbl_stream_collide_shape)."""
        c, p, ty = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        self._check(self.lib.lbl_stream_collide_shape(self._h, ctypes.byref(c), ctypes.byref(p), ctypes.byref(ty)),
                    "lbl_stream_collide_shape")
        return {"columns_per_thread": c.value, "prefetch": bool(p.value), "strip_rows": ty.value}

    def set_launch_shape(self, prefetch: bool = True, strip_rows: int = 0):
        """Set the stream-collide launch shape (lbl_set_stream_collide_shape); strip_rows 0
        takes the heuristic's."""
        self._check(self.lib.lbl_set_stream_collide_shape(self._h, int(bool(prefetch)), int(strip_rows)),
                    "lbl_set_stream_collide_shape")

    # -- y-slab split (lbl_slab_set; the exchange between ranks is lbl.slab's) ----------
    def slab_set(self, ny_global: int, row0: int, halo: int):
        """Make this context the rows [row0, row0 + ny - 2 halo) of a grid of ny_global rows,
        with `halo` rows on each side (lbl_slab_set; between construction and init)."""
        self._check(self.lib.lbl_slab_set(self._h, int(ny_global), int(row0), int(halo)), "lbl_slab_set")

    def slab_forecast_steps(self) -> int:
        """The most steps one chunked forecast can begin (lbl_slab_forecast_steps)."""
        n = ctypes.c_int()
        self._check(self.lib.lbl_slab_forecast_steps(self._h, ctypes.byref(n)), "lbl_slab_forecast_steps")
        return n.value

    def slab_forecast_begin(self, t0: int, nsteps: int):
        """Compute the forcing of the next nsteps steps at once (lbl_slab_forecast_begin)."""
        self._check(self.lib.lbl_slab_forecast_begin(self._h, int(t0), int(nsteps)), "lbl_slab_forecast_begin")

    def slab_forecast_chunk(self, k: int):
        """Advance k begun steps on the context's stream (lbl_slab_forecast_chunk)."""
        self._check(self.lib.lbl_slab_forecast_chunk(self._h, int(k)), "lbl_slab_forecast_chunk")

    def slab_halo_bytes(self, rows: int) -> int:
        """Bytes of one packed halo buffer of `rows` rows (lbl_slab_halo_bytes)."""
        n = ctypes.c_size_t()
        self._check(self.lib.lbl_slab_halo_bytes(self._h, int(rows), ctypes.byref(n)), "lbl_slab_halo_bytes")
        return n.value

    def slab_pack(self, rows: int, to_prev: int, to_next: int):
        """Pack the rows the neighbours need into two device buffers (addresses), on the
        context's stream (lbl_slab_pack)."""
        self._check(self.lib.lbl_slab_pack(self._h, int(rows), ctypes.c_void_p(to_prev), ctypes.c_void_p(to_next)),
                    "lbl_slab_pack")

    def slab_unpack(self, rows: int, from_prev: int, from_next: int):
        """Unpack the neighbours' packed rows into the halos, on the context's stream
        (lbl_slab_unpack)."""
        self._check(self.lib.lbl_slab_unpack(self._h, int(rows), ctypes.c_void_p(from_prev),
                                             ctypes.c_void_p(from_next)), "lbl_slab_unpack")

    def set_closure_refresh(self, steps: int):
        """Run the closure's network every `steps` steps and hold each cell's multiplier
        between (lbl_set_closure_refresh); 1 = every step."""
        self._check(self.lib.lbl_set_closure_refresh(self._h, int(steps)), "lbl_set_closure_refresh")

    def inject(self, what: int, value: int = 0):
        """Fault injection for failure-path tests (lbl_inject): INJECT_TMA_STALL makes the
        TMA stream-collide's bounded waits run out after `value` polls; INJECT_NONE clears."""
        self._check(self.lib.lbl_inject(self._h, what, value), "lbl_inject")

    def set_closure(self, params=None, nu_ref: float = 0.0, dx_ref: float = 0.0):
        """Learned eddy-viscosity closure in the stream-collide (params: 1313 floats), or
        plain Smagorinsky again (params None).  nu_ref, dx_ref: the training's feature
        scales (0: this run's nu and h_ref/255)."""
        if params is None:
            self._check(self.lib.lbl_set_closure(self._h, None, 0.0, 0.0), "lbl_set_closure")
            return
        w = np.ascontiguousarray(params, dtype=np.float32)
        if w.size != CLOSURE_PARAMS:
            raise ValueError(f"closure parameters: {w.size} values, expected {CLOSURE_PARAMS}")
        self._check(self.lib.lbl_set_closure(self._h, _fp(w), float(nu_ref), float(dx_ref)), "lbl_set_closure")

    def set_io_prefix(self, prefix: str):
        """Directory prefix of the LETKF matrix dumps (cfg.write_mat)."""
        self._check(self.lib.lbl_set_io_prefix(self._h, prefix.encode()), "lbl_set_io_prefix")

    def cycle_phases(self) -> tuple:
        """(analysis_ms, forecast_ms) of the last graph, from events recorded inside it."""
        a, f = ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.lbl_get_cycle_phases(self._h, ctypes.byref(a), ctypes.byref(f)), "lbl_get_cycle_phases")
        return a.value, f.value

    def event_record(self, slot: int):
        """Record CUDA event `slot` (0..7) on the engine's stream."""
        self._check(self.lib.lbl_event_record(self._h, slot), "lbl_event_record")

    def event_elapsed(self, a: int, b: int) -> float:
        """Milliseconds between recorded events a and b (waits for b)."""
        ms = ctypes.c_double()
        self._check(self.lib.lbl_event_elapsed(self._h, a, b, ctypes.byref(ms)), "lbl_event_elapsed")
        return ms.value

    def timer_transit(self, tag: str, which: int = TIMER_MAIN):
        self._check(self.lib.lbl_timer_transit(self._h, which, tag.encode()), "lbl_timer_transit")

    def timer_clear(self, which: int = TIMER_MAIN):
        self._check(self.lib.lbl_timer_clear(self._h, which), "lbl_timer_clear")


# --- functions named after the reference's host interface -----------------------
def update(dat: Ensemble, t: int):
    """One LBM step of every member (src/lbm.h:16-29)."""
    dat.update(t, 1)


class DataAssimilator:
    """LETKF facade (src/assimilate.h:14-82); observations are read from `io_prefix`."""

    def __init__(self, dat: Ensemble, io_prefix: str = "io"):
        self.io_prefix = io_prefix

    def assimilate(self, dat: Ensemble, t: int):
        dat.assimilate_files(t, self.io_prefix)

    def get_timer(self, dat: Ensemble) -> str:
        return dat.timer_csv(TIMER_LETKF)


def output(dat: Ensemble, t: int, io_prefix: str = "io"):
    """Field files and ensemble statistics (src/io.cu:22-266)."""
    dat.output(t, io_prefix)


def version() -> str:
    return load_library().lbl_version().decode()


# ---- evaluation measures over the output files (host only) ----------------------------

def bindiff(dir0: str, dir1: str, step: int) -> Tuple[float, int]:
    """RMSE of (u, v) between two output directories at one step (bindiff/main.cpp)."""
    lib = load_library()
    r, n = ctypes.c_double(), ctypes.c_longlong()
    err = ctypes.create_string_buffer(512)
    rc = lib.lbl_bindiff(dir0.encode(), dir1.encode(), step, ctypes.byref(r), ctypes.byref(n), err, 512)
    if rc != 0:
        raise LblError(rc, err.value.decode())
    return r.value, n.value


def ensemble_stat(nature_dir: str, ens_dir: str, n_ens: int, step: int) -> dict:
    """Spread and RMSE of the ensemble mean against nature (ensemble_stat/main.cpp)."""
    lib = load_library()
    out = (ctypes.c_double * 5)()
    err = ctypes.create_string_buffer(512)
    rc = lib.lbl_ensemble_stat(nature_dir.encode(), ens_dir.encode(), n_ens, step, out, err, 512)
    if rc != 0:
        raise LblError(rc, err.value.decode())
    return dict(zip(("spread", "rmse", "rho_spread", "rho_rmse", "max"), list(out)))


def energy_spectrum(u, v) -> np.ndarray:
    """E(k), k = 0..nx/2, of postprocess/fourier.ipynb cell 2 for one (u, v) field."""
    lib = load_library()
    u = np.ascontiguousarray(u, dtype=np.float32)
    v = np.ascontiguousarray(v, dtype=np.float32)
    ny, nx = u.shape
    ek = np.empty(nx // 2 + 1, np.float64)
    rc = lib.lbl_energy_spectrum(_fp(u), _fp(v), nx, ny, ek.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    if rc != 0:
        raise LblError(rc, "lbl_energy_spectrum")
    return ek


# ---- learned closure: data, training, inference (no counterpart in the reference) ------

def closure_generate(fine: Config, filter: int, spinup: int, n_snapshots: int, spacing: int,
                     device: int = 0) -> Tuple[np.ndarray, np.ndarray]:
    """(features [n][6], targets [n]) from box-filtered runs of the fine configuration."""
    lib = load_library()
    nc = (fine.nx // filter) * (fine.ny // filter) * fine.n_ens * n_snapshots
    feat = np.empty((nc, CLOSURE_FEATURES), np.float32)
    tgt = np.empty(nc, np.float32)
    n = ctypes.c_size_t()
    err = ctypes.create_string_buffer(512)
    cfg = fine.copy()
    rc = lib.lbl_closure_generate(ctypes.byref(cfg), filter, spinup, n_snapshots, spacing, device, _fp(feat),
                                  _fp(tgt), nc, ctypes.byref(n), err, 512)
    if rc != 0:
        raise LblError(rc, err.value.decode())
    return feat[: n.value], tgt[: n.value]


def closure_grad(params, features, targets, device: int = 0) -> Tuple[float, np.ndarray]:
    """Mean-square loss and its gradient (the GPU's fused forward/backward)."""
    lib = load_library()
    w = np.ascontiguousarray(params, dtype=np.float32)
    x = np.ascontiguousarray(features, dtype=np.float32)
    t = np.ascontiguousarray(targets, dtype=np.float32)
    g = np.empty(CLOSURE_PARAMS, np.float32)
    loss = ctypes.c_float()
    rc = lib.lbl_closure_grad(_fp(w), _fp(x), _fp(t), t.size, device, _fp(g), ctypes.byref(loss))
    if rc != 0:
        raise LblError(rc, "lbl_closure_grad")
    return float(loss.value), g


def closure_train(features, targets, iters: int, batch: int = 8192, lr: float = 1e-3, seed: int = 1,
                  device: int = 0, init=None) -> Tuple[np.ndarray, np.ndarray]:
    """Adam on the GPU; returns (parameters, minibatch loss curve)."""
    lib = load_library()
    x = np.ascontiguousarray(features, dtype=np.float32)
    t = np.ascontiguousarray(targets, dtype=np.float32)
    w = np.empty(CLOSURE_PARAMS, np.float32)
    curve = np.empty(iters, np.float32)
    w0 = None if init is None else np.ascontiguousarray(init, dtype=np.float32)
    rc = lib.lbl_closure_train(_fp(x), _fp(t), t.size, iters, batch, lr, seed, device,
                               None if w0 is None else _fp(w0), _fp(w), _fp(curve))
    if rc != 0:
        raise LblError(rc, "lbl_closure_train")
    return w, curve


def closure_infer(params, features, path: int = 0, device: int = 0) -> np.ndarray:
    """Multipliers for feature rows: path 0 = the tensor-core form of the stream-collide,
    path 1 = the per-thread FP32 form."""
    lib = load_library()
    w = np.ascontiguousarray(params, dtype=np.float32)
    x = np.ascontiguousarray(features, dtype=np.float32)
    out = np.empty(x.shape[0], np.float32)
    rc = lib.lbl_closure_infer(_fp(w), _fp(x), x.shape[0], path, device, _fp(out))
    if rc != 0:
        raise LblError(rc, "lbl_closure_infer")
    return out


class Batch:
    """Several ensembles cycled together: per cycle one CUDA graph with every
    experiment's analysis and forcing beside each other and one batched persistent
    stream-collide launch per step for all of them (lbl_batch_*)."""

    def __init__(self, ensembles, strip_rows: int = 0):
        self.lib = load_library()
        self.members = list(ensembles)
        arr = (ctypes.c_void_p * len(self.members))(*[e._h.value for e in self.members])
        h = ctypes.c_void_p()
        rc = self.lib.lbl_batch_create(arr, len(self.members), strip_rows, ctypes.byref(h))
        self._h = h
        if rc != 0:
            msg = self.lib.lbl_batch_last_error(h).decode() if h.value else "lbl_batch_create"
            if h.value:
                self.lib.lbl_batch_destroy(h)
            self._h = ctypes.c_void_p()
            raise LblError(rc, msg)

    def _check(self, rc, what):
        if rc != 0:
            raise LblError(rc, f"{what}: {self.lib.lbl_batch_last_error(self._h).decode()}")

    def cycle_async(self, t: int, observations=None, n_fc: int = 100):
        """observations: None, or one (rho, u, v) tuple (or None) per ensemble."""
        n = len(self.members)
        if observations is None:
            self._check(self.lib.lbl_batch_cycle_async(self._h, t, None, None, None, n_fc), "lbl_batch_cycle_async")
            return
        keep = []
        ptrs = [(ctypes.POINTER(ctypes.c_float) * n)() for _ in range(3)]
        for i, (ens, obs) in enumerate(zip(self.members, observations)):
            if obs is None:
                continue
            for k, a in enumerate(obs):
                a = _f32(a, ens.nxy)
                keep.append(a)
                ptrs[k][i] = _fp(a)
        self._check(self.lib.lbl_batch_cycle_async(self._h, t, *ptrs, n_fc), "lbl_batch_cycle_async")

    def sync(self):
        self._check(self.lib.lbl_batch_sync(self._h), "lbl_batch_sync")

    def close(self):
        if self._h and self._h.value:
            self.lib.lbl_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
