"""ctypes binding of libcfdgpu.so (the C ABI in include/cfdgpu.h and
include/cfdgpu_host.h).

The Solver class follows the reference's plugin contract
(euler_equations/euler_simulation_code/headers/problem_base.hpp:18-40 and
headers/simulation.hpp:36-67): upload the initial grid, then per step
``compute_dt`` followed by ``step``; ``advance`` runs the same loop on the
device.  There is no CPU fallback: constructing a Solver without the built
library or without a CUDA device raises.
"""
from __future__ import annotations

import ctypes as C
import math
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "lib" / "libcfdgpu.so"

EULER, ALLAIRE = 0, 1
FP64, MIXED, FP64_FAST = 0, 1, 2  # CFD_PREC_*
TRANSMISSIVE, REFLECTIVE = 0, 1
LIMITERS = {"minmod": 0, "vanleer": 1, "mc": 2, "unlimited": 3}
FLUX = {"MUSCL": 0, "Godunov": 1}
SPLIT = {"naive": 0, "strang": 1}
WAVESPEED = {"davis": 0, "pvrs": 1}
GHOSTED_AOS, SOA, GHOSTED_AOS_AS_REFERENCE = 0, 1, 2
RECIPE = {"four_quadrant": 1, "shock_bubbles": 2, "water_shock_air_bubble": 3}
COUNTERS = ["unphysical_input", "slope_zeroed", "first_order", "fixup", "unphysical_output"]


class CfdError(RuntimeError):
    pass


class Config(C.Structure):
    """Mirror of ``cfd_config``."""

    _fields_ = [
        ("model", C.c_int), ("precision", C.c_int), ("nx", C.c_int), ("ny", C.c_int),
        ("x0", C.c_double), ("y0", C.c_double), ("dx", C.c_double), ("dy", C.c_double),
        ("gamma1", C.c_double), ("pinf1", C.c_double), ("gamma2", C.c_double),
        ("pinf2", C.c_double), ("bc", C.c_int * 4), ("cfl", C.c_double), ("T", C.c_double),
        ("limiter", C.c_int), ("flux_solver", C.c_int), ("splitting", C.c_int),
        ("wavespeed", C.c_int), ("z_min", C.c_double), ("fix_dy_halfstep", C.c_int),
        ("stream", C.c_void_p),
    ]

    @property
    def nvar(self) -> int:
        return 4 if self.model == EULER else 6

    @property
    def ghosts(self) -> int:
        return 1 if self.flux_solver == FLUX["Godunov"] else 2

    def ghosted_shape(self) -> tuple[int, int, int]:
        g = self.ghosts
        return (self.ny + 2 * g, self.nx + 2 * g, self.nvar)

    def copy(self) -> "Config":
        c = Config()
        C.pointer(c)[0] = self
        return c


class Status(C.Structure):
    _fields_ = [
        ("n", C.c_int), ("done", C.c_int), ("t", C.c_double), ("dt_next", C.c_double),
        ("maxu", C.c_double), ("maxv", C.c_double), ("mass1", C.c_double), ("mass2", C.c_double),
        ("counters", C.c_ulonglong * 8),
    ]

    def counter_dict(self) -> dict[str, int]:
        return {k: int(self.counters[i]) for i, k in enumerate(COUNTERS)}


class Settings(C.Structure):
    """cfd_settings (include/cfdgpu_host.h)."""
    _fields_ = [("Nx", C.c_int), ("Ny", C.c_int), ("CFL", C.c_double),
                ("splitting_scheme", C.c_char * 64), ("test_case", C.c_char * 128),
                ("output_freq", C.c_int), ("outputpath", C.c_char * 512),
                ("basename", C.c_char * 768), ("flux_solver", C.c_char * 32),
                ("riemann_solver", C.c_char * 32), ("problem", C.c_char * 32),
                ("precision", C.c_char * 16), ("limiter", C.c_char * 16),
                ("wavespeed", C.c_char * 16), ("steps", C.c_int), ("alpha_clip", C.c_double),
                ("fix_dy_halfstep", C.c_int), ("seed", C.c_uint64), ("nbubbles", C.c_int)]


class ServerOptions(C.Structure):
    _fields_ = [("precision", C.c_int), ("budget_bytes", C.c_size_t),
                ("budget_fraction", C.c_double), ("ticks_per_round", C.c_int),
                ("stream", C.c_void_p), ("host_pinned_bytes", C.c_size_t)]


class RequestInfo(C.Structure):
    _fields_ = [("state", C.c_int), ("error", C.c_int), ("steps", C.c_int), ("t", C.c_double),
                ("submit_s", C.c_double), ("queue_s", C.c_double), ("run_s", C.c_double),
                ("latency_s", C.c_double)]


class ServerStats(C.Structure):
    _fields_ = [("completed", C.c_int64), ("admitted", C.c_int64), ("queued", C.c_int64),
                ("running", C.c_int64), ("max_running", C.c_int64), ("rounds", C.c_int64),
                ("cell_updates", C.c_double), ("busy_s", C.c_double), ("wall_s", C.c_double),
                ("device_s", C.c_double), ("used_bytes", C.c_size_t), ("budget_bytes", C.c_size_t)]


REQ_DONE, REQ_FAILED = 2, 3

_lib: C.CDLL | None = None


def lib() -> C.CDLL:
    """Loads libcfdgpu.so; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise CfdError(f"{LIB_PATH} not built (run cfd-art_b200/build.py)")
        L = C.CDLL(str(LIB_PATH))
        vp, dp, ip = C.c_void_p, C.POINTER(C.c_double), C.c_int
        cfgp = C.POINTER(Config)
        sig = {
            "cfd_version": (C.c_char_p, []),
            "cfd_last_error": (ip, [C.c_char_p, C.c_size_t]),
            "cfd_nvar": (ip, [ip]),
            "cfd_device_bytes": (ip, [cfgp, C.POINTER(C.c_size_t)]),
            "cfd_create": (ip, [cfgp, C.POINTER(vp)]),
            "cfd_destroy": (ip, [vp]),
            "cfd_upload": (ip, [vp, dp, ip, ip, C.c_double]),
            "cfd_upload_device": (ip, [vp, vp, ip, C.c_double]),
            "cfd_upload_recipe": (ip, [vp, ip, C.c_uint64, ip, ip, C.c_double]),
            "cfd_upload_case": (ip, [vp, C.c_char_p, C.c_uint64, ip, C.c_double]),
            "cfd_download": (ip, [vp, dp, ip]),
            "cfd_schlieren": (ip, [vp, ip, dp]),
            "cfd_compute_dt": (ip, [vp, ip, C.c_double, dp]),
            "cfd_step": (ip, [vp, C.c_double]),
            "cfd_advance": (ip, [vp, ip]),
            "cfd_get_status": (ip, [vp, C.POINTER(Status)]),
            "cfd_reset_counters": (ip, [vp]),
            "cfd_set_reference_ghosts": (ip, [vp, ip]),
            "cfd_checkpoint_save": (ip, [vp, C.c_char_p]),
            "cfd_checkpoint_load": (ip, [vp, C.c_char_p]),
            "cfd_checkpoint_info": (ip, [C.c_char_p, cfgp, C.POINTER(ip), dp]),
            "cfd_batch_save": (ip, [vp, ip, C.c_char_p]),
            "cfd_batch_restore": (ip, [vp, C.c_char_p, ip, C.POINTER(ip)]),
            "cfd_set_kernel_timing": (ip, [vp, ip]),
            "cfd_kernel_times": (ip, [vp, dp, C.POINTER(ip)]),
            "cfd_reset_kernel_times": (ip, [vp]),
            "cfd_synchronize": (ip, [vp]),
            "cfd_state_device": (ip, [vp, C.POINTER(vp), C.POINTER(C.c_int64), C.POINTER(ip)]),
            "cfd_face_flux": (ip, [cfgp, ip, dp, C.c_double, C.c_double, dp, dp, dp]),
            "cfd_ic_grid_elems": (ip, [cfgp, C.POINTER(C.c_size_t)]),
            "cfd_case_config": (ip, [ip, C.c_char_p, ip, ip, ip, cfgp]),
            "cfd_case_ic": (ip, [cfgp, C.c_char_p, C.c_uint64, dp]),
            "cfd_recipe_config": (ip, [ip, ip, ip, cfgp]),
            "cfd_recipe_ic": (ip, [cfgp, ip, C.c_uint64, ip, dp]),
            "cfd_write_state": (ip, [cfgp, dp, C.c_char_p, C.c_double]),
            "cfd_write_schlieren": (ip, [cfgp, dp, C.c_char_p, C.c_double]),
            "cfd_write_schlieren_field": (ip, [cfgp, dp, C.c_char_p, C.c_double]),
            "cfd_write_masschange": (ip, [cfgp, C.c_char_p, ip, dp, dp, dp]),
            "cfd_write_lineout": (ip, [cfgp, dp, C.c_char_p, ip]),
            "cfd_read_settings": (ip, [C.c_char_p, C.POINTER(Settings)]),
            "cfd_settings_config": (ip, [C.POINTER(Settings), cfgp]),
            "cfd_settings_ic": (ip, [C.POINTER(Settings), cfgp, dp]),
            "cfd_batch_create": (ip, [vp, C.c_size_t, C.POINTER(vp)]),
            "cfd_batch_destroy": (ip, [vp]),
            "cfd_batch_member_bytes": (ip, [cfgp, C.POINTER(C.c_size_t)]),
            "cfd_batch_add": (ip, [vp, cfgp, dp, ip, C.POINTER(ip)]),
            "cfd_batch_add_recipe": (ip, [vp, cfgp, ip, C.c_uint64, ip, ip, C.POINTER(ip)]),
            "cfd_batch_remove": (ip, [vp, ip]),
            "cfd_batch_size": (ip, [vp, C.POINTER(ip), C.POINTER(C.c_size_t),
                                    C.POINTER(C.c_size_t)]),
            "cfd_batch_step": (ip, [vp, ip]),
            "cfd_batch_step_timed": (ip, [vp, ip, dp, dp, C.POINTER(ip)]),
            "cfd_batch_autotune": (ip, [vp, ip, dp]),
            "cfd_batch_set_shapes": (ip, [vp, ip, ip, ip]),
            "cfd_batch_get_shapes": (ip, [vp, ip, C.POINTER(ip), C.POINTER(ip)]),
            "cfd_batch_set_march_rows": (ip, [vp, ip, ip]),
            "cfd_batch_get_march_rows": (ip, [vp, ip, C.POINTER(ip)]),
            "cfd_batch_get_segment_rows": (ip, [vp, ip, ip, C.POINTER(ip)]),
            "cfd_batch_status": (ip, [vp, ip, C.POINTER(Status)]),
            "cfd_batch_poll_issue": (ip, [vp]),
            "cfd_batch_poll_collect": (ip, [vp, ip, C.POINTER(ip), C.POINTER(ip), C.POINTER(ip), dp,
                                        C.POINTER(ip)]),
            "cfd_batch_poll": (ip, [vp, ip, C.POINTER(ip), C.POINTER(ip), C.POINTER(ip), dp,
                                    C.POINTER(ip)]),
            "cfd_batch_download": (ip, [vp, ip, dp, ip]),
            "cfd_server_create": (ip, [C.POINTER(ServerOptions), C.POINTER(vp)]),
            "cfd_server_submit": (ip, [vp, cfgp, dp, ip, C.POINTER(C.c_int64)]),
            "cfd_server_submit_recipe": (ip, [vp, cfgp, ip, C.c_uint64, ip, ip,
                                              C.POINTER(C.c_int64)]),
            "cfd_server_wait": (ip, [vp, C.c_int64, C.c_double, C.POINTER(RequestInfo), dp]),
            "cfd_server_release": (ip, [vp, C.c_int64]),
            "cfd_server_get_stats": (ip, [vp, C.POINTER(ServerStats)]),
            "cfd_server_destroy": (ip, [vp]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def last_error() -> str:
    buf = C.create_string_buffer(1024)
    lib().cfd_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(rc: int, what: str = "") -> None:
    if rc != 0:
        raise CfdError(f"{what} failed ({rc}): {last_error()}")


def _dp(a: np.ndarray):
    if a.dtype != np.float64 or not a.flags.c_contiguous:
        raise ValueError("expected a C-contiguous float64 array")
    return a.ctypes.data_as(C.POINTER(C.c_double))


def case_config(model: int, test_case: str, nx: int, ny: int, flux_solver: str = "MUSCL") -> Config:
    cfg = Config()
    check(lib().cfd_case_config(model, test_case.encode(), nx, ny, FLUX[flux_solver],
                                C.byref(cfg)), f"case_config({test_case})")
    return cfg


def case_ic(cfg: Config, test_case: str, seed: int = 0) -> np.ndarray:
    grid = np.zeros(cfg.ghosted_shape())
    check(lib().cfd_case_ic(C.byref(cfg), test_case.encode(), seed, _dp(grid)),
          f"case_ic({test_case})")
    return grid


def recipe_config(name: str, nx: int, ny: int) -> Config:
    cfg = Config()
    check(lib().cfd_recipe_config(RECIPE[name], nx, ny, C.byref(cfg)), f"recipe_config({name})")
    return cfg


def recipe_ic(cfg: Config, name: str, seed: int = 20261203, nbubbles: int = 32) -> np.ndarray:
    grid = np.zeros(cfg.ghosted_shape())
    check(lib().cfd_recipe_ic(C.byref(cfg), RECIPE[name], seed, nbubbles, _dp(grid)),
          f"recipe_ic({name})")
    return grid


def checkpoint_info(path) -> tuple[Config, int, float]:
    """Configuration, step count and time stored in a checkpoint file."""
    cfg = Config()
    n = C.c_int()
    t = C.c_double()
    check(lib().cfd_checkpoint_info(str(path).encode(), C.byref(cfg), C.byref(n), C.byref(t)),
          "cfd_checkpoint_info")
    return cfg, n.value, t.value


def face_flux(cfg: Config, stencils: np.ndarray, dt: float, dx: float):
    """Device flux of independent faces: stencils (nfaces, 4|2, nvar)."""
    st = np.ascontiguousarray(stencils, dtype=np.float64)
    nf = st.shape[0]
    nv = cfg.nvar
    flux = np.zeros((nf, nv))
    us = np.zeros(nf)
    zs = np.zeros(nf)
    check(lib().cfd_face_flux(C.byref(cfg), nf, _dp(st), dt, dx, _dp(flux), _dp(us), _dp(zs)),
          "face_flux")
    return flux, us, (zs if cfg.model == ALLAIRE else None)


class Solver:
    """One device-resident solve (cfd_create ... cfd_destroy)."""

    def __init__(self, cfg: Config):
        self.cfg = cfg.copy()
        h = C.c_void_p()
        check(lib().cfd_create(C.byref(self.cfg), C.byref(h)), "cfd_create")
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().cfd_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def upload(self, grid: np.ndarray, n: int = 0, t: float = 0.0, layout: int = GHOSTED_AOS):
        check(lib().cfd_upload(self._h, _dp(grid), layout, n, t), "cfd_upload")

    def upload_device(self, ptr: int, n: int = 0, t: float = 0.0):
        check(lib().cfd_upload_device(self._h, C.c_void_p(ptr), n, t), "cfd_upload_device")

    def upload_recipe(self, name: str, seed: int = 20261203, nbubbles: int = 32, n: int = 0,
                      t: float = 0.0):
        """Builds a recipe's initial condition on the device."""
        check(lib().cfd_upload_recipe(self._h, RECIPE[name], seed, nbubbles, n, t),
              f"cfd_upload_recipe({name})")

    def upload_case(self, test_case: str, seed: int = 0, n: int = 0, t: float = 0.0):
        """Builds a named test case's initial condition on the device."""
        check(lib().cfd_upload_case(self._h, test_case.encode(), seed, n, t),
              f"cfd_upload_case({test_case})")

    def save(self, path) -> None:
        check(lib().cfd_checkpoint_save(self._h, str(path).encode()), "cfd_checkpoint_save")

    def load(self, path) -> None:
        check(lib().cfd_checkpoint_load(self._h, str(path).encode()), "cfd_checkpoint_load")

    def set_reference_ghosts(self, enable: bool = True) -> None:
        check(lib().cfd_set_reference_ghosts(self._h, int(enable)), "cfd_set_reference_ghosts")

    def download(self, layout: int = GHOSTED_AOS, out: np.ndarray | None = None) -> np.ndarray:
        c = self.cfg
        if out is None:
            shape = c.ghosted_shape() if layout != SOA else (c.nvar, c.ny, c.nx)
            out = np.empty(shape)
        check(lib().cfd_download(self._h, _dp(out), layout), "cfd_download")
        return out

    def schlieren(self, ghosts: int = GHOSTED_AOS) -> np.ndarray:
        """|grad rho| of every interior cell, computed on the device, (ny, nx)."""
        out = np.empty((self.cfg.ny, self.cfg.nx))
        check(lib().cfd_schlieren(self._h, ghosts, _dp(out)), "cfd_schlieren")
        return out

    def compute_dt(self, n: int, t: float) -> float:
        dt = C.c_double()
        check(lib().cfd_compute_dt(self._h, n, t, C.byref(dt)), "cfd_compute_dt")
        return dt.value

    def step(self, dt: float) -> None:
        check(lib().cfd_step(self._h, dt), "cfd_step")

    def advance(self, max_steps: int) -> None:
        check(lib().cfd_advance(self._h, max_steps), "cfd_advance")

    def status(self) -> Status:
        st = Status()
        check(lib().cfd_get_status(self._h, C.byref(st)), "cfd_get_status")
        return st

    def set_kernel_timing(self, on: bool) -> None:
        check(lib().cfd_set_kernel_timing(self._h, int(on)), "cfd_set_kernel_timing")

    def kernel_times(self):
        ms = (C.c_double * 2)()
        n = (C.c_int * 2)()
        check(lib().cfd_kernel_times(self._h, ms, n), "cfd_kernel_times")
        return [ms[0], ms[1]], [n[0], n[1]]

    def reset_kernel_times(self) -> None:
        check(lib().cfd_reset_kernel_times(self._h), "cfd_reset_kernel_times")

    def reset_counters(self) -> None:
        check(lib().cfd_reset_counters(self._h), "cfd_reset_counters")

    def synchronize(self) -> None:
        check(lib().cfd_synchronize(self._h), "cfd_synchronize")

    def state_device(self):
        p = C.c_void_p()
        plane = C.c_int64()
        pitch = C.c_int()
        check(lib().cfd_state_device(self._h, C.byref(p), C.byref(plane), C.byref(pitch)),
              "cfd_state_device")
        return p.value, plane.value, pitch.value

    def run_reference_loop(self, max_steps: int, n: int = 0, t: float = 0.0):
        """The reference time loop (headers/simulation.hpp:48-61) driven from
        the host: dt = compute_dt(n, t); step(dt); t += dt; n++; snap."""
        T = self.cfg.T
        taken = 0
        while t < T and taken < max_steps:
            dt = self.compute_dt(n, t)
            self.step(dt)
            t += dt
            n += 1
            taken += 1
            if math.fabs(t - T) < 1e-12:
                t = T
        return taken, n, t


class Batch:
    """Batched mixed-precision solves (cfd_batch_*): members of uneven sizes
    advanced together, each with its own dt and stop condition."""

    def __init__(self, stream: int | None = None, budget_bytes: int = 0):
        h = C.c_void_p()
        check(lib().cfd_batch_create(C.c_void_p(stream) if stream else None, budget_bytes,
                                     C.byref(h)), "cfd_batch_create")
        self._h = h
        self.cfgs: dict[int, Config] = {}

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().cfd_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @staticmethod
    def member_bytes(cfg: Config) -> int:
        n = C.c_size_t()
        check(lib().cfd_batch_member_bytes(C.byref(cfg), C.byref(n)), "cfd_batch_member_bytes")
        return n.value

    def add(self, cfg: Config, grid: np.ndarray, max_steps: int = 0) -> int:
        i = C.c_int()
        check(lib().cfd_batch_add(self._h, C.byref(cfg), _dp(grid), max_steps, C.byref(i)),
              "cfd_batch_add")
        self.cfgs[i.value] = cfg.copy()
        return i.value

    def add_recipe(self, cfg: Config, name: str, seed: int = 20261203, nbubbles: int = 32,
                   max_steps: int = 0) -> int:
        """Adds a member whose initial condition is built on the device."""
        i = C.c_int()
        check(lib().cfd_batch_add_recipe(self._h, C.byref(cfg), RECIPE[name], seed, nbubbles,
                                         max_steps, C.byref(i)), "cfd_batch_add_recipe")
        self.cfgs[i.value] = cfg.copy()
        return i.value

    def save(self, mid: int, path) -> None:
        check(lib().cfd_batch_save(self._h, mid, str(path).encode()), "cfd_batch_save")

    def restore(self, path, max_steps: int = -1) -> int:
        i = C.c_int()
        check(lib().cfd_batch_restore(self._h, str(path).encode(), max_steps, C.byref(i)),
              "cfd_batch_restore")
        cfg, _, _ = checkpoint_info(path)
        self.cfgs[i.value] = cfg
        return i.value

    def try_add(self, cfg: Config, grid: np.ndarray, max_steps: int = 0) -> int | None:
        """Like add, but returns None when the member does not fit the budget."""
        i = C.c_int()
        rc = lib().cfd_batch_add(self._h, C.byref(cfg), _dp(grid), max_steps, C.byref(i))
        if rc == -6:
            return None
        check(rc, "cfd_batch_add")
        self.cfgs[i.value] = cfg.copy()
        return i.value

    def remove(self, mid: int) -> None:
        check(lib().cfd_batch_remove(self._h, mid), "cfd_batch_remove")
        self.cfgs.pop(mid, None)

    def size(self):
        n = C.c_int()
        used = C.c_size_t()
        budget = C.c_size_t()
        check(lib().cfd_batch_size(self._h, C.byref(n), C.byref(used), C.byref(budget)),
              "cfd_batch_size")
        return n.value, used.value, budget.value

    def step(self, ticks: int) -> None:
        check(lib().cfd_batch_step(self._h, ticks), "cfd_batch_step")

    def step_timed(self, ticks: int):
        mx, my, n = C.c_double(), C.c_double(), C.c_int()
        check(lib().cfd_batch_step_timed(self._h, ticks, C.byref(mx), C.byref(my), C.byref(n)),
              "cfd_batch_step_timed")
        return mx.value, my.value, n.value

    def autotune(self, steps_per_trial: int = 2) -> float:
        ms = C.c_double()
        check(lib().cfd_batch_autotune(self._h, steps_per_trial, C.byref(ms)), "cfd_batch_autotune")
        return ms.value

    def set_shapes(self, model: int, sx: int, sy: int) -> None:
        check(lib().cfd_batch_set_shapes(self._h, model, sx, sy), "cfd_batch_set_shapes")

    def get_shapes(self, model: int):
        a, b = C.c_int(), C.c_int()
        check(lib().cfd_batch_get_shapes(self._h, model, C.byref(a), C.byref(b)),
              "cfd_batch_get_shapes")
        return a.value, b.value

    def set_march_rows(self, model: int, rows: int) -> None:
        """Strip length of the marching y sweep (16..64, 0 = chosen per tile list)."""
        check(lib().cfd_batch_set_march_rows(self._h, model, rows), "cfd_batch_set_march_rows")

    def march_rows(self, model: int) -> int:
        r = C.c_int()
        check(lib().cfd_batch_get_march_rows(self._h, model, C.byref(r)), "cfd_batch_get_march_rows")
        return r.value

    def segment_rows(self, model: int, precision: int = MIXED) -> int:
        """Rows of the x sweep's warp-segment tiles in the current tile list."""
        r = C.c_int()
        check(lib().cfd_batch_get_segment_rows(self._h, model, precision, C.byref(r)),
              "cfd_batch_get_segment_rows")
        return r.value

    def status(self, mid: int) -> Status:
        st = Status()
        check(lib().cfd_batch_status(self._h, mid, C.byref(st)), "cfd_batch_status")
        return st

    def poll(self):
        n = len(self.cfgs) + 1
        ids = (C.c_int * n)()
        steps = (C.c_int * n)()
        done = (C.c_int * n)()
        t = (C.c_double * n)()
        cnt = C.c_int()
        check(lib().cfd_batch_poll(self._h, n, ids, steps, done, t, C.byref(cnt)), "cfd_batch_poll")
        return [(ids[i], steps[i], bool(done[i]), t[i]) for i in range(cnt.value)]

    def poll_issue(self) -> None:
        """Queues a status read behind the work queued so far (see poll_collect)."""
        check(lib().cfd_batch_poll_issue(self._h), "cfd_batch_poll_issue")

    def poll_collect(self):
        """Waits for the read queued by poll_issue; entries as poll()."""
        n = len(self.cfgs) + 1
        ids = (C.c_int * n)()
        steps = (C.c_int * n)()
        done = (C.c_int * n)()
        t = (C.c_double * n)()
        cnt = C.c_int()
        check(lib().cfd_batch_poll_collect(self._h, n, ids, steps, done, t, C.byref(cnt)),
              "cfd_batch_poll_collect")
        return [(ids[i], steps[i], bool(done[i]), t[i]) for i in range(min(cnt.value, n))]

    def download(self, mid: int, layout: int = GHOSTED_AOS,
                 out: np.ndarray | None = None) -> np.ndarray:
        c = self.cfgs[mid]
        if out is None:
            shape = c.ghosted_shape() if layout == GHOSTED_AOS else (c.nvar, c.ny, c.nx)
            out = np.empty(shape)
        check(lib().cfd_batch_download(self._h, mid, _dp(out), layout), "cfd_batch_download")
        return out


class Server:
    """Continuous-batching server (cfd_server_*): submit solves from any
    thread, wait for their final grids; a worker thread owns the GPU."""

    def __init__(self, precision: int = MIXED, budget_bytes: int = 0, budget_fraction: float = 0.8,
                 ticks_per_round: int = 16, stream: int | None = None, host_pinned_bytes: int = 0):
        o = ServerOptions(precision, budget_bytes, budget_fraction, ticks_per_round,
                          C.c_void_p(stream) if stream else None, host_pinned_bytes)
        h = C.c_void_p()
        check(lib().cfd_server_create(C.byref(o), C.byref(h)), "cfd_server_create")
        self._h = h
        self.cfgs: dict[int, Config] = {}

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().cfd_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def submit(self, cfg: Config, grid: np.ndarray, steps: int) -> int:
        rid = C.c_int64()
        check(lib().cfd_server_submit(self._h, C.byref(cfg), _dp(np.ascontiguousarray(grid)),
                                      steps, C.byref(rid)), "cfd_server_submit")
        self.cfgs[rid.value] = cfg.copy()
        return rid.value

    def submit_recipe(self, cfg: Config, name: str, seed: int, nbubbles: int, steps: int) -> int:
        """Queues a solve whose initial condition is built on the device."""
        rid = C.c_int64()
        check(lib().cfd_server_submit_recipe(self._h, C.byref(cfg), RECIPE[name], seed, nbubbles,
                                             steps, C.byref(rid)), "cfd_server_submit_recipe")
        self.cfgs[rid.value] = cfg.copy()
        return rid.value

    def wait(self, rid: int, timeout: float = -1.0, want_result: bool = True,
             out: np.ndarray | None = None):
        """Waits for request `rid`; returns its info and its final grid (into
        `out` when given: a C-contiguous float64 array of the ghosted shape)."""
        info = RequestInfo()
        if out is not None:
            shape = self.cfgs[rid].ghosted_shape()
            if out.shape != tuple(shape) or out.dtype != np.float64 or not out.flags.c_contiguous:
                raise ValueError(f"out must be a C-contiguous float64 array of shape {tuple(shape)}")
        elif want_result:
            out = np.empty(self.cfgs[rid].ghosted_shape())
        check(lib().cfd_server_wait(self._h, rid, timeout, C.byref(info),
                                    _dp(out) if out is not None else None), "cfd_server_wait")
        return info, out

    def release(self, rid: int) -> None:
        check(lib().cfd_server_release(self._h, rid), "cfd_server_release")
        self.cfgs.pop(rid, None)

    def stats(self) -> ServerStats:
        st = ServerStats()
        check(lib().cfd_server_get_stats(self._h, C.byref(st)), "cfd_server_get_stats")
        return st
