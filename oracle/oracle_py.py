"""ctypes bindings for the CPU oracles.  TEST INFRASTRUCTURE ONLY.

Two oracles live under ``oracle/``:

* ``_ref/libref_euler.so`` / ``_ref/libref_allaire.so``: the reference's own
  C++ sources (euler_equations/euler_simulation_code, allaire_2d) compiled
  against the Eigen-subset shim plus the hook drivers ``ref_*_hook.cpp``.
* ``_build/liboracle.so``: the plain-C restatement ``cfd_oracle.c``.
* ``_build/libopcount.so``: the same restatement compiled with a counting
  double (``opcount.cpp``), for exact operation counts per cell-update.

Only the tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline /
reference arm import this module.  The shipped library never does.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_DIR = HERE / "_ref"
PORT_DIR = HERE / "_build"

LIM = {"minmod": 0, "vanleer": 1, "mc": 2, "unlimited": 3}
FLUX = {"MUSCL": 0, "Godunov": 1}
SPLIT = {"naive": 0, "strang": 1}
WS = {"davis": 0, "pvrs": 1}


class RefParams(C.Structure):
    """Mirror of ``ref_params`` in oracle/ref_common.h."""

    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int),
        ("x0", C.c_double), ("y0", C.c_double), ("dx", C.c_double), ("dy", C.c_double),
        ("gamma1", C.c_double), ("pinf1", C.c_double),
        ("gamma2", C.c_double), ("pinf2", C.c_double),
        ("bc", C.c_int * 4),
        ("cfl", C.c_double), ("T", C.c_double),
        ("limiter", C.c_int), ("flux_solver", C.c_int), ("splitting", C.c_int),
        ("wavespeed", C.c_int), ("z_min", C.c_double), ("fix_dy_halfstep", C.c_int),
    ]


def make_params(nx, ny, dx, dy, gamma1, pinf1=0.0, gamma2=1.4, pinf2=0.0, x0=0.0, y0=0.0,
                bc=(0, 0, 0, 0), cfl=0.8, T=float("inf"), limiter="minmod", flux_solver="MUSCL",
                splitting="naive", wavespeed="davis", z_min=0.0, fix_dy_halfstep=0) -> RefParams:
    p = RefParams()
    p.nx, p.ny = int(nx), int(ny)
    p.x0, p.y0, p.dx, p.dy = float(x0), float(y0), float(dx), float(dy)
    p.gamma1, p.pinf1, p.gamma2, p.pinf2 = float(gamma1), float(pinf1), float(gamma2), float(pinf2)
    for k in range(4):
        p.bc[k] = int(bc[k])
    p.cfl, p.T = float(cfl), float(T)
    p.limiter = LIM[limiter] if isinstance(limiter, str) else int(limiter)
    p.flux_solver = FLUX[flux_solver] if isinstance(flux_solver, str) else int(flux_solver)
    p.splitting = SPLIT[splitting] if isinstance(splitting, str) else int(splitting)
    p.wavespeed = WS[wavespeed] if isinstance(wavespeed, str) else int(wavespeed)
    p.z_min = float(z_min)
    p.fix_dy_halfstep = int(fix_dy_halfstep)
    return p


def _dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


_libs: dict[str, C.CDLL] = {}


def _load(name: str, path: Path) -> C.CDLL:
    if name not in _libs:
        if not path.exists():
            raise FileNotFoundError(f"{path} is not built (run `make -C oracle`)")
        _libs[name] = C.CDLL(str(path))
    return _libs[name]


def ref_available(model: str = "euler") -> bool:
    return (REF_DIR / f"libref_{model}.so").exists()


def port_available() -> bool:
    return (PORT_DIR / "liboracle.so").exists()


def ref_lib(model: str) -> C.CDLL:
    lib = _load("ref_" + model, REF_DIR / f"libref_{model}.so")
    pre = f"ref_{model}_"
    getattr(lib, pre + "run").restype = C.c_int
    getattr(lib, pre + "run").argtypes = [C.POINTER(RefParams), C.POINTER(C.c_double),
                                          C.POINTER(C.c_double), C.c_int, C.POINTER(C.c_int),
                                          C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int]
    getattr(lib, pre + "compute_dt").restype = C.c_double
    getattr(lib, pre + "compute_dt").argtypes = [C.POINTER(RefParams), C.POINTER(C.c_double),
                                                 C.c_int, C.c_double]
    getattr(lib, pre + "case_ic").restype = C.c_int
    getattr(lib, pre + "case_ic").argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_char_p,
                                              C.POINTER(C.c_double), C.POINTER(RefParams)]
    getattr(lib, pre + "write").restype = C.c_int
    getattr(lib, pre + "write").argtypes = [C.POINTER(RefParams), C.POINTER(C.c_double),
                                            C.c_char_p, C.c_int, C.c_double]
    return lib


def nvar_of(model: str) -> int:
    return 4 if model == "euler" else 6


def ghosts_of(p: RefParams) -> int:
    return 1 if p.flux_solver == FLUX["Godunov"] else 2


def ref_case_ic(model: str, test_case: str, nx: int, ny: int, flux_solver: str = "MUSCL"):
    """Reference set_ICs for a named test case -> (ghosted AoS grid, RefParams)."""
    lib = ref_lib(model)
    g = 1 if flux_solver == "Godunov" else 2
    grid = np.zeros((ny + 2 * g, nx + 2 * g, nvar_of(model)))
    p = make_params(nx, ny, 1.0, 1.0, 1.4)
    getattr(lib, f"ref_{model}_case_ic")(test_case.encode(), nx, ny, flux_solver.encode(),
                                         _dptr(grid), C.byref(p))
    return grid, p


def ref_run(model: str, p: RefParams, grid: np.ndarray, max_steps: int, n: int = 0, t: float = 0.0,
            future: np.ndarray | None = None, threads: int = 1):
    """Run the reference time loop on a ghosted grid (modified in place).

    Returns (steps_taken, n, t, dt_log)."""
    lib = ref_lib(model)
    dt_log = np.zeros(max(max_steps, 1))
    nn = C.c_int(n)
    tt = C.c_double(t)
    taken = getattr(lib, f"ref_{model}_run")(C.byref(p), _dptr(grid),
                                             _dptr(future) if future is not None else None,
                                             int(max_steps), C.byref(nn), C.byref(tt),
                                             _dptr(dt_log), int(threads))
    return taken, nn.value, tt.value, dt_log[:taken]


def ref_compute_dt(model: str, p: RefParams, grid: np.ndarray, n: int, t: float) -> float:
    lib = ref_lib(model)
    return getattr(lib, f"ref_{model}_compute_dt")(C.byref(p), _dptr(grid), int(n), float(t))


def ref_face_flux(model: str, p: RefParams, stencil: np.ndarray, dt: float, dx: float):
    lib = ref_lib(model)
    nv = nvar_of(model)
    flux = np.zeros(nv)
    us = C.c_double()
    st = np.ascontiguousarray(stencil, dtype=np.float64)
    if model == "euler":
        lib.ref_euler_face_flux.argtypes = [C.POINTER(RefParams), C.POINTER(C.c_double), C.c_double,
                                            C.c_double, C.POINTER(C.c_double),
                                            C.POINTER(C.c_double)]
        lib.ref_euler_face_flux(C.byref(p), _dptr(st), dt, dx, _dptr(flux), C.byref(us))
        return flux, us.value, None
    zs = C.c_double()
    lib.ref_allaire_face_flux.argtypes = [C.POINTER(RefParams), C.POINTER(C.c_double), C.c_double,
                                          C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                          C.POINTER(C.c_double)]
    lib.ref_allaire_face_flux(C.byref(p), _dptr(st), dt, dx, _dptr(flux), C.byref(us), C.byref(zs))
    return flux, us.value, zs.value


def ref_write(model: str, p: RefParams, grid: np.ndarray, basename: str, n: int, t: float):
    lib = ref_lib(model)
    getattr(lib, f"ref_{model}_write")(C.byref(p), _dptr(grid), basename.encode(), int(n), float(t))


def ref_simulate(model: str, settings_path: str) -> int:
    """The reference's main() on a settings file: runs simulation::run_simulation
    and writes its output files.  Its output cadence keeps static state, so call
    it once per process."""
    lib = ref_lib(model)
    f = getattr(lib, f"ref_{model}_simulate")
    f.argtypes = [C.c_char_p]
    f.restype = C.c_int
    return f(str(settings_path).encode())


# --------------------------------------------------------------------------
# plain-C restatement (cfd_oracle.c)

def port_lib() -> C.CDLL:
    lib = _load("port", PORT_DIR / "liboracle.so")
    lib.oracle_run.restype = C.c_int
    lib.oracle_run.argtypes = [C.c_int, C.POINTER(RefParams), C.POINTER(C.c_double),
                               C.POINTER(C.c_double), C.c_int, C.POINTER(C.c_int),
                               C.POINTER(C.c_double), C.POINTER(C.c_double)]
    lib.oracle_face_flux.restype = None
    lib.oracle_face_flux.argtypes = [C.c_int, C.POINTER(RefParams), C.POINTER(C.c_double),
                                     C.c_double, C.c_double, C.POINTER(C.c_double),
                                     C.POINTER(C.c_double), C.POINTER(C.c_double)]
    lib.oracle_recipe_ic.restype = C.c_int
    lib.oracle_recipe_ic.argtypes = [C.c_int, C.c_int, C.c_int, C.c_ulonglong, C.c_int,
                                     C.POINTER(C.c_double), C.POINTER(RefParams)]
    lib.oracle_compute_dt.restype = C.c_double
    lib.oracle_compute_dt.argtypes = [C.c_int, C.POINTER(RefParams), C.POINTER(C.c_double),
                                      C.c_int, C.c_double, C.POINTER(C.c_double)]
    return lib


MODEL_ID = {"euler": 0, "allaire": 1}


def port_run(model: str, p: RefParams, grid: np.ndarray, max_steps: int, n: int = 0,
             t: float = 0.0, future: np.ndarray | None = None):
    lib = port_lib()
    dt_log = np.zeros(max(max_steps, 1))
    nn = C.c_int(n)
    tt = C.c_double(t)
    taken = lib.oracle_run(MODEL_ID[model], C.byref(p), _dptr(grid),
                           _dptr(future) if future is not None else None, int(max_steps),
                           C.byref(nn), C.byref(tt), _dptr(dt_log))
    return taken, nn.value, tt.value, dt_log[:taken]


RECIPE = {"four_quadrant": 0, "shock_bubbles": 1, "water_shock_air_bubble": 2}


def port_recipe_ic(recipe: str, nx: int, ny: int, seed: int = 20261203, nbubbles: int = 32):
    """Seeded workload recipe built on the CPU side (oracle_recipes.c):
    (ghosted AoS grid, RefParams, model name).  Equal bit for bit to the
    library's host builder; the reference arm of bench.py uses it so that the
    reference's loop runs without the library loaded."""
    model = "allaire" if recipe == "water_shock_air_bubble" else "euler"
    grid = np.zeros((ny + 4, nx + 4, nvar_of(model)))
    p = RefParams()
    r = port_lib().oracle_recipe_ic(RECIPE[recipe], int(nx), int(ny), int(seed), int(nbubbles),
                                    _dptr(grid), C.byref(p))
    if r:
        raise ValueError(f"unknown recipe {recipe}")
    return grid, p, model


def port_face_flux(model: str, p: RefParams, stencil: np.ndarray, dt: float, dx: float):
    lib = port_lib()
    nv = nvar_of(model)
    flux = np.zeros(nv)
    us = C.c_double()
    zs = C.c_double()
    st = np.ascontiguousarray(stencil, dtype=np.float64)
    lib.oracle_face_flux(MODEL_ID[model], C.byref(p), _dptr(st), dt, dx, _dptr(flux), C.byref(us),
                         C.byref(zs))
    return flux, us.value, (zs.value if model == "allaire" else None)


def port_compute_dt(model: str, p: RefParams, grid: np.ndarray, n: int, t: float):
    lib = port_lib()
    mass = np.zeros(2)
    dt = lib.oracle_compute_dt(MODEL_ID[model], C.byref(p), _dptr(grid), int(n), float(t),
                               _dptr(mass))
    return dt, mass


# --------------------------------------------------------------------------
# counted restatement (opcount.cpp)

OP_CATEGORIES = ("add", "mul", "div", "sqrt", "cmp", "sign")
OP_PHASES = ("dt", "step", "other")


def opcount_lib() -> C.CDLL:
    lib = _load("opcount", PORT_DIR / "libopcount.so")
    u64p = C.POINTER(C.c_uint64)
    lib.opcount_run.restype = C.c_int
    lib.opcount_run.argtypes = [C.c_int, C.POINTER(RefParams), C.POINTER(C.c_double), C.c_int,
                                C.POINTER(C.c_int), C.POINTER(C.c_double), u64p]
    lib.opcount_face.restype = None
    lib.opcount_face.argtypes = [C.c_int, C.POINTER(RefParams), C.POINTER(C.c_double),
                                 C.c_double, C.c_double, C.POINTER(C.c_double),
                                 C.POINTER(C.c_double), C.POINTER(C.c_double), u64p]
    nc, nph = C.c_int(), C.c_int()
    lib.opcount_layout(C.byref(nc), C.byref(nph))
    if (nc.value, nph.value) != (len(OP_CATEGORIES), len(OP_PHASES)):
        raise RuntimeError("libopcount.so count layout differs from oracle_py")
    return lib


def _counts_dict(raw: np.ndarray) -> dict[str, dict[str, int]]:
    m = raw.reshape(len(OP_PHASES), len(OP_CATEGORIES))
    return {ph: {c: int(m[i, j]) for j, c in enumerate(OP_CATEGORIES)}
            for i, ph in enumerate(OP_PHASES)}


def opcount_run(model: str, p: RefParams, grid: np.ndarray, max_steps: int, n: int = 0,
                t: float = 0.0):
    """Counted time loop (same states as port_run, grid advanced in place).

    Returns (steps_taken, n, t, counts) with counts[phase][category] totals
    over the run; phases "dt" (compute_dt) and "step" (the split update)."""
    lib = opcount_lib()
    raw = np.zeros(len(OP_PHASES) * len(OP_CATEGORIES), dtype=np.uint64)
    nn = C.c_int(n)
    tt = C.c_double(t)
    taken = lib.opcount_run(MODEL_ID[model], C.byref(p), _dptr(grid), int(max_steps),
                            C.byref(nn), C.byref(tt), raw.ctypes.data_as(C.POINTER(C.c_uint64)))
    if taken < 0:
        raise MemoryError("opcount_run could not allocate its grids")
    return taken, nn.value, tt.value, _counts_dict(raw)


def opcount_face(model: str, p: RefParams, stencil: np.ndarray, dt: float, dx: float):
    """Counted single face: (flux, u_star, z_star, counts["step"])."""
    lib = opcount_lib()
    nv = nvar_of(model)
    flux = np.zeros(nv)
    us = C.c_double()
    zs = C.c_double()
    raw = np.zeros(len(OP_PHASES) * len(OP_CATEGORIES), dtype=np.uint64)
    st = np.ascontiguousarray(stencil, dtype=np.float64)
    lib.opcount_face(MODEL_ID[model], C.byref(p), _dptr(st), dt, dx, _dptr(flux), C.byref(us),
                     C.byref(zs), raw.ctypes.data_as(C.POINTER(C.c_uint64)))
    return flux, us.value, (zs.value if model == "allaire" else None), _counts_dict(raw)["step"]


def reference_dir() -> Path:
    """The reference checkout: $CFD_REFERENCE_DIR, else a `reference`
    directory beside the repository."""
    env = os.environ.get("CFD_REFERENCE_DIR")
    return Path(env) if env else HERE.parent.parent / "reference"


def build(quiet: bool = True, ref: bool | None = None) -> None:
    """Build the oracles with oracle/Makefile (the reference part, and the
    reference's main loop linked with the GPU adapter, only where the
    reference sources are present)."""
    import subprocess

    targets = ["port", "opcount"]
    ref_src = reference_dir()
    if ref is None:
        ref = ref_src.exists()
    if ref:
        targets.append("ref")
        if (HERE.parent / "cfd-art_b200" / "lib" / "libcfdgpu.so").exists():
            targets.append("adapter")  # the reference's main loop on the GPU adapter
    subprocess.run(["make", "-C", str(HERE), f"REF={ref_src}", "-j8", *targets], check=True,
                   stdout=subprocess.DEVNULL if quiet else None)
