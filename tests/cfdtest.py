"""Helpers for the tests: golden fixtures, oracle parameter conversion."""
from __future__ import annotations

from pathlib import Path

import numpy as np

import oracle_py as O

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
# (model, reference test case, nx, ny, steps, configuration overrides) run
# against the oracle: every limiter, both splittings, Godunov, PVRS speeds,
# the alpha clip, the dy half step, walls, tiny and ragged grids
PARITY_CASES = [
    ("euler", "totem_pole_3", 30, 61, 80, {}),
    ("euler", "multiple_circles_1", 67, 35, 40, {"limiter": 1}),
    ("euler", "cross", 129, 70, 30, {"limiter": 2, "cfl": 0.8}),
    ("euler", "totem_pole_1", 33, 24, 30, {"limiter": 3}),
    ("euler", "totem_pole_3", 30, 61, 30, {"fix_dy_halfstep": 1}),
    ("euler", "circular_explosion", 26, 30, 30, {"splitting": 1}),
    ("euler", "totem_pole_2", 20, 21, 30, {"flux_solver": 1}),
    ("euler", "circular_explosion", 2, 2, 10, {}),
    ("euler", "cross", 2, 50, 20, {}),
    ("euler", "cross", 50, 3, 20, {}),
    ("allaire", "ST2_y", 10, 60, 50, {}),
    ("allaire", "TTC3_x_pure", 60, 8, 40, {"limiter": 2}),
    ("allaire", "circular_explosion", 30, 30, 20, {"limiter": 1}),
    ("allaire", "shocked_helium_bubble", 40, 20, 20, {}),
    ("allaire", "underwater_explosion_modified", 32, 32, 20, {}),
    ("allaire", "tin_air_implosion", 24, 48, 10, {}),
    ("allaire", "ST2_x", 60, 10, 40, {"wavespeed": 1, "z_min": 1e-6}),
    ("allaire", "ST1_x", 40, 6, 20, {"flux_solver": 1}),
    ("allaire", "RMI_SF6", 64, 16, 20, {"splitting": 1}),
]

# face known-answer fixtures of the reference build (make_golden.py)
KATS = ["kat_faces_euler", "kat_faces_allaire", "kat_faces_euler_low_energy",
        "kat_faces_allaire_low_energy"]


def load_golden(name: str) -> dict:
    with np.load(GOLDEN / f"{name}.npz", allow_pickle=False) as z:
        return {k: z[k] for k in z.files}


def params_from(fx: dict) -> O.RefParams:
    p = O.RefParams()
    for f, _ in p._fields_:
        v = fx["p_" + f]
        if f == "bc":
            for k in range(4):
                p.bc[k] = int(v[k])
        else:
            setattr(p, f, v.item())
    return p


def ghost_grid(interior: np.ndarray, g: int) -> np.ndarray:
    """Interior (ny, nx, nv) -> ghosted grid with zero ghost strips."""
    ny, nx, nv = interior.shape
    out = np.zeros((ny + 2 * g, nx + 2 * g, nv))
    out[g:-g, g:-g] = interior
    return out


def rel_l1(a: np.ndarray, b: np.ndarray) -> float:
    return float(np.abs(a - b).sum() / np.abs(b).sum())


def density(state: np.ndarray, model: str) -> np.ndarray:
    return state[..., 0] if model == "euler" else state[..., 0] + state[..., 1]


def config_from_params(p: O.RefParams, model: str):
    """cfd_config equivalent of an oracle parameter block."""
    import cfdgpu as G

    c = G.Config()
    c.model = G.EULER if model == "euler" else G.ALLAIRE
    c.precision = G.FP64
    c.nx, c.ny = p.nx, p.ny
    c.x0, c.y0, c.dx, c.dy = p.x0, p.y0, p.dx, p.dy
    c.gamma1, c.pinf1, c.gamma2, c.pinf2 = p.gamma1, p.pinf1, p.gamma2, p.pinf2
    for k in range(4):
        c.bc[k] = p.bc[k]
    c.cfl, c.T = p.cfl, p.T
    c.limiter, c.flux_solver, c.splitting = p.limiter, p.flux_solver, p.splitting
    c.wavespeed, c.z_min, c.fix_dy_halfstep = p.wavespeed, p.z_min, p.fix_dy_halfstep
    return c


def params_from_config(c, **over) -> O.RefParams:
    model = "euler" if c.model == 0 else "allaire"
    p = O.make_params(c.nx, c.ny, c.dx, c.dy, c.gamma1, c.pinf1, c.gamma2, c.pinf2, c.x0, c.y0,
                      tuple(c.bc), c.cfl, c.T, c.limiter, c.flux_solver, c.splitting, c.wavespeed,
                      c.z_min, c.fix_dy_halfstep)
    for k, v in over.items():
        setattr(p, k, v)
    return p, model


def masschange_close(ours: str, ref: str) -> bool:
    """Mass-change logs (E/sourcecode/euler_io.cpp:1219-1233) equal up to the
    rounding of their sums: the reference sums serially, the GPU in a tree.
    Times must be identical."""
    a = [line.split() for line in ours.splitlines() if line.strip()]
    b = [line.split() for line in ref.splitlines() if line.strip()]
    if len(a) != len(b):
        return False
    for ra, rb in zip(a, b):
        if ra[0] != rb[0] or len(ra) != len(rb):  # times are bit-identical
            return False
        for x, y in zip(map(float, ra[1:]), map(float, rb[1:])):
            if abs(x - y) > max(1e-13, 1e-5 * abs(y)):
                return False
    return True
