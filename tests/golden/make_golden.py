"""Generates the golden fixtures in tests/golden/ from the reference itself.

    python tests/golden/make_golden.py            # everything
    python tests/golden/make_golden.py outputs    # only the whole-run output files
    python tests/golden/make_golden.py adapter    # only the adapter's extra runs (golden/adapter/)
    python tests/golden/make_golden.py --out DIR  # everything, written under DIR instead

Requires oracle/_ref/libref_{euler,allaire}.so (built by `make -C oracle ref`
from the reference sources) and oracle/_build/liboracle.so (the CPU-side
builder of the seeded recipe initial conditions, which the reference does
not have).
Every fixture records the reference's own run: its set_ICs where the case is
one of its test cases, its time loop, its flux solver.
"""
from __future__ import annotations

import hashlib
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
OUT = HERE  # where fixtures are written (--out DIR: elsewhere, e.g. to compare)
sys.path.insert(0, str(ROOT / "oracle"))

import oracle_py as O  # noqa: E402


def interior(grid: np.ndarray, g: int) -> np.ndarray:
    return np.ascontiguousarray(grid[g:-g, g:-g, :])


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest()


def case_run(model, case, nx, ny, steps, **over):
    grid, p = O.ref_case_ic(model, case, nx, ny)
    ic = grid.copy()
    p.cfl = over.pop("cfl", 0.5)
    for k, v in over.items():
        if k in O.LIM and False:
            pass
        setattr(p, k, O.LIM[v] if k == "limiter" and isinstance(v, str) else v)
    taken, n, t, dts = O.ref_run(model, p, grid, steps)
    return ic, grid, p, taken, n, t, dts


def params_dict(p: O.RefParams) -> dict:
    d = {f[0]: getattr(p, f[0]) for f in p._fields_}
    d["bc"] = list(p.bc)
    return d


def save(name, model, ic, grid, p, taken, n, t, dts, store_full=True):
    g = O.ghosts_of(p)
    fin = interior(grid, g)
    out = dict(model=np.array(model), ic=interior(ic, g), rho=fin[:, :, 0] if model == "euler"
               else fin[:, :, 0] + fin[:, :, 1], n=np.array(n), t=np.array(t), dts=dts,
               taken=np.array(taken), sha256=np.array(digest(fin)))
    if store_full:
        out["state"] = fin
    for k, v in params_dict(p).items():
        out["p_" + k] = np.array(v)
    np.savez_compressed(OUT / f"{name}.npz", **out)
    print(f"{name}: {taken} steps, t={t:.6g}, sha256={digest(fin)[:16]}")


def kat_faces(model, nfaces, seed):
    """Known-answer faces: random 4-cell stencils through the reference flux."""
    rng = np.random.default_rng(seed)
    if model == "euler":
        p = O.make_params(2, 2, 1.0, 1.0, 1.4, limiter="minmod")
        W = np.stack([rng.lognormal(0, 1, (nfaces, 4)), rng.normal(0, 2, (nfaces, 4)),
                      rng.normal(0, 2, (nfaces, 4)), rng.lognormal(0, 1.5, (nfaces, 4))], -1)
        rho, u, v, pr = W[..., 0], W[..., 1], W[..., 2], W[..., 3]
        e = pr / (0.4 * rho)
        U = np.stack([rho, rho * u, rho * v, rho * e + 0.5 * rho * (u * u + v * v)], -1)
    else:
        p = O.make_params(2, 2, 1.0, 1.0, 4.4, 6e8, 1.4, 0.0, limiter="minmod")
        z = rng.uniform(0, 1, (nfaces, 4))
        z[rng.uniform(size=z.shape) < 0.2] = 1.0
        z[rng.uniform(size=z.shape) < 0.2] = 0.0
        r1 = rng.uniform(900, 1100, (nfaces, 4))
        r2 = rng.uniform(0.5, 2, (nfaces, 4))
        u = rng.normal(0, 50, (nfaces, 4))
        v = rng.normal(0, 50, (nfaces, 4))
        pr = rng.lognormal(np.log(1e6), 2, (nfaces, 4))
        eps = z / 3.4 + (1 - z) / 0.4
        k = (z * 4.4 * 6e8 / 3.4) / eps
        rho = z * r1 + (1 - z) * r2
        e = (pr + k) * eps / rho
        U = np.stack([z * r1, (1 - z) * r2, rho * u, rho * v, rho * e + 0.5 * rho * (u * u + v * v), z], -1)
    dt, dx = 1e-3 if model == "euler" else 1e-7, 1e-2
    F = np.zeros((nfaces, U.shape[-1]))
    us = np.zeros(nfaces)
    zs = np.zeros(nfaces)
    for f in range(nfaces):
        fl, a, b = O.ref_face_flux(model, p, U[f], dt, dx)
        F[f] = fl
        us[f] = a
        zs[f] = b if b is not None else 0.0
    np.savez_compressed(OUT / f"kat_faces_{model}.npz", stencils=U, flux=F, u_star=us,
                        z_star=zs, dt=np.array(dt), dx=np.array(dx),
                        **{"p_" + k: np.array(v) for k, v in params_dict(p).items()})
    print(f"kat_faces_{model}: {nfaces} faces")


def kat_faces_low_energy(model, nfaces, seed):
    """Adversarial known-answer faces for the physicality tests of MUSCL-
    Hancock (E/headers/flux_solver_MUSCLhancock.hpp:178-189, 212-223): cells
    whose specific internal energy is a tiny fraction r of their kinetic
    energy (r log-uniform in [1e-15, 1e-10], i.e. on both sides of the
    1e-13 relative margin below which the device defers to the reference's
    exact recomputation), with fast flow, so that the extrapolated and
    evolved face states sit at e ~ 0 and the reference's zero-slope and
    first-order fallbacks fire on some faces and not on others.  Stencils
    whose cells fail the reference's own input assert, or whose flux is not
    finite, are dropped."""
    rng = np.random.default_rng(seed)
    n = 4 * nfaces
    r = 10.0 ** rng.uniform(-15, -10, (n, 4))
    if model == "euler":
        p = O.make_params(2, 2, 1.0, 1.0, 1.4, limiter="minmod")
        rho = rng.lognormal(0, 1, (n, 4))
        u = rng.normal(0, 20, (n, 4))
        v = rng.normal(0, 20, (n, 4))
        ke = 0.5 * (u * u + v * v)
        e = r * ke
        U = np.stack([rho, rho * u, rho * v, rho * e + rho * ke], -1)
        ru = U[..., 0]
        e_chk = U[..., 3] / ru - 0.5 * ((U[..., 1] / ru) ** 2 + (U[..., 2] / ru) ** 2)
    else:
        # air only (z = 0): with any stiffened-gas share a state this close
        # to e = 0 has a negative squared sound speed (p -> -k), and its flux
        # is NaN in the reference
        p = O.make_params(2, 2, 1.0, 1.0, 4.4, 6e8, 1.4, 0.0, limiter="minmod")
        z = np.zeros((n, 4))
        r1 = rng.uniform(900, 1100, (n, 4))
        r2 = rng.uniform(0.5, 2, (n, 4))
        u = rng.normal(0, 300, (n, 4))
        v = rng.normal(0, 300, (n, 4))
        ke = 0.5 * (u * u + v * v)
        rho = z * r1 + (1 - z) * r2
        e = r * ke
        U = np.stack([z * r1, (1 - z) * r2, rho * u, rho * v, rho * e + rho * ke, z], -1)
        ru = U[..., 0] + U[..., 1]
        e_chk = U[..., 4] / ru - 0.5 * ((U[..., 2] / ru) ** 2 + (U[..., 3] / ru) ** 2)
    U = U[(e_chk >= 0.0).all(axis=1)]
    dt, dx = (1e-3, 1e-2) if model == "euler" else (1e-6, 1e-2)
    rows = []
    for f in range(len(U)):
        fl, a, b = O.ref_face_flux(model, p, U[f], dt, dx)
        if np.isfinite(fl).all() and np.isfinite(a):  # known answers, not NaN
            rows.append((U[f], fl, a, b if b is not None else 0.0))
        if len(rows) == nfaces:
            break
    U = np.ascontiguousarray(np.stack([r[0] for r in rows]))
    F = np.stack([r[1] for r in rows])
    us = np.array([r[2] for r in rows])
    zs = np.array([r[3] for r in rows])
    np.savez_compressed(OUT / f"kat_faces_{model}_low_energy.npz", stencils=U, flux=F,
                        u_star=us, z_star=zs, dt=np.array(dt), dx=np.array(dx),
                        **{"p_" + k: np.array(v) for k, v in params_dict(p).items()})
    print(f"kat_faces_{model}_low_energy: {len(U)} faces")


def main():
    assert O.ref_available("euler") and O.ref_available("allaire"), "build oracle/_ref first"
    # reference test cases through the reference's own set_ICs and time loop
    save("euler_totem_pole_3_30x61", "euler", *case_run("euler", "totem_pole_3", 30, 61, 100000))
    save("euler_cross_48x40_vanleer", "euler",
         *case_run("euler", "cross", 48, 40, 60, limiter="vanleer", cfl=0.8))
    save("euler_circular_explosion_40x36_strang", "euler",
         *case_run("euler", "circular_explosion", 40, 36, 40, splitting=1))
    save("allaire_ST2_x_100x10", "allaire", *case_run("allaire", "ST2_x", 100, 10, 100000))
    save("allaire_ST1_y_12x80_mc", "allaire",
         *case_run("allaire", "ST1_y", 12, 80, 60, limiter="mc"))

    # four-quadrant Riemann problem, 200x200 to t = 0.3 (van Leer, CFL 0.8):
    # the recipe IC is built by the CPU-side recipe builder
    # (oracle/oracle_recipes.c, bit-identical to the library's host hook),
    # stepped by the reference
    ic, pr, _ = O.port_recipe_ic("four_quadrant", 200, 200)
    p = O.make_params(200, 200, pr.dx, pr.dy, 1.4, limiter="vanleer", cfl=0.8, T=0.3)
    grid = ic.copy()
    taken, n, t, dts = O.ref_run("euler", p, grid, 100000)
    save("euler_four_quadrant_200x200", "euler", ic, grid, p, taken, n, t, dts, store_full=False)

    # water shock on an air bubble (PVRS wave speeds, z clipped to [1e-6, 1-1e-6])
    ic, pr, _ = O.port_recipe_ic("water_shock_air_bubble", 64, 32)
    p = O.make_params(64, 32, pr.dx, pr.dy, 4.4, 6e8, 1.4, 0.0, cfl=0.6, wavespeed="pvrs",
                      z_min=1e-6)
    grid = ic.copy()
    taken, n, t, dts = O.ref_run("allaire", p, grid, 40)
    save("allaire_water_shock_64x32_pvrs", "allaire", ic, grid, p, taken, n, t, dts)

    kat_faces("euler", 256, 1)
    kat_faces("allaire", 256, 2)
    kat_faces_low_energy("euler", 1024, 3)
    kat_faces_low_energy("allaire", 1024, 4)

    # long horizons at the benchmarked configurations' step counts on reduced
    # grids: shock + bubbles (Euler, 2000 steps at CFL 0.8) and the water
    # shock on an air bubble (Allaire, PVRS speeds, alpha clip, 1500 steps at
    # CFL 0.6), from the CPU-side recipe builder (oracle/oracle_recipes.c)
    for recipe, model, nx, ny, nb, steps in (("shock_bubbles", "euler", 64, 64, 8, 2000),
                                             ("water_shock_air_bubble", "allaire", 64, 32, 1,
                                              1500)):
        ic, p, _ = O.port_recipe_ic(recipe, nx, ny, 20261203, nb)
        grid = ic.copy()
        taken, n, t, dts = O.ref_run(model, p, grid, steps)
        save(f"{model}_{recipe}_{nx}x{ny}_{steps}steps", model, ic, grid, p, taken, n, t, dts)

    for name, model, settings in OUTPUT_RUNS:
        output_run(name, model, settings)


# Whole runs of the reference's main() on a settings file: every output file
# it writes (states, schlieren frames, lineouts, mass change), byte for byte.
OUTPUT_RUNS = [
    ("outputs_euler_cross_20x16", "euler",
     "Nx 20\nNy 16\nCFL 0.5\nsplitting_scheme naive_splitting\ntest_case cross\n"
     "output_freq 3\noutputpath {out}\nflux_solver MUSCL\nriemann_solver HLLC\nproblem euler\n"),
    ("outputs_allaire_shocked_helium_bubble_26x8", "allaire",
     "Nx 26\nNy 8\nCFL 0.5\nsplitting_scheme strang_splitting\n"
     "test_case shocked_helium_bubble\noutput_freq 2\noutputpath {out}\nflux_solver MUSCL\n"
     "riemann_solver HLLC\nproblem allaire\n"),
]


# More whole runs, for the reference-loop adapter's CPU check only (kept in
# golden/adapter/ so that the GPU driver test does not collect them): the
# Godunov scheme (one ghost layer) for both models, Strang splitting for
# Euler, naive splitting for Allaire.
ADAPTER_RUNS = [
    ("godunov_totem_pole_2_20x20", "euler",
     "Nx 20\nNy 20\nCFL 0.5\nsplitting_scheme naive_splitting\ntest_case totem_pole_2\n"
     "output_freq 2\noutputpath {out}\nflux_solver Godunov\nriemann_solver HLLC\nproblem euler\n"),
    ("strang_circular_explosion_24x20", "euler",
     "Nx 24\nNy 20\nCFL 0.5\nsplitting_scheme strang_splitting\ntest_case circular_explosion\n"
     "output_freq 2\noutputpath {out}\nflux_solver MUSCL\nriemann_solver HLLC\nproblem euler\n"),
    ("naive_ST2_x_40x6", "allaire",
     "Nx 40\nNy 6\nCFL 0.5\nsplitting_scheme naive_splitting\ntest_case ST2_x\n"
     "output_freq 2\noutputpath {out}\nflux_solver MUSCL\nriemann_solver HLLC\nproblem allaire\n"),
    ("godunov_ST1_x_30x6", "allaire",
     "Nx 30\nNy 6\nCFL 0.5\nsplitting_scheme strang_splitting\ntest_case ST1_x\n"
     "output_freq 2\noutputpath {out}\nflux_solver Godunov\nriemann_solver HLLC\nproblem allaire\n"),
]


def output_run(name: str, model: str, settings: str, dest: Path | None = None) -> None:
    dest = OUT if dest is None else dest
    import os
    import subprocess
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "out") + "/"
        os.makedirs(out)
        sf = os.path.join(d, "settingsfile.txt")
        with open(sf, "w") as f:
            f.write(settings.format(out=out))
        code = (f"import sys; sys.path.insert(0, {str(ROOT / 'oracle')!r}); import oracle_py as O; "
                f"sys.exit(O.ref_simulate({model!r}, {sf!r}))")
        subprocess.run([sys.executable, "-c", code], check=True, stdout=subprocess.DEVNULL,
                       env={**os.environ, "OMP_NUM_THREADS": "1"})
        files = {fn: np.frombuffer(open(os.path.join(out, fn), "rb").read(), np.uint8)
                 for fn in sorted(os.listdir(out))}
    dest.mkdir(exist_ok=True)
    np.savez_compressed(dest / f"{name}.npz", settings=np.array(settings), **files)
    print(f"{name}: {len(files)} files")


if __name__ == "__main__":
    args = sys.argv[1:]
    if args[:1] == ["--out"]:
        OUT = Path(args[1]).resolve()
        OUT.mkdir(parents=True, exist_ok=True)
        args = args[2:]
    if args == ["outputs"]:
        for run in OUTPUT_RUNS:
            output_run(*run)
    elif args == ["adapter"]:
        for run in ADAPTER_RUNS:
            output_run(*run, dest=OUT / "adapter")
    else:
        main()
        for run in ADAPTER_RUNS:
            output_run(*run, dest=OUT / "adapter")
