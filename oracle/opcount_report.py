"""Exact FP64 operation counts of the reference's update, per face and per
cell-update.  MEASUREMENT INFRASTRUCTURE ONLY (reads the counted CPU
restatement, oracle/_build/libopcount.so; never the shipped library).

    python oracle/opcount_report.py            # markdown tables on stdout

Counts follow the reference's expression trees (cfd_oracle.c restates them
operation by operation): every add/sub, mul, div and sqrt executed, plus the
comparisons and fabs/copysign, on

* one face of MUSCL-Hancock + HLLC on smooth stencils (no fallback taken;
  E/headers/flux_solver_MUSCLhancock.hpp:128-227,
  A/headers/flux_solver_MUSCLhancock.hpp:272-376);
* whole steps of the two bench workloads' recipes (Mach-2 shock over 32
  bubbles; water shock on an air bubble), where the limiter branches,
  fallbacks and fix-ups taken depend on the flow, so the averages belong to
  the stated grid and step count.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path[:0] = [str(HERE), str(HERE.parent / "cfd-art_b200")]

import oracle_py as O  # noqa: E402

FLOPS = ("add", "mul", "div", "sqrt")
SEED = 20261203


def smooth_stencil(model: str) -> np.ndarray:
    """Four cells of a smooth, subsonic flow in +x: every slope limited by
    the smooth branch, both half-step states physical."""
    rows = []
    for k in range(4):
        rho, u, v, p = 1.0 + 0.01 * k, 0.3 + 0.002 * k, 0.1, 1.0 + 0.02 * k
        if model == "euler":
            e = p / (0.4 * rho)
            rows.append([rho, rho * u, rho * v, rho * e + 0.5 * rho * (u * u + v * v)])
        else:
            z = 0.5 + 0.01 * k
            a1, a2 = z * 1000.0 * rho, (1.0 - z) * rho
            r = a1 + a2
            eps = z / 3.4 + (1.0 - z) / 0.4
            kk = (z * 4.4 * 6e8 / 3.4) / eps
            e = (p * 1e5 + kk) * eps / r
            rows.append([a1, a2, r * u, r * v, r * e + 0.5 * r * (u * u + v * v), z])
    return np.array(rows, dtype=np.float64)


def face_counts(model: str) -> dict[str, int]:
    if model == "euler":
        p = O.make_params(8, 8, 1e-2, 1e-2, 1.4, limiter="vanleer")
    else:
        p = O.make_params(8, 8, 1e-2, 1e-2, 4.4, 6e8, 1.4, 0.0, limiter="vanleer",
                          wavespeed="pvrs", z_min=1e-6)
    st = smooth_stencil(model)
    flux, us, zs, c = O.opcount_face(model, p, st, 1e-5, 1e-2)
    f2, us2, zs2 = O.port_face_flux(model, p, st, 1e-5, 1e-2)
    if not (np.array_equal(flux, f2) and us == us2 and zs == zs2):
        raise AssertionError("counted face differs from the plain restatement")
    return c


def jacobian_structural_ops(nv: int, nonzeros: int) -> int:
    """Operations of the dense half-step product (s*A[i][j])*d[j], summed
    over j, done on the Jacobian's structural zeros, for both face states."""
    dense = nv * nv * 2 + nv * (nv - 1)
    sparse = nonzeros * 2 + (nonzeros - nv)
    return 2 * (dense - sparse)


def workload_counts(recipe: str, nx: int, ny: int, nbub: int, steps: int):
    import cfdgpu as G

    model = "euler" if recipe == "shock_bubbles" else "allaire"
    cfg = G.recipe_config(recipe, nx, ny)
    ic = G.recipe_ic(cfg, recipe, seed=SEED, nbubbles=nbub)
    p = O.make_params(nx, ny, cfg.dx, cfg.dy, cfg.gamma1, cfg.pinf1, cfg.gamma2, cfg.pinf2,
                      bc=tuple(cfg.bc), cfl=cfg.cfl, T=cfg.T, limiter=cfg.limiter,
                      wavespeed=cfg.wavespeed, z_min=cfg.z_min)
    taken, _, _, c = O.opcount_run(model, p, ic, steps)
    cu = nx * ny * taken
    return model, taken, cu, c


def fmt(d: dict[str, float]) -> str:
    return " | ".join(f"{d[k]:.2f}" if isinstance(d[k], float) else str(d[k])
                      for k in O.OP_CATEGORIES)


def main() -> None:
    hdr = "| " + " | ".join(O.OP_CATEGORIES) + " | FP64 arithmetic (add+mul+div+sqrt) |"
    sep = "|" + "---|" * (len(O.OP_CATEGORIES) + 2)
    print("## One face, smooth stencil (MUSCL-Hancock, van Leer, HLLC)\n")
    print("| model " + hdr)
    print(sep)
    for model in ("euler", "allaire"):
        c = face_counts(model)
        print(f"| {model} | {fmt(c)} | {sum(c[k] for k in FLOPS)} |")
    print()
    print(f"Of these, the dense primitive-Jacobian product (`(s*A[i][j])*d[j]` over all j, "
          f"for both face states) spends {jacobian_structural_ops(4, 7)} (Euler) and "
          f"{jacobian_structural_ops(6, 10)} (Allaire) operations on the matrix's structural "
          f"zeros.\n")
    print("## Per cell-update on the bench workloads' recipes\n")
    print("| workload | phase | " + " | ".join(O.OP_CATEGORIES) + " | FP64 arithmetic |")
    print("|---|---|" + "---|" * (len(O.OP_CATEGORIES) + 1))
    for recipe, nx, ny, nb, steps in (("shock_bubbles", 512, 512, 32, 20),
                                      ("water_shock_air_bubble", 512, 256, 1, 20)):
        model, taken, cu, c = workload_counts(recipe, nx, ny, nb, steps)
        name = f"{recipe} {nx}x{ny}, {taken} steps"
        tot = {k: 0.0 for k in O.OP_CATEGORIES}
        for ph in ("dt", "step"):
            per = {k: c[ph][k] / cu for k in O.OP_CATEGORIES}
            for k in per:
                tot[k] += per[k]
            print(f"| {name} | {ph} | {fmt(per)} | {sum(per[k] for k in FLOPS):.2f} |")
        print(f"| {name} | total | {fmt(tot)} | {sum(tot[k] for k in FLOPS):.2f} |")


if __name__ == "__main__":
    main()
