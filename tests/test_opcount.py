"""The operation-counting build of the CPU restatement (oracle/opcount.cpp).

Its counts are the FP64 work per face and per cell-update of the reference's
expression trees.  They only mean something if the counted build does the
same arithmetic as the plain one, so it must reproduce the golden fixtures
(runs of the reference's own build) and the reference face KATs bit for bit;
the per-face and compute_dt figures are then pinned.
"""
import numpy as np
import pytest

import oracle_py as O
from cfdtest import GOLDEN, KATS, ghost_grid, load_golden, params_from

pytestmark = pytest.mark.skipif(not (O.PORT_DIR / "libopcount.so").exists(),
                                reason="oracle/_build/libopcount.so not built")

FIXTURES = sorted(p.stem for p in GOLDEN.glob("*.npz") if not p.stem.startswith(("kat_", "outputs_")))


@pytest.mark.parametrize("name", FIXTURES)
def test_counted_run_reproduces_golden_run(name):
    fx = load_golden(name)
    model = str(fx["model"])
    p = params_from(fx)
    g = O.ghosts_of(p)
    grid = ghost_grid(fx["ic"], g)
    taken, n, t, counts = O.opcount_run(model, p, grid, int(fx["taken"]))
    assert taken == int(fx["taken"]) and n == int(fx["n"]) and t == float(fx["t"])
    fin = grid[g:-g, g:-g]
    rho = fin[..., 0] if model == "euler" else fin[..., 0] + fin[..., 1]
    assert np.array_equal(rho, fx["rho"])
    if "state" in fx:
        assert np.array_equal(fin, fx["state"])
    assert counts["step"]["div"] > 0 and counts["dt"]["sqrt"] == p.nx * p.ny * taken


@pytest.mark.parametrize("name", KATS)
def test_counted_faces_reproduce_reference_kats(name):
    model = name.split("_")[2]
    fx = load_golden(name)
    p = params_from(fx)
    dt, dx = float(fx["dt"]), float(fx["dx"])
    for f in range(fx["stencils"].shape[0]):
        flux, us, zs, c = O.opcount_face(model, p, fx["stencils"][f], dt, dx)
        assert np.array_equal(flux, fx["flux"][f]), f
        assert us == fx["u_star"][f]
        if model == "allaire":
            assert zs == fx["z_star"][f]
        assert c["sqrt"] >= 2  # HLLC's two sound speeds at least


# Pinned per-face figures (MUSCL-Hancock + van Leer + HLLC, smooth stencil,
# no fallback); oracle/opcount_report.py prints the same table.
FACE = {
    "euler": {"add": 178, "mul": 257, "div": 60, "sqrt": 4, "cmp": 20, "sign": 1},
    "allaire": {"add": 392, "mul": 423, "div": 156, "sqrt": 4, "cmp": 53, "sign": 18},
}


@pytest.mark.parametrize("model", ["euler", "allaire"])
def test_face_counts_pinned(model):
    import opcount_report as R

    assert R.face_counts(model) == FACE[model]


# compute_dt does the same work on every cell (E/sourcecode/euler_timestep.cpp:7-44,
# A/sourcecode/allaire_diffuse_timestep.cpp:8-48), then once per step picks dt:
# the CFL cap of the first five steps, min(dx/max_u, dy/max_v) times CFL, and
# the end-time test.
DT_PER_STEP_FIRST_FIVE = {"add": 1, "mul": 1, "div": 2, "sqrt": 0, "cmp": 3, "sign": 0}
DT_PER_CELL = {
    "euler": {"add": 8, "mul": 7, "div": 4, "sqrt": 1, "cmp": 2, "sign": 2},
    "allaire": {"add": 26, "mul": 13, "div": 16, "sqrt": 1, "cmp": 2, "sign": 2},
}


@pytest.mark.parametrize("name", ["euler_cross_48x40_vanleer", "allaire_ST2_x_100x10"])
def test_compute_dt_counts_per_cell(name):
    fx = load_golden(name)
    model = str(fx["model"])
    p = params_from(fx)
    grid = ghost_grid(fx["ic"], O.ghosts_of(p))
    taken, _, _, counts = O.opcount_run(model, p, grid, 3)
    cells = p.nx * p.ny * taken
    assert taken == 3
    assert counts["dt"] == {k: v * cells + DT_PER_STEP_FIRST_FIVE[k] * taken
                            for k, v in DT_PER_CELL[model].items()}
