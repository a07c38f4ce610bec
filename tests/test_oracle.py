"""The CPU oracle pinned against the reference.

The plain-C restatement (oracle/cfd_oracle.c) must reproduce, bit for bit,
(a) the golden fixtures recorded from the reference's own build
(tests/golden/make_golden.py) and (b) the reference build itself where it is
present (oracle/_ref, built from the reference sources in this container).
"""
import numpy as np
import pytest

import oracle_py as O
from cfdtest import GOLDEN, KATS, density, ghost_grid, load_golden, params_from, rel_l1

FIXTURES = sorted(p.stem for p in GOLDEN.glob("*.npz") if not p.stem.startswith(("kat_", "outputs_")))

pytestmark = pytest.mark.skipif(not O.port_available(), reason="oracle/_build not built")


@pytest.mark.parametrize("name", FIXTURES)
def test_port_reproduces_golden_run(name):
    fx = load_golden(name)
    model = str(fx["model"])
    p = params_from(fx)
    g = O.ghosts_of(p)
    grid = ghost_grid(fx["ic"], g)
    taken, n, t, dts = O.port_run(model, p, grid, int(fx["taken"]))
    assert taken == int(fx["taken"]) and n == int(fx["n"])
    assert t == float(fx["t"])
    assert np.array_equal(dts, fx["dts"])
    fin = grid[g:-g, g:-g]
    assert np.array_equal(density(fin, model), fx["rho"])
    if "state" in fx:
        assert np.array_equal(fin, fx["state"])
    assert rel_l1(density(fin, model), fx["rho"]) <= 1e-12


@pytest.mark.parametrize("name", KATS)
def test_port_reproduces_reference_faces(name):
    model = name.split("_")[2]
    fx = load_golden(name)
    p = params_from(fx)
    dt, dx = float(fx["dt"]), float(fx["dx"])
    for f in range(fx["stencils"].shape[0]):
        flux, us, zs = O.port_face_flux(model, p, fx["stencils"][f], dt, dx)
        assert np.array_equal(flux, fx["flux"][f]), f
        assert us == fx["u_star"][f]
        if model == "allaire":
            assert zs == fx["z_star"][f]


LIVE = [
    ("euler", "totem_pole_3", 30, 61, 60, {}),
    ("euler", "multiple_circles_1", 40, 40, 40, {"limiter": 1}),
    ("euler", "cross", 33, 29, 30, {"limiter": 2, "cfl": 0.8}),
    ("euler", "totem_pole_1", 32, 24, 30, {"limiter": 3}),
    ("euler", "totem_pole_3", 30, 61, 30, {"fix_dy_halfstep": 1}),
    ("euler", "circular_explosion", 26, 30, 30, {"splitting": 1}),
    ("euler", "totem_pole_2", 20, 20, 30, {"flux_solver": 1}),
    ("allaire", "ST2_y", 10, 60, 50, {}),
    ("allaire", "TTC3_x_pure", 60, 8, 40, {"limiter": 2}),
    ("allaire", "circular_explosion", 30, 30, 20, {"limiter": 1}),
    ("allaire", "shocked_helium_bubble", 40, 20, 20, {}),
    ("allaire", "ST2_x", 60, 10, 40, {"wavespeed": 1, "z_min": 1e-6}),
    ("allaire", "ST1_x", 40, 6, 20, {"flux_solver": 1}),
    ("allaire", "shocked_helium_bubble", 30, 12, 20, {"splitting": 1}),
    ("allaire", "ST2_y", 8, 40, 30, {"fix_dy_halfstep": 1, "limiter": 1}),
    ("allaire", "TTC3_x_pure", 40, 6, 30, {"flux_solver": 1, "splitting": 1}),
    ("allaire", "ST2_x", 40, 8, 30, {"bc": (1, 0, 1, 1), "wavespeed": 1}),
    ("euler", "totem_pole_2", 20, 24, 30, {"flux_solver": 1, "splitting": 1}),
    ("euler", "cross", 24, 20, 30, {"bc": (1, 1, 1, 1)}),
]


@pytest.mark.skipif(not O.ref_available("allaire"), reason="reference build absent")
@pytest.mark.parametrize("model,case,nx,ny,steps,over", LIVE)
def test_port_matches_reference_build(model, case, nx, ny, steps, over):
    fs = "Godunov" if over.get("flux_solver") == 1 else "MUSCL"
    grid, p = O.ref_case_ic(model, case, nx, ny, fs)
    p.cfl = over.get("cfl", 0.5)
    for k, v in over.items():
        if k == "bc":  # reflective walls where the test case has none
            for side in range(4):
                p.bc[side] = v[side]
        elif k != "cfl":
            setattr(p, k, v)
    g2 = grid.copy()
    a = O.ref_run(model, p, grid, steps)
    b = O.port_run(model, p, g2, steps)
    assert a[:3] == b[:3]
    assert np.array_equal(a[3], b[3])
    assert np.array_equal(grid, g2)


@pytest.mark.skipif(not O.ref_available("euler"), reason="reference build absent")
@pytest.mark.parametrize("model", ["euler", "allaire"])
def test_port_compute_dt_matches_reference(model):
    case = "cross" if model == "euler" else "ST2_x"
    grid, p = O.ref_case_ic(model, case, 24, 20)
    p.cfl = 0.7
    for n in (0, 4, 5, 9):
        for t in (0.0, p.T - 1e-5):
            assert O.port_compute_dt(model, p, grid, n, t)[0] == O.ref_compute_dt(model, p, grid, n, t)


OUTPUT_RUNS = sorted(p.stem for p in GOLDEN.glob("outputs_*.npz"))


@pytest.mark.parametrize("run", OUTPUT_RUNS)
def test_port_and_writers_reproduce_reference_final_outputs(tmp_path, run):
    """The oracle run to T with the reference's buffer semantics (ghost cells
    as its grid holds them), written by the library's host writers, gives the
    reference's final output files byte for byte."""
    import ctypes as C

    import cfdgpu as G
    from cfdtest import params_from_config

    fx = load_golden(run)
    sf = tmp_path / "settingsfile.txt"
    sf.write_text(str(fx["settings"]).format(out=str(tmp_path) + "/"))
    L = G.lib()
    st = G.Settings()
    assert L.cfd_read_settings(str(sf).encode(), C.byref(st)) == 0
    cfg = G.Config()
    assert L.cfd_settings_config(C.byref(st), C.byref(cfg)) == 0
    grid = np.zeros(cfg.ghosted_shape())
    gp = grid.ctypes.data_as(C.POINTER(C.c_double))
    assert L.cfd_settings_ic(C.byref(st), C.byref(cfg), gp) == 0
    p, model = params_from_config(cfg)
    taken, n, t, _ = O.port_run(model, p, grid, 10**7)
    assert t == cfg.T
    base = st.basename
    assert L.cfd_write_state(C.byref(cfg), gp, base, t) == 0
    assert L.cfd_write_schlieren(C.byref(cfg), gp, base, t) == 0
    names = [f"-state-{t:f}.dat", f"-schlieren-{t:f}.dat"]
    if model == "allaire":
        assert L.cfd_write_lineout(C.byref(cfg), gp, base, n) == 0
        names += [f"-lineoutx-{n}.dat", f"-lineouty-{n}.dat"]
    prefix = base.decode().rsplit("/", 1)[1]
    for suffix in names:
        name = prefix + suffix
        assert name in fx, name
        assert (tmp_path / name).read_bytes() == fx[name].tobytes(), name


@pytest.mark.parametrize("recipe,nx,ny,nb,seed", [
    ("four_quadrant", 64, 48, 0, 0),
    ("shock_bubbles", 300, 200, 32, 5),
    ("shock_bubbles", 97, 131, 4, 20261203),
    ("water_shock_air_bubble", 200, 100, 1, 7),
    ("water_shock_air_bubble", 64, 32, 1, 20261203),
])
def test_port_recipes_equal_library_builder(recipe, nx, ny, nb, seed):
    """The CPU-side recipe builder that bench.py's reference arm uses (so that
    the reference runs without the library loaded) gives the library host
    builder's grid and parameters bit for bit."""
    import cfdgpu as G

    grid, p, _model = O.port_recipe_ic(recipe, nx, ny, seed, nb)
    cfg = G.recipe_config(recipe, nx, ny)
    ic = G.recipe_ic(cfg, recipe, seed=seed, nbubbles=nb)
    assert np.array_equal(grid, ic) and np.array_equal(np.signbit(grid), np.signbit(ic))
    assert (p.dx, p.dy, p.cfl, p.limiter, p.wavespeed, p.z_min, p.gamma1, p.pinf1, p.gamma2,
            p.pinf2) == (cfg.dx, cfg.dy, cfg.cfl, cfg.limiter, cfg.wavespeed, cfg.z_min,
                         cfg.gamma1, cfg.pinf1, cfg.gamma2, cfg.pinf2)
    assert tuple(p.bc) == tuple(cfg.bc) and (p.T == cfg.T or (np.isinf(p.T) and np.isinf(cfg.T)))
