"""Host-side hooks of the library (no GPU needed): the restated reference
initial conditions, settings parsing and the output formats."""
import ctypes as C
import filecmp
import re

import numpy as np
import pytest

import cfdgpu as G
import oracle_py as O
from cfdtest import GOLDEN, ROOT, load_golden

EULER_CASES = ["circular_explosion", "multiple_circles_1", "multiple_circles_2", "cross",
               "totem_pole_1", "totem_pole_2", "totem_pole_3"]
ALLAIRE_CASES = ["ST1_x", "ST1_y", "ST2_x", "ST2_y", "TTC1_x_pure", "TTC2_y_pure", "TTC3_x_pure",
                 "TTC4_y_pure", "TTC5_x_pure", "circular_explosion", "shocked_helium_bubble",
                 "shocked_R22_bubble", "underwater_shocked_bubble", "underwater_explosion",
                 "underwater_explosion_modified", "shocked_SF6", "TSTM", "RMI_SF6",
                 "tin_air_implosion"]


def _cmp_params(cfg, p):
    assert (cfg.dx, cfg.dy, cfg.x0, cfg.y0, cfg.T) == (p.dx, p.dy, p.x0, p.y0, p.T)
    assert cfg.gamma1 == p.gamma1 and cfg.pinf1 == p.pinf1
    assert list(cfg.bc) == list(p.bc)


@pytest.mark.skipif(not O.ref_available("euler"), reason="reference build absent")
@pytest.mark.parametrize("case", EULER_CASES)
@pytest.mark.parametrize("fs", ["MUSCL", "Godunov"])
def test_euler_case_ic_matches_reference(case, fs):
    ref, p = O.ref_case_ic("euler", case, 37, 29, fs)
    cfg = G.case_config(G.EULER, case, 37, 29, fs)
    _cmp_params(cfg, p)
    ours = G.case_ic(cfg, case)
    assert np.array_equal(ours, ref)


@pytest.mark.skipif(not O.ref_available("allaire"), reason="reference build absent")
@pytest.mark.parametrize("case", ALLAIRE_CASES)
def test_allaire_case_ic_matches_reference(case):
    ref, p = O.ref_case_ic("allaire", case, 31, 23)
    cfg = G.case_config(G.ALLAIRE, case, 31, 23)
    _cmp_params(cfg, p)
    assert cfg.gamma2 == p.gamma2 and cfg.pinf2 == p.pinf2
    ours = G.case_ic(cfg, case)
    assert np.array_equal(ours, ref)


@pytest.mark.parametrize("name,model,case", [
    ("euler_totem_pole_3_30x61", G.EULER, "totem_pole_3"),
    ("euler_cross_48x40_vanleer", G.EULER, "cross"),
    ("allaire_ST2_x_100x10", G.ALLAIRE, "ST2_x"),
    ("allaire_ST1_y_12x80_mc", G.ALLAIRE, "ST1_y"),
])
def test_case_ic_matches_golden(name, model, case):
    fx = load_golden(name)
    ny, nx, _ = fx["ic"].shape
    cfg = G.case_config(model, case, nx, ny)
    assert cfg.dx == fx["p_dx"] and cfg.dy == fx["p_dy"]
    assert np.array_equal(G.case_ic(cfg, case)[2:-2, 2:-2], fx["ic"])


def test_recipe_ic_matches_golden():
    fx = load_golden("euler_four_quadrant_200x200")
    cfg = G.recipe_config("four_quadrant", 200, 200)
    assert np.array_equal(G.recipe_ic(cfg, "four_quadrant")[2:-2, 2:-2], fx["ic"])
    fx = load_golden("allaire_water_shock_64x32_pvrs")
    cfg = G.recipe_config("water_shock_air_bubble", 64, 32)
    assert np.array_equal(G.recipe_ic(cfg, "water_shock_air_bubble")[2:-2, 2:-2], fx["ic"])


def test_shock_bubbles_recipe_is_physical_and_seeded():
    cfg = G.recipe_config("shock_bubbles", 128, 128)
    a = G.recipe_ic(cfg, "shock_bubbles", seed=7, nbubbles=32)
    b = G.recipe_ic(cfg, "shock_bubbles", seed=7, nbubbles=32)
    c = G.recipe_ic(cfg, "shock_bubbles", seed=8, nbubbles=32)
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    rho = a[..., 0]
    e = a[..., 3] / rho - 0.5 * ((a[..., 1] / rho) ** 2 + (a[..., 2] / rho) ** 2)
    assert (rho > 0).all() and (e > 0).all()
    # post-shock state left of x = 0.1, bubbles only right of x = 0.12
    assert np.allclose(rho[2:-2, 2], 8.0 / 3.0)
    assert rho.min() >= 0.1 - 1e-12 and rho.max() <= 10.0 + 1e-9


def test_settings_file_roundtrip(tmp_path):
    f = tmp_path / "settingsfile.txt"
    f.write_text("Nx 30\nNy 61\nCFL 0.5\nsplitting_scheme naive_splitting\n"
                 "test_case totem_pole_3\noutput_freq 40\noutputpath ./out/\n"
                 "flux_solver MUSCL\nriemann_solver HLLC\nproblem euler\nunknown_key 3\n")
    L = G.lib()
    st = G.Settings()
    assert L.cfd_read_settings(str(f).encode(), C.byref(st)) == 0
    assert (st.Nx, st.Ny, st.CFL, st.output_freq) == (30, 61, 0.5, 40)
    assert st.splitting_scheme == b"naive_splitting" and st.test_case == b"totem_pole_3"
    assert st.flux_solver == b"MUSCL" and st.riemann_solver == b"HLLC" and st.problem == b"euler"
    # basename as headers/settings_file.hpp:69 builds it
    assert st.basename == b"./out/euler-totem_pole_3-MUSCL-30-61"
    assert st.seed == 20261203 and st.nbubbles == 32 and st.steps == 0
    cfg = G.Config()
    assert L.cfd_settings_config(C.byref(st), C.byref(cfg)) == 0
    ref = G.case_config(G.EULER, "totem_pole_3", 30, 61)
    assert (cfg.model, cfg.nx, cfg.ny, cfg.dx, cfg.dy, cfg.T, list(cfg.bc)) == \
        (ref.model, ref.nx, ref.ny, ref.dx, ref.dy, ref.T, list(ref.bc))
    assert cfg.cfl == 0.5 and cfg.splitting == G.SPLIT["naive"]
    grid = np.zeros(cfg.ghosted_shape())
    assert L.cfd_settings_ic(C.byref(st), C.byref(cfg), grid.ctypes.data_as(C.POINTER(C.c_double))) == 0
    assert np.array_equal(grid, G.case_ic(cfg, "totem_pole_3"))


def test_settings_precision_fp64_fast(tmp_path):
    """`precision fp64_fast` selects the fast FP64 form (a batch member's
    form); a single solver rejects it, before any device call, as it rejects
    the mixed form."""
    f = tmp_path / "settingsfile.txt"
    f.write_text("Nx 64\nNy 64\nCFL 0.8\nsplitting_scheme naive_splitting\n"
                 "test_case shock_bubbles\noutput_freq 0\noutputpath o/\n"
                 "flux_solver MUSCL\nriemann_solver HLLC\nproblem euler\nprecision fp64_fast\n")
    L = G.lib()
    st = G.Settings()
    assert L.cfd_read_settings(str(f).encode(), C.byref(st)) == 0
    cfg = G.Config()
    assert L.cfd_settings_config(C.byref(st), C.byref(cfg)) == 0
    assert cfg.precision == G.FP64_FAST
    with pytest.raises(G.CfdError, match="batch members"):
        G.Solver(cfg)


def test_settings_extensions(tmp_path):
    f = tmp_path / "settingsfile.txt"
    f.write_text("Nx 64\nNy 32\nCFL 0.6\nsplitting_scheme strang_splitting\n"
                 "test_case water_shock_air_bubble\noutput_freq 0\noutputpath o/\n"
                 "flux_solver MUSCL\nriemann_solver HLLC\nproblem allaire\nprecision mixed\n"
                 "limiter vanleer\nwavespeed pvrs\nsteps 7\nalpha_clip 1e-5\nseed 5\n")
    L = G.lib()
    st = G.Settings()
    assert L.cfd_read_settings(str(f).encode(), C.byref(st)) == 0
    cfg = G.Config()
    assert L.cfd_settings_config(C.byref(st), C.byref(cfg)) == 0
    assert cfg.model == G.ALLAIRE and cfg.precision == G.MIXED
    assert cfg.splitting == G.SPLIT["strang"] and cfg.limiter == G.LIMITERS["vanleer"]
    assert cfg.wavespeed == G.WAVESPEED["pvrs"] and cfg.z_min == 1e-5 and st.steps == 7
    grid = np.zeros(cfg.ghosted_shape())
    assert L.cfd_settings_ic(C.byref(st), C.byref(cfg), grid.ctypes.data_as(C.POINTER(C.c_double))) == 0
    assert np.array_equal(grid, G.recipe_ic(cfg, "water_shock_air_bubble", seed=5))
    st.riemann_solver = b"Roe"
    assert L.cfd_settings_config(C.byref(st), C.byref(cfg)) != 0


def test_header_symbols_exported():
    """Every function declared in include/*.h is exported by libcfdgpu.so."""
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        txt = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names |= set(re.findall(r"\b(cfd_[a-z_0-9]+)\s*\(", txt))
    assert names, "no declarations found"
    L = G.lib()
    missing = [n for n in sorted(names) if not hasattr(L, n)]
    assert not missing, missing


def test_invalid_configs_rejected_without_touching_a_device():
    L = G.lib()
    cfg = G.recipe_config("four_quadrant", 16, 16)
    h = C.c_void_p()
    for field, bad in [("nx", 1), ("ny", 0), ("dx", 0.0), ("gamma1", 1.0), ("limiter", 7),
                       ("cfl", -1.0), ("z_min", 0.7)]:
        c = cfg.copy()
        setattr(c, field, bad)
        assert L.cfd_create(C.byref(c), C.byref(h)) == -1, field
        assert G.last_error()


def _schlieren_field(grid, model, dx, dy, g=2):
    """|grad rho| of the interior cells of a ghosted AoS grid by central
    differences, each operation as the writers form it."""
    rho = grid[..., 0] if model == "euler" else grid[..., 0] + grid[..., 1]
    gx = (rho[g:-g, g + 1:rho.shape[1] - g + 1] - rho[g:-g, g - 1:-g - 1]) / (2.0 * dx)
    gy = (rho[g + 1:rho.shape[0] - g + 1, g:-g] - rho[g - 1:-g - 1, g:-g]) / (2.0 * dy)
    return np.ascontiguousarray(np.sqrt(gx * gx + gy * gy))


@pytest.mark.skipif(not O.ref_available("euler"), reason="reference build absent")
@pytest.mark.parametrize("model,case", [("euler", "cross"), ("allaire", "ST2_x")])
def test_output_writers_match_reference(tmp_path, model, case):
    grid, p = O.ref_case_ic(model, case, 24, 18)
    p.cfl = 0.5
    O.ref_run(model, p, grid, 5)
    t = 0.0123456789
    O.ref_write(model, p, grid, str(tmp_path / "ref"), 5, t)
    cfg = G.case_config(G.EULER if model == "euler" else G.ALLAIRE, case, 24, 18)
    L = G.lib()
    gp = grid.ctypes.data_as(C.POINTER(C.c_double))
    assert L.cfd_write_state(C.byref(cfg), gp, str(tmp_path / "ours").encode(), t) == 0
    assert L.cfd_write_schlieren(C.byref(cfg), gp, str(tmp_path / "ours").encode(), t) == 0
    for kind in ("state", "schlieren"):
        a = tmp_path / f"ref-{kind}-0.012346.dat"
        b = tmp_path / f"ours-{kind}-0.012346.dat"
        assert a.exists() and b.exists()
        assert filecmp.cmp(a, b, shallow=False), kind
    # the field writer (used with the device-computed field) writes the same
    # file from |grad rho| formed the same way
    field = _schlieren_field(grid, model, cfg.dx, cfg.dy)
    fp = field.ctypes.data_as(C.POINTER(C.c_double))
    assert L.cfd_write_schlieren_field(C.byref(cfg), fp, str(tmp_path / "field").encode(), t) == 0
    assert filecmp.cmp(tmp_path / "ref-schlieren-0.012346.dat",
                       tmp_path / "field-schlieren-0.012346.dat", shallow=False)
    if model == "allaire":
        assert L.cfd_write_lineout(C.byref(cfg), gp, str(tmp_path / "ours").encode(), 5) == 0
        for kind in ("lineoutx", "lineouty"):
            a, b = tmp_path / f"ref-{kind}-5.dat", tmp_path / f"ours-{kind}-5.dat"
            assert a.exists() and b.exists()
            assert filecmp.cmp(a, b, shallow=False), kind


def test_checkpoint_info_rejects_non_checkpoints(tmp_path):
    f = tmp_path / "x.ckpt"
    f.write_bytes(b"CFDCKPT\0" + b"\0" * 16)
    with pytest.raises(G.CfdError):
        G.checkpoint_info(f)
    with pytest.raises(G.CfdError):
        G.checkpoint_info(tmp_path / "missing.ckpt")


_GOOD_SETTINGS = {"Nx": "30", "Ny": "20", "CFL": "0.5", "splitting_scheme": "naive_splitting",
                  "test_case": "cross", "output_freq": "3", "outputpath": "./o/",
                  "flux_solver": "MUSCL", "riemann_solver": "HLLC", "problem": "euler"}


@pytest.mark.parametrize("change,message", [
    ({"problem": "navier"}, "unknown problem 'navier'"),
    ({"flux_solver": "WENO"}, "unknown flux_solver 'WENO'"),
    ({"riemann_solver": None}, "unknown riemann_solver ''"),
    ({"splitting_scheme": "lie"}, "unknown splitting_scheme 'lie'"),
    ({"test_case": "nonesuch"}, "unknown Euler test case 'nonesuch'"),
    ({"problem": "allaire", "test_case": "cross"}, "unknown Allaire test case 'cross'"),
    ({"test_case": "water_shock_air_bubble"}, "is not a euler problem"),
    ({"Nx": None}, "need at least 2 cells"),
    ({"Ny": "-4"}, "need at least 2 cells"),
    ({"Nx": "abc"}, "need at least 2 cells"),
    ({"limiter": "superbee"}, "unknown limiter 'superbee'"),
    ({"wavespeed": "roe"}, "unknown wavespeed 'roe'"),
    ({"precision": "fp16"}, "unknown precision 'fp16'"),
])
def test_corrupted_settings_rejected_with_a_message(tmp_path, change, message):
    """A settings file the reference would assert on (or one with a bad
    value of an added key) fails with CFD_ERR_INVALID and says why; the
    reference's parser itself ignores unknown keys, and so does ours."""
    kv = {**_GOOD_SETTINGS, **change}
    f = tmp_path / "settingsfile.txt"
    f.write_text("".join(f"{k} {v}\n" for k, v in kv.items() if v is not None))
    L = G.lib()
    st = G.Settings()
    assert L.cfd_read_settings(str(f).encode(), C.byref(st)) == 0
    L.cfd_version()  # a successful call leaves the previous message alone
    cfg = G.Config()
    assert L.cfd_settings_config(C.byref(st), C.byref(cfg)) == -1
    assert message in G.last_error()


def test_host_hook_errors_carry_messages(tmp_path):
    L = G.lib()
    st = G.Settings()
    assert L.cfd_read_settings(str(tmp_path / "absent.txt").encode(), C.byref(st)) == -1
    assert "cannot open settings file" in G.last_error()
    cfg = G.Config()
    assert L.cfd_case_config(G.EULER, b"nonesuch", 8, 8, 0, C.byref(cfg)) == -1
    assert "unknown Euler test case 'nonesuch'" in G.last_error()
    assert L.cfd_recipe_config(99, 8, 8, C.byref(cfg)) == -1
    assert "unknown recipe 99" in G.last_error()
    cfg = G.recipe_config("four_quadrant", 8, 8)
    grid = np.zeros(cfg.ghosted_shape())
    gp = grid.ctypes.data_as(C.POINTER(C.c_double))
    assert L.cfd_recipe_ic(C.byref(cfg), 3, C.c_uint64(1), 1, gp) == -1
    assert "does not apply to this configuration" in G.last_error()
    base = str(tmp_path / "no_such_dir" / "run").encode()
    assert L.cfd_write_state(C.byref(cfg), gp, base, C.c_double(0.0)) == -1
    assert "cannot open output file" in G.last_error()
    assert L.cfd_write_lineout(C.byref(cfg), gp, base, 0) == -1
    assert "Allaire grids only" in G.last_error()
    assert L.cfd_checkpoint_info(str(tmp_path / "absent.ckpt").encode(), None, None, None) == -1
    assert "cannot open checkpoint" in G.last_error()
