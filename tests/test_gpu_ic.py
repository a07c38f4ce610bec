"""Device-built initial conditions (shape programs evaluated on the GPU) are
bit-identical to the host builders, which are pinned to the reference's own
set_ICs by the host-hook tests; the solver, batch and server paths that take
a recipe instead of a host grid give the same results as the host-grid paths."""
import numpy as np
import pytest

import cfdgpu as G

pytestmark = pytest.mark.gpu

EULER_CASES = ["circular_explosion", "multiple_circles_1", "multiple_circles_2", "cross",
               "totem_pole_1", "totem_pole_2", "totem_pole_3", "internet"]
ALLAIRE_CASES = ["ST1_x", "ST1_y", "ST2_x", "ST2_y", "TTC1_x_pure", "TTC2_y_pure", "TTC3_x_pure",
                 "TTC4_y_pure", "TTC5_x_pure", "circular_explosion", "shocked_helium_bubble",
                 "shocked_R22_bubble", "underwater_shocked_bubble", "underwater_explosion",
                 "underwater_explosion_modified"]
PER_CELL_CASES = ["shocked_SF6", "TSTM", "RMI_SF6", "tin_air_implosion"]


def _interior_soa(grid: np.ndarray, g: int) -> np.ndarray:
    return np.ascontiguousarray(np.moveaxis(grid[g:-g, g:-g, :], 2, 0))


def _same_bits(a: np.ndarray, b: np.ndarray) -> bool:
    return np.array_equal(a.view(np.uint64), b.view(np.uint64))


@pytest.mark.parametrize("recipe,nx,ny,nb,seed", [
    ("four_quadrant", 200, 200, 0, 0),
    ("shock_bubbles", 300, 257, 32, 5),
    ("shock_bubbles", 1024, 1024, 32, 20261203),
    ("shock_bubbles", 97, 203, 16, 11),
    ("water_shock_air_bubble", 256, 128, 0, 9),
    ("water_shock_air_bubble", 130, 66, 0, 3),
])
def test_device_recipe_matches_host(recipe, nx, ny, nb, seed):
    cfg = G.recipe_config(recipe, nx, ny)
    host = G.recipe_ic(cfg, recipe, seed=seed, nbubbles=nb)
    with G.Solver(cfg) as s:
        s.upload_recipe(recipe, seed=seed, nbubbles=nb)
        dev = s.download(G.SOA)
        st_dev = s.status()
    assert _same_bits(dev, _interior_soa(host, 2))
    with G.Solver(cfg) as s:
        s.upload(host)
        st_host = s.status()
    assert (st_dev.maxu, st_dev.maxv, st_dev.mass1, st_dev.mass2, st_dev.dt_next) == \
        (st_host.maxu, st_host.maxv, st_host.mass1, st_host.mass2, st_host.dt_next)


@pytest.mark.parametrize("model,case", [(G.EULER, c) for c in EULER_CASES] +
                         [(G.ALLAIRE, c) for c in ALLAIRE_CASES])
def test_device_case_matches_host(model, case):
    cfg = G.case_config(model, case, 70, 58)
    host = G.case_ic(cfg, case, seed=4)
    with G.Solver(cfg) as s:
        s.upload_case(case, seed=4)
        dev = s.download(G.SOA)
    assert _same_bits(dev, _interior_soa(host, 2))


def test_device_case_godunov_grid():
    cfg = G.case_config(G.EULER, "cross", 45, 33, flux_solver="Godunov")
    host = G.case_ic(cfg, "cross")
    with G.Solver(cfg) as s:
        s.upload_case("cross")
        dev = s.download(G.SOA)
    assert _same_bits(dev, _interior_soa(host, 1))


@pytest.mark.parametrize("case", PER_CELL_CASES)
def test_device_per_cell_cases_equal_host(case):
    """The Allaire cases with per-cell formulas (A/sourcecode/allaire_diffuse_io.cpp:659-983)
    built on the device: equal to the host build (which equals the
    reference's set_ICs bit for bit), with sin / cos / atan2 from CUDA."""
    cfg = G.case_config(G.ALLAIRE, case, 96, 80)
    host = G.case_ic(cfg, case)
    with G.Solver(cfg) as s:
        s.upload_case(case)
        dev = s.download(G.SOA)
    assert _same_bits(dev, _interior_soa(host, 2))


def test_recipe_for_wrong_model_rejected():
    cfg = G.recipe_config("water_shock_air_bubble", 64, 32)
    with G.Solver(cfg) as s:
        with pytest.raises(G.CfdError):
            s.upload_recipe("shock_bubbles")


def test_device_recipe_run_equals_host_upload_run():
    cfg = G.recipe_config("shock_bubbles", 256, 192)
    host = G.recipe_ic(cfg, "shock_bubbles", seed=77, nbubbles=24)
    with G.Solver(cfg) as a, G.Solver(cfg) as b:
        a.upload(host)
        b.upload_recipe("shock_bubbles", seed=77, nbubbles=24)
        a.advance(60)
        b.advance(60)
        assert np.array_equal(a.download(), b.download())


def test_batch_add_recipe_equals_add():
    mem = [("shock_bubbles", 96, 200, 12, 31), ("water_shock_air_bubble", 128, 64, 0, 32),
           ("shock_bubbles", 300, 64, 6, 33)]
    outs = []
    for use_recipe in (False, True):
        with G.Batch() as b:
            ids = []
            for rec, nx, ny, nb, seed in mem:
                cfg = G.recipe_config(rec, nx, ny)
                if use_recipe:
                    ids.append(b.add_recipe(cfg, rec, seed=seed, nbubbles=nb, max_steps=40))
                else:
                    ids.append(b.add(cfg, G.recipe_ic(cfg, rec, seed=seed, nbubbles=nb), 40))
            b.step(40)
            outs.append([b.download(i) for i in ids])
    for x, y in zip(*outs):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("precision", [G.MIXED, G.FP64])
def test_server_submit_recipe_equals_submit(precision):
    reqs = [("shock_bubbles", 128, 128, 8, 41, 30), ("water_shock_air_bubble", 96, 48, 0, 42, 25)]
    results = []
    for use_recipe in (False, True):
        srv = G.Server(precision)
        try:
            ids = []
            for rec, nx, ny, nb, seed, steps in reqs:
                cfg = G.recipe_config(rec, nx, ny)
                if use_recipe:
                    ids.append(srv.submit_recipe(cfg, rec, seed, nb, steps))
                else:
                    ids.append(srv.submit(cfg, G.recipe_ic(cfg, rec, seed=seed, nbubbles=nb),
                                          steps))
            got = [srv.wait(i) for i in ids]
        finally:
            srv.close()
        for (info, _), r in zip(got, reqs):
            assert info.state == G.REQ_DONE and info.steps == r[5]
        results.append([out for _, out in got])
    for x, y in zip(*results):
        assert np.array_equal(x, y)
