"""The fast FP64 form (batch members of precision CFD_PREC_FP64_FAST): FP64
arithmetic with contracted multiply-adds and refined hardware reciprocals and
square roots.  Bar: relative L1 density error <= 1e-12 against the reference
(its recorded runs, and the bit-identical FP64 form at the benchmarked grids
over their full stated step counts), the same step counts and times to
rounding; and the batch's invariances (a member's result does not depend on
what else runs with it, checkpoints continue bit for bit)."""
import numpy as np
import pytest

import cfdgpu as G
from cfdtest import (GOLDEN, PARITY_CASES, config_from_params, density, ghost_grid, load_golden,
                     params_from, rel_l1)

pytestmark = pytest.mark.gpu
TOL_L1 = 1e-12  # relative L1 density error bound of the plain FP64 form

# recorded reference runs the batch can take (naive splitting)
RUNS = sorted(p.stem for p in GOLDEN.glob("*.npz")
              if not p.stem.startswith(("kat_", "outputs_")) and "strang" not in p.stem)


def _fast_cfg(cfg):
    c = cfg.copy()
    c.precision = G.FP64_FAST
    return c


def _fast_run(cfg, ic, steps):
    with G.Batch() as b:
        i = b.add(_fast_cfg(cfg), ic, max_steps=steps)
        b.step(steps)
        return b.download(i), b.status(i)


def _errors(a, b, model):
    ra = density(a, model)
    rb = density(b, model)
    return rel_l1(ra, rb), float(np.abs(ra - rb).max() / np.abs(rb).max())


def _final_state(fx):
    """The recorded final interior state (for density-only fixtures, a state
    whose density is the recorded one)."""
    if "state" in fx:
        return fx["state"]
    rho = fx["rho"]
    s = np.zeros(rho.shape + (4,))
    s[..., 0] = rho
    return s


@pytest.mark.parametrize("name", RUNS)
def test_fast64_matches_reference_run(name):
    fx = load_golden(name)
    model = str(fx["model"])
    p = params_from(fx)
    g = 1 if p.flux_solver == 1 else 2
    cfg = config_from_params(p, model)
    out, st = _fast_run(cfg, ghost_grid(fx["ic"], g), int(fx["taken"]))
    assert st.n == int(fx["n"])
    assert abs(st.t - float(fx["t"])) <= 1e-12 * max(1.0, abs(float(fx["t"])))
    l1, linf = _errors(out[g:-g, g:-g], _final_state(fx), model)
    print(f"{name}: fast FP64 vs reference L1 {l1:.2e} Linf {linf:.2e}")
    assert l1 <= TOL_L1


@pytest.mark.parametrize("model,case,nx,ny,steps,over",
                         [c for c in PARITY_CASES if c[5].get("splitting") != 1])
def test_fast64_matches_bit_exact_on_reference_cases(model, case, nx, ny, steps, over):
    """The bit-identical form's parity cases (the batch runs naive
    splitting): every limiter, Godunov, PVRS speeds, the alpha clip, the dy
    half step, walls, 2x2 / 2x50 / 50x3 grids."""
    fs = "Godunov" if over.get("flux_solver") == 1 else "MUSCL"
    cfg = G.case_config(G.EULER if model == "euler" else G.ALLAIRE, case, nx, ny, fs)
    cfg.cfl = over.get("cfl", 0.5)
    for k, v in over.items():
        if k != "cfl":
            setattr(cfg, k, v)
    ic = G.case_ic(cfg, case)
    g = 1 if fs == "Godunov" else 2
    with G.Solver(cfg) as s:
        s.upload(ic)
        s.advance(steps)
        ref, sr = s.download(), s.status()
    out, sf = _fast_run(cfg, ic, steps)
    assert sf.n == sr.n
    assert abs(sf.t - sr.t) <= 1e-12 * max(abs(sr.t), 1e-300)
    l1, linf = _errors(out[g:-g, g:-g], ref[g:-g, g:-g], model)
    print(f"{model} {case} {nx}x{ny} {over}: fast FP64 vs bit-exact L1 {l1:.2e} Linf {linf:.2e}")
    assert np.isfinite(out[g:-g, g:-g]).all()
    assert l1 <= TOL_L1


@pytest.mark.parametrize("recipe,nx,ny,nb,steps", [
    ("shock_bubbles", 4096, 4096, 32, 2000),
    ("water_shock_air_bubble", 2048, 1024, 1, 1500),
])
def test_fast64_vs_bit_exact_at_benchmarked_configs(recipe, nx, ny, nb, steps):
    """The benchmarked grids over their full stated step counts against the
    bit-identical FP64 form (which equals the reference bit for bit)."""
    cfg = G.recipe_config(recipe, nx, ny)
    ic = G.recipe_ic(cfg, recipe, nbubbles=nb)
    with G.Solver(cfg) as s:
        s.upload(ic)
        s.advance(steps)
        ref, sr = s.download(), s.status()
    out, sf = _fast_run(cfg, ic, steps)
    assert sf.n == sr.n == steps
    model = "euler" if cfg.model == G.EULER else "allaire"
    l1, linf = _errors(out[2:-2, 2:-2], ref[2:-2, 2:-2], model)
    print(f"{recipe} {nx}x{ny} {steps} steps: fast FP64 vs bit-exact L1 {l1:.2e} Linf {linf:.2e}, "
          f"t rel diff {abs(sf.t - sr.t) / sr.t:.1e}")
    assert np.isfinite(out).all()
    assert abs(sf.t - sr.t) <= 1e-12 * sr.t
    assert l1 <= TOL_L1


def test_fast64_member_alone_equals_in_mix():
    """A fast FP64 member gives the same bits alone and in a batch with
    other fast and mixed members of both models."""
    cfg_a = G.recipe_config("shock_bubbles", 300, 200)
    ic_a = G.recipe_ic(cfg_a, "shock_bubbles", nbubbles=8)
    alone, _ = _fast_run(cfg_a, ic_a, 60)
    cfg_b = G.recipe_config("water_shock_air_bubble", 256, 128)
    ic_b = G.recipe_ic(cfg_b, "water_shock_air_bubble")
    cfg_c = G.recipe_config("shock_bubbles", 97, 333)
    ic_c = G.recipe_ic(cfg_c, "shock_bubbles", nbubbles=4)
    with G.Batch() as b:
        b.add(cfg_c, ic_c, 80)                 # mixed Euler
        b.add(_fast_cfg(cfg_b), ic_b, 40)      # fast Allaire
        i = b.add(_fast_cfg(cfg_a), ic_a, 60)  # the member under test
        b.add(_fast_cfg(cfg_c), ic_c, 90)      # fast Euler
        b.add(cfg_b, ic_b, 70)                 # mixed Allaire
        b.step(100)
        in_mix = b.download(i)
        assert b.status(i).n == 60
    assert np.array_equal(alone, in_mix)


def test_fast64_checkpoint_resume_is_bit_exact(tmp_path):
    cfg = _fast_cfg(G.recipe_config("water_shock_air_bubble", 128, 64))
    ic = G.recipe_ic(cfg, "water_shock_air_bubble")
    with G.Batch() as b:
        i = b.add(cfg, ic, 50)
        b.step(50)
        straight = b.download(i)
    ck = tmp_path / "m.ckpt"
    with G.Batch() as b:
        i = b.add(cfg, ic, 50)
        b.step(20)
        b.save(i, ck)
    with G.Batch() as b:
        j = b.restore(ck)
        assert b.status(j).n == 20
        b.step(30)
        resumed = b.download(j)
    assert np.array_equal(straight, resumed)


def test_fast64_served_equals_batch():
    """Through the server (continuous batching, host buffers), each fast
    FP64 result equals the same solve run alone in a batch."""
    reqs = [("shock_bubbles", 200, 160, 4, 70), ("water_shock_air_bubble", 128, 64, 1, 50),
            ("shock_bubbles", 96, 256, 8, 40)]
    ics = []
    for recipe, nx, ny, nb, steps in reqs:
        cfg = G.recipe_config(recipe, nx, ny)
        ics.append((cfg, G.recipe_ic(cfg, recipe, nbubbles=nb), steps))
    with G.Server(G.FP64_FAST, budget_fraction=0.5, ticks_per_round=8) as srv:
        ids = [srv.submit(cfg, ic, steps) for cfg, ic, steps in ics]
        served = [srv.wait(i)[1] for i in ids]
    for (cfg, ic, steps), got in zip(ics, served):
        alone, st = _fast_run(cfg, ic, steps)
        assert st.n == steps
        assert np.array_equal(alone, got)
