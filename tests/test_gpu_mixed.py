"""Mixed-precision batched form: accuracy against the FP64 path, batching
invariance (a member's result does not depend on what else is in the batch or
on the tile shapes), per-member stop conditions and budget admission."""
import numpy as np
import pytest

import cfdgpu as G
from cfdtest import PARITY_CASES, density, load_golden, rel_l1

pytestmark = pytest.mark.gpu
TOL_MIXED_L1 = 1e-4  # relative L1 density error of the mixed form vs FP64


def _fp64_run(cfg, ic, steps):
    with G.Solver(cfg) as s:
        s.upload(ic)
        s.advance(steps)
        st = s.status()
        return s.download(), st


def _mixed_run(cfg, ic, steps):
    with G.Batch() as b:
        i = b.add(cfg, ic, max_steps=steps)
        b.step(steps)
        st = b.status(i)
        return b.download(i), st


def _errors(a, b, model):
    ra = density(a[2:-2, 2:-2], model)
    rb = density(b[2:-2, 2:-2], model)
    return rel_l1(ra, rb), float(np.abs(ra - rb).max() / np.abs(rb).max())


@pytest.mark.parametrize("model,case,nx,ny,steps,over",
                         [c for c in PARITY_CASES if c[5].get("splitting") != 1])
def test_mixed_on_reference_cases(model, case, nx, ny, steps, over):
    """The mixed form on the bit-identical form's parity cases (the batch
    runs naive splitting): every limiter, Godunov, PVRS speeds, the alpha
    clip, the dy half step, walls, 2x2 / 2x50 / 50x3 grids.  Finite, the same
    step count, relative L1 density error within the mixed bound.  (Unlimited
    slopes at a contact give a face state of exactly zero density, which the
    reference's physicality test rejects.)  The physicality decisions of the
    mixed form are taken in FP32: with unlimited (non-TVD) slopes, states
    extrapolated at a strong jump land within FP32 rounding of the boundary
    and a decision taken the other way puts that face to first order, so that
    case gets a 1e-3 bound; limited slopes keep the extrapolated states inside
    their neighbours' range and no decision is near the boundary."""
    fs = "Godunov" if over.get("flux_solver") == 1 else "MUSCL"
    cfg = G.case_config(G.EULER if model == "euler" else G.ALLAIRE, case, nx, ny, fs)
    cfg.cfl = over.get("cfl", 0.5)
    for k, v in over.items():
        if k != "cfl":
            setattr(cfg, k, v)
    ic = G.case_ic(cfg, case)
    g = 1 if fs == "Godunov" else 2
    ref, sr = _fp64_run(cfg, ic, steps)
    mc = cfg.copy()
    mc.precision = G.MIXED
    out, sm = _mixed_run(mc, ic, steps)
    assert sm.n == sr.n
    assert np.isfinite(out[g:-g, g:-g]).all()
    ra = density(out[g:-g, g:-g], model)
    rb = density(ref[g:-g, g:-g], model)
    l1 = rel_l1(ra, rb)
    print(f"{model} {case} {nx}x{ny} {over}: mixed vs bit-exact L1 {l1:.2e}")
    assert l1 <= (1e-3 if cfg.limiter == G.LIMITERS["unlimited"] else TOL_MIXED_L1)


def test_mixed_four_quadrant_vs_reference_golden():
    fx = load_golden("euler_four_quadrant_200x200")
    cfg = G.recipe_config("four_quadrant", 200, 200)
    ic = G.recipe_ic(cfg, "four_quadrant")
    out, st = _mixed_run(cfg, ic, 100000)
    assert st.t == 0.3
    l1 = rel_l1(out[2:-2, 2:-2, 0], fx["rho"])
    linf = float(np.abs(out[2:-2, 2:-2, 0] - fx["rho"]).max() / fx["rho"].max())
    print(f"four-quadrant 200^2 to t=0.3: mixed vs reference L1 {l1:.2e} Linf {linf:.2e}")
    assert l1 <= TOL_MIXED_L1


@pytest.mark.parametrize("recipe,nx,ny,steps", [
    ("shock_bubbles", 512, 512, 300),
    ("water_shock_air_bubble", 256, 128, 300),
])
def test_mixed_vs_fp64(recipe, nx, ny, steps):
    cfg = G.recipe_config(recipe, nx, ny)
    ic = G.recipe_ic(cfg, recipe, nbubbles=32)
    ref, sr = _fp64_run(cfg, ic, steps)
    out, sm = _mixed_run(cfg, ic, steps)
    assert sm.n == sr.n == steps
    assert abs(sm.t - sr.t) <= 1e-4 * sr.t
    model = "euler" if cfg.model == G.EULER else "allaire"
    l1, linf = _errors(out, ref, model)
    print(f"{recipe} {nx}x{ny} {steps} steps: mixed vs FP64 L1 {l1:.2e} Linf {linf:.2e}")
    assert np.isfinite(out).all()
    assert l1 <= TOL_MIXED_L1


@pytest.mark.parametrize("recipe,nx,ny,nb,steps", [
    ("shock_bubbles", 4096, 4096, 32, 2000),
    ("water_shock_air_bubble", 2048, 1024, 1, 1500),
])
def test_mixed_vs_fp64_at_benchmarked_configs(recipe, nx, ny, nb, steps):
    """The mixed form against the plain FP64 form (bit-identical to the
    reference) at the benchmarked grids over their full stated step counts."""
    cfg = G.recipe_config(recipe, nx, ny)
    ic = G.recipe_ic(cfg, recipe, nbubbles=nb)
    ref, sr = _fp64_run(cfg, ic, steps)
    out, sm = _mixed_run(cfg, ic, steps)
    assert sm.n == sr.n == steps
    model = "euler" if cfg.model == G.EULER else "allaire"
    l1, linf = _errors(out, ref, model)
    print(f"{recipe} {nx}x{ny} {steps} steps: mixed vs FP64 L1 {l1:.2e} Linf {linf:.2e}, "
          f"t {sm.t:.9g} vs {sr.t:.9g}")
    assert np.isfinite(out).all()
    assert l1 <= TOL_MIXED_L1


@pytest.mark.parametrize("case,nx,ny", [("ST2_x", 200, 20), ("cross", 96, 80),
                                        ("shocked_helium_bubble", 130, 36)])
def test_mixed_reference_cases(case, nx, ny):
    model = G.ALLAIRE if case in ("ST2_x", "shocked_helium_bubble") else G.EULER
    cfg = G.case_config(model, case, nx, ny)
    ic = G.case_ic(cfg, case)
    steps = 150
    ref, sr = _fp64_run(cfg, ic, steps)
    out, sm = _mixed_run(cfg, ic, steps)
    l1, linf = _errors(out, ref, "euler" if model == G.EULER else "allaire")
    print(f"{case}: mixed vs FP64 L1 {l1:.2e} Linf {linf:.2e} (n={sm.n}, t={sm.t:.4g})")
    assert l1 <= TOL_MIXED_L1


@pytest.mark.parametrize("case,nx,ny", [("circular_explosion", 160, 140), ("totem_pole_1", 150, 170)])
def test_mixed_reflective_walls(case, nx, ny):
    """Wall-dominated Euler cases (reflective sides hit by blast waves): the
    reflective ghost sign must follow each tile's own boundary cells."""
    cfg = G.case_config(G.EULER, case, nx, ny)
    ic = G.case_ic(cfg, case)
    ref, _ = _fp64_run(cfg, ic, 250)
    out, _ = _mixed_run(cfg, ic, 250)
    l1, linf = _errors(out, ref, "euler")
    print(f"{case}: mixed vs FP64 L1 {l1:.2e} Linf {linf:.2e}")
    assert l1 <= TOL_MIXED_L1


def _members():
    out = []
    for k, (rec, nx, ny) in enumerate([("shock_bubbles", 96, 200), ("shock_bubbles", 300, 64),
                                       ("water_shock_air_bubble", 128, 64),
                                       ("shock_bubbles", 64, 64),
                                       ("water_shock_air_bubble", 90, 45)]):
        cfg = G.recipe_config(rec, nx, ny)
        out.append((cfg, G.recipe_ic(cfg, rec, seed=100 + k, nbubbles=6), 40 + 5 * k))
    return out


def test_member_alone_equals_member_in_mix():
    mem = _members()
    with G.Batch() as b:
        ids = [b.add(c, ic, steps) for c, ic, steps in mem]
        b.step(80)  # more ticks than any member needs
        mixed = [b.download(i) for i in ids]
        stats = [b.status(i) for i in ids]
    for (c, ic, steps), out, st in zip(mem, mixed, stats):
        assert st.n == steps and st.done
        alone, st1 = _mixed_run(c, ic, steps)
        assert st1.n == st.n and st1.t == st.t
        assert np.array_equal(alone, out)


def test_tile_shapes_do_not_change_results():
    """The y sweep's three tile shapes and its marching strips (shape 3) give
    the same bits (the x sweep has one form, the warp segments)."""
    mem = _members()[:3]
    outs = []
    for shape in range(4):
        with G.Batch() as b:
            for model in (G.EULER, G.ALLAIRE):
                b.set_shapes(model, 0, shape)
            ids = [b.add(c, ic, 20) for c, ic, _ in mem]
            b.step(20)
            outs.append([b.download(i) for i in ids])
    for k in range(len(mem)):
        for o in outs[1:]:
            assert np.array_equal(outs[0][k], o[k])


@pytest.mark.parametrize("prec", [G.MIXED, G.FP64_FAST])
def test_segment_rows_do_not_change_results(prec):
    """The x segments' row count is chosen per tile list (a lone small grid
    gets short tiles so that they fill the resident warps, a full batch
    longer ones); a member's result is the same bits either way."""
    cfg = G.recipe_config("water_shock_air_bubble", 300, 200)
    cfg.precision = prec
    ic = G.recipe_ic(cfg, "water_shock_air_bubble")
    big = G.recipe_config("water_shock_air_bubble", 2048, 1024)
    big.precision = prec
    big_ic = G.recipe_ic(big, "water_shock_air_bubble")
    with G.Batch() as b:
        i = b.add(cfg, ic, 25)
        alone_rows = b.segment_rows(G.ALLAIRE, prec)
        assert b.segment_rows(G.EULER, prec) == 0  # no Euler member
        b.step(25)
        alone = b.download(i)
    with G.Batch() as b:
        b.add(big, big_ic, 25)
        b.add(big, big_ic, 25)
        i = b.add(cfg, ic, 25)
        mix_rows = b.segment_rows(G.ALLAIRE, prec)
        b.step(25)
        in_mix = b.download(i)
    print(f"precision {prec}: segment rows alone {alone_rows}, in the mix {mix_rows}")
    assert 12 <= alone_rows < mix_rows <= 32
    assert np.array_equal(alone, in_mix)


def test_march_strip_lengths_do_not_change_results():
    """Marching strips of any length (the automatic choice, the shortest, an
    odd one that leaves ragged last strips, the longest) give the tiles' bits;
    lengths outside 16..64 are refused."""
    mem = _members()
    outs = {}
    for rows in ("tiles", 0, 16, 37, 64):
        with G.Batch() as b:
            for model in (G.EULER, G.ALLAIRE):
                if rows == "tiles":
                    b.set_shapes(model, 0, 0)
                else:
                    b.set_shapes(model, 0, 3)
                    b.set_march_rows(model, rows)
            ids = [b.add(c, ic, 30) for c, ic, _ in mem]
            if rows != "tiles":
                for model in (G.EULER, G.ALLAIRE):
                    used = b.march_rows(model)
                    assert 16 <= used <= 64 and (rows == 0 or used == rows)
            b.step(30)
            outs[rows] = [b.download(i) for i in ids]
    for rows in (0, 16, 37, 64):
        for k in range(len(mem)):
            assert np.array_equal(outs["tiles"][k], outs[rows][k]), (rows, k)
    with G.Batch() as b:
        for bad in (15, 65, -1):
            with pytest.raises(G.CfdError):
                b.set_march_rows(G.EULER, bad)
        assert b.march_rows(G.ALLAIRE) == 0  # no members: no strips


def test_two_phase_status_read_matches_poll():
    """poll_issue / poll_collect report what poll reports for the same point
    of the stream, mark finished members, and refuse a second issue."""
    mem = _members()[:3]
    with G.Batch() as b:
        ids = [b.add(c, ic, steps) for c, ic, steps in mem]
        assert b.poll_collect() == []  # nothing issued
        b.step(30)
        b.poll_issue()
        with pytest.raises(G.CfdError):
            b.poll_issue()
        got = b.poll_collect()
        assert got == b.poll()
        assert sorted(i for i, _, _, _ in got) == sorted(ids)
        b.step(60)  # every member reaches its step limit
        b.poll_issue()
        got = b.poll_collect()
        assert all(done for _, _, done, _ in got)
        assert {i: n for i, n, _, _ in got} == {i: st for i, (_, _, st) in zip(ids, mem)}


def test_autotune_keeps_results_and_picks_shapes():
    mem = _members()
    with G.Batch() as b:
        ids = [b.add(c, ic, 30) for c, ic, _ in mem]
        ms = b.autotune(2)  # 2 steps x (1 x form + 4 y forms) x 2 models of real work
        assert ms > 0
        b.step(30)
        tuned = [b.download(i) for i in ids]
    for (c, ic, _), out in zip(mem, tuned):
        alone, _ = _mixed_run(c, ic, 30)
        assert np.array_equal(alone, out)


def test_budget_admission():
    cfg = G.recipe_config("shock_bubbles", 512, 512)
    ic = G.recipe_ic(cfg, "shock_bubbles", nbubbles=4)
    need = G.Batch.member_bytes(cfg)
    with G.Batch(budget_bytes=int(need * 2.5)) as b:
        a1 = b.try_add(cfg, ic, 10)
        a2 = b.try_add(cfg, ic, 10)
        a3 = b.try_add(cfg, ic, 10)
        assert a1 is not None and a2 is not None and a3 is None
        n, used, budget = b.size()
        assert n == 2 and used <= budget
        b.remove(a1)
        assert b.try_add(cfg, ic, 10) is not None


def test_batch_forms_on_anisotropic_cells_with_dy_half_step():
    """Cells 4.6 times longer in x than in y (144 x 662 on the unit square,
    as in the batched workload) over 500 steps, with the y sweep's half step
    on dy: the mixed form within its bound and the fast FP64 form within the
    plain form's, against the bit-identical form.  (With the reference's dx
    half step, E/sourcecode/euler_colsweep.cpp:43, such a run is
    ill-conditioned: round-off grows to per cent between any two forms.)"""
    cfg = G.recipe_config("shock_bubbles", 144, 662)
    cfg.fix_dy_halfstep = 1
    ic = G.recipe_ic(cfg, "shock_bubbles", nbubbles=8)
    ref, sr = _fp64_run(cfg, ic, 500)
    out, sm = _mixed_run(cfg, ic, 500)
    fast_cfg = cfg.copy()
    fast_cfg.precision = G.FP64_FAST
    fast, sf = _mixed_run(fast_cfg, ic, 500)
    assert sm.n == sf.n == sr.n == 500
    l1_m, _ = _errors(out, ref, "euler")
    l1_f, _ = _errors(fast, ref, "euler")
    print(f"144x662 dy half step, 500 steps: mixed L1 {l1_m:.2e}, fast FP64 L1 {l1_f:.2e}")
    assert l1_m <= TOL_MIXED_L1
    assert l1_f <= 1e-12
