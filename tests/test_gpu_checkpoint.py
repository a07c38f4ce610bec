"""Checkpoint / resume: a solve saved after some steps and loaded into a new
solver (or batch) continues bit for bit like the uninterrupted solve."""
import numpy as np
import pytest

import cfdgpu as G

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("model,case,nx,ny,split", [
    (G.EULER, "cross", 64, 48, "naive"),
    (G.EULER, "circular_explosion", 50, 40, "strang"),
    (G.ALLAIRE, "shocked_helium_bubble", 60, 20, "naive"),
])
def test_solver_resume_is_bit_exact(tmp_path, model, case, nx, ny, split):
    cfg = G.case_config(model, case, nx, ny)
    cfg.splitting = G.SPLIT[split]
    ic = G.case_ic(cfg, case)
    path = tmp_path / "run.ckpt"
    with G.Solver(cfg) as a:
        a.set_reference_ghosts(True)
        a.upload(ic)
        a.advance(50)
        want, want_ref, st_a = a.download(), a.download(G.GHOSTED_AOS_AS_REFERENCE), a.status()
    with G.Solver(cfg) as b:
        b.set_reference_ghosts(True)
        b.upload(ic)
        b.advance(30)
        b.save(path)
    info_cfg, n, t = G.checkpoint_info(path)
    assert n == 30 and info_cfg.nx == nx and info_cfg.model == model
    with G.Solver(cfg) as c:
        c.set_reference_ghosts(True)
        c.load(path)
        c.advance(20)
        got, got_ref, st_c = c.download(), c.download(G.GHOSTED_AOS_AS_REFERENCE), c.status()
    assert np.array_equal(got, want) and np.array_equal(got_ref, want_ref)
    assert (st_c.n, st_c.t, st_c.dt_next) == (st_a.n, st_a.t, st_a.dt_next)


def test_load_rejects_other_solves(tmp_path):
    cfg = G.case_config(G.EULER, "cross", 32, 32)
    path = tmp_path / "a.ckpt"
    with G.Solver(cfg) as s:
        s.upload(G.case_ic(cfg, "cross"))
        s.save(path)
    other = G.case_config(G.EULER, "cross", 32, 30)
    with G.Solver(other) as s:
        with pytest.raises(G.CfdError):
            s.load(path)
    bad = tmp_path / "bad.ckpt"
    bad.write_bytes(path.read_bytes()[:300])
    with G.Solver(cfg) as s:
        with pytest.raises(G.CfdError):
            s.load(bad)
    with G.Batch() as b:  # an FP64 checkpoint is not a batch member
        with pytest.raises(G.CfdError):
            b.restore(path)


def test_batch_member_resume_is_bit_exact(tmp_path):
    mem = [("shock_bubbles", 96, 80, 9, 60), ("water_shock_air_bubble", 80, 40, 10, 45)]
    want = []
    with G.Batch() as b:
        ids = [b.add_recipe(G.recipe_config(r, nx, ny), r, seed=sd, max_steps=st)
               for r, nx, ny, sd, st in mem]
        b.step(70)
        want = [(b.download(i), b.status(i)) for i in ids]
    paths = [tmp_path / f"m{k}.ckpt" for k in range(len(mem))]
    with G.Batch() as b:
        ids = [b.add_recipe(G.recipe_config(r, nx, ny), r, seed=sd, max_steps=st)
               for r, nx, ny, sd, st in mem]
        b.step(25)
        for i, p in zip(ids, paths):
            b.save(i, p)
    with G.Batch() as b:
        ids = [b.restore(p) for p in paths]
        b.step(50)
        got = [(b.download(i), b.status(i)) for i in ids]
    for (wa, ws), (ga, gs) in zip(want, got):
        assert np.array_equal(ga, wa)
        assert (gs.n, gs.t, gs.done) == (ws.n, ws.t, ws.done)
