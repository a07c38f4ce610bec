"""Continuous-batching server: results served in a mix equal the same
requests served alone (and the FP64 server equals the FP64 solver bit for
bit); requests that arrive while others run join and overlap; admission
respects the device-memory budget."""
import threading
import time

import numpy as np
import pytest

import cfdgpu as G
from cfdtest import density, rel_l1

pytestmark = pytest.mark.gpu


def _requests():
    reqs = []
    for k, (rec, nx, ny, steps) in enumerate([("shock_bubbles", 256, 256, 60),
                                              ("water_shock_air_bubble", 192, 96, 45),
                                              ("shock_bubbles", 128, 320, 80),
                                              ("shock_bubbles", 96, 96, 30),
                                              ("water_shock_air_bubble", 64, 32, 70)]):
        cfg = G.recipe_config(rec, nx, ny)
        reqs.append((cfg, G.recipe_ic(cfg, rec, seed=7 + k, nbubbles=5), steps))
    return reqs


@pytest.mark.parametrize("precision", [G.MIXED, G.FP64])
def test_served_in_mix_equals_served_alone(precision):
    reqs = _requests()
    with G.Server(precision, ticks_per_round=7) as srv:
        ids = [srv.submit(c, ic, n) for c, ic, n in reqs]
        mixed = [srv.wait(i) for i in ids]
        st = srv.stats()
    assert st.completed == len(reqs) and st.max_running >= 2  # they overlapped
    for (c, ic, n), (info, out) in zip(reqs, mixed):
        assert info.state == G.REQ_DONE and info.steps == n
        with G.Server(precision, ticks_per_round=5) as alone:
            i = alone.submit(c, ic, n)
            info1, out1 = alone.wait(i)
        assert info1.steps == n and info1.t == info.t
        assert np.array_equal(out1, out)


def test_wait_into_the_clients_buffer():
    """A result lands in the buffer the client passes (the same bits as a
    fresh array); a buffer of the wrong shape or type is refused before
    the call."""
    c, ic, n = _requests()[1]
    with G.Server(G.MIXED, ticks_per_round=8) as srv:
        a, b = srv.submit(c, ic, n), srv.submit(c, ic, n)
        with pytest.raises(ValueError):
            srv.wait(a, out=np.empty((3, 3, c.nvar)))
        with pytest.raises(ValueError):
            srv.wait(a, out=np.empty(c.ghosted_shape(), dtype=np.float32))
        buf = np.full(c.ghosted_shape(), np.nan)
        info, got = srv.wait(a, out=buf)
        _, fresh = srv.wait(b)
    assert got is buf and info.steps == n
    assert np.array_equal(buf, fresh)


def test_fp64_served_equals_solver():
    c, ic, n = _requests()[0]
    with G.Server(G.FP64, ticks_per_round=16) as srv:
        info, out = srv.wait(srv.submit(c, ic, n))
    with G.Solver(c) as s:
        s.upload(ic)
        s.advance(n)
        ref = s.download()
    assert np.array_equal(out[2:-2, 2:-2], ref[2:-2, 2:-2])


def test_mixed_served_close_to_fp64_served():
    reqs = _requests()
    with G.Server(G.MIXED) as m, G.Server(G.FP64) as f:
        pairs = [(m.submit(c, ic, n), f.submit(c, ic, n), c) for c, ic, n in reqs]
        for im, jf, c in pairs:
            (_, a), (_, b) = m.wait(im), f.wait(jf)
            model = "euler" if c.model == G.EULER else "allaire"
            assert rel_l1(density(a[2:-2, 2:-2], model), density(b[2:-2, 2:-2], model)) <= 1e-4


def test_late_arrivals_join_running_work_and_budget_holds():
    cfg = G.recipe_config("shock_bubbles", 1024, 1024)
    ic = G.recipe_ic(cfg, "shock_bubbles", nbubbles=8)
    need = G.Batch.member_bytes(cfg)
    with G.Server(G.MIXED, budget_bytes=int(need * 2.5), ticks_per_round=4) as srv:
        first = srv.submit(cfg, ic, 6000)  # ~0.6 s of work
        time.sleep(0.05)
        late = [srv.submit(cfg, ic, 20) for _ in range(4)]  # at most 2 resident at a time
        peak = 0
        for _ in range(2000):
            st = srv.stats()
            peak = max(peak, st.running)
            assert st.used_bytes <= st.budget_bytes
            if st.completed == 5:
                break
            time.sleep(0.01)
        infos = [srv.wait(i, want_result=False)[0] for i in [first] + late]
        st = srv.stats()
    assert st.completed == 5 and st.max_running == 2 and peak <= 2
    # the late requests finished while the long first one was still running
    assert min(i.latency_s for i in infos[1:]) < infos[0].latency_s


def test_submissions_from_many_threads():
    cfg = G.recipe_config("shock_bubbles", 64, 64)
    ic = G.recipe_ic(cfg, "shock_bubbles", nbubbles=4)
    with G.Server(G.MIXED, ticks_per_round=8) as srv:
        ids, lock = [], threading.Lock()

        def client(k):
            i = srv.submit(cfg, ic, 20 + k)
            with lock:
                ids.append((i, 20 + k))

        th = [threading.Thread(target=client, args=(k,)) for k in range(8)]
        [t.start() for t in th]
        [t.join() for t in th]
        for i, n in ids:
            info, _ = srv.wait(i, want_result=False)
            assert info.state == G.REQ_DONE and info.steps == n


@pytest.mark.parametrize("precision", [G.MIXED, G.FP64])
def test_pinned_arena_gives_the_same_results(precision):
    """Request grids in the server's pinned host arena (room for about two at
    a time here, so later requests reuse freed room and the rest fall back to
    pageable memory) give the results of a server without one."""
    reqs = _requests()
    room = 2 * max(ic.nbytes for _, ic, _ in reqs)
    outs = {}
    for pinned in (0, room):
        with G.Server(precision, ticks_per_round=6, host_pinned_bytes=pinned) as srv:
            got = []
            for _ in range(2):  # the second pass reuses arena room the first released
                ids = [srv.submit(c, ic, n) for c, ic, n in reqs]
                got.append([srv.wait(i)[1] for i in ids])
                for i in ids:
                    srv.release(i)
            outs[pinned] = got
    for a, b in zip(outs[0][0], outs[room][0]):
        assert np.array_equal(a, b)
    for a, b in zip(outs[room][0], outs[room][1]):
        assert np.array_equal(a, b)
