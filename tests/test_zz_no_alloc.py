"""cfd_compute_dt_noalloc: compute_dt for callers that may not allocate
device memory (a host application that owns every device allocation through
its own pool or budget, or a latency-critical loop that cannot take the
device-wide synchronisation of cudaMalloc / cudaFree).  It must give what the
solver's own cfd_compute_dt / cfd_get_status give on the same state, call
after call, while only using the caller's buffers and the library's fixed
scratch array.  This file is collected last on purpose."""
import ctypes as C

import pytest

import cfdgpu as G

pytestmark = pytest.mark.gpu

TOL_MASS = 1e-12  # relative; the mass sums differ only in summation order


def _noalloc_fn():
    L = G.lib()
    f = L.cfd_compute_dt_noalloc
    f.restype = C.c_int
    f.argtypes = [C.POINTER(G.Config), C.c_void_p, C.c_int64, C.c_int, C.c_int, C.c_double,
                  C.c_void_p, C.c_void_p]
    return f


@pytest.mark.parametrize("recipe,nx,ny", [("shock_bubbles", 640, 480),
                                          ("water_shock_air_bubble", 256, 128)])
def test_noalloc_compute_dt_matches_solver_on_consecutive_calls(recipe, nx, ny):
    import torch

    f = _noalloc_fn()
    cfg = G.recipe_config(recipe, nx, ny)
    ic = G.recipe_ic(cfg, recipe, nbubbles=16)
    out = torch.zeros(5, dtype=torch.float64, device="cuda")  # caller-owned output
    with G.Solver(cfg) as s:
        s.upload(ic)
        # calls at n = 0 (CFL capped at 0.2) and after 6 steps (the full CFL)
        for call, advance in enumerate((0, 6)):
            s.advance(advance)
            st = s.status()  # synchronises the solver's stream
            assert st.n == advance
            dt_ref = s.compute_dt(st.n, st.t)
            ptr, plane, pitch = s.state_device()
            rc = f(C.byref(cfg), ptr, plane, pitch, st.n, st.t, out.data_ptr(), None)
            assert rc == 0, G.last_error()
            torch.cuda.synchronize()
            dt, mu, mv, m1, m2 = out.tolist()
            assert dt == dt_ref, call
            assert mu == st.maxu and mv == st.maxv, call
            assert abs(m1 - st.mass1) <= TOL_MASS * abs(st.mass1), call
            assert abs(m2 - st.mass2) <= TOL_MASS * max(abs(st.mass2), 1e-300), call


def test_noalloc_clamps_the_last_step_to_the_end_time():
    """A finite end time: when t + dt passes T the step is cut to T - t
    (E/sourcecode/euler_timestep.cpp:41), as the solver's compute_dt cuts it."""
    import torch

    f = _noalloc_fn()
    cfg = G.recipe_config("shock_bubbles", 320, 256)
    ic = G.recipe_ic(cfg, "shock_bubbles", nbubbles=8)
    with G.Solver(cfg) as s:
        s.upload(ic)
        full = s.compute_dt(7, 0.0)
    cfg.T = 10.0 * full
    out = torch.zeros(5, dtype=torch.float64, device="cuda")
    with G.Solver(cfg) as s:
        s.upload(ic)
        ptr, plane, pitch = s.state_device()
        for n, t in ((7, 0.0), (7, cfg.T - 0.25 * full), (2, cfg.T - 0.1 * full)):
            dt_ref = s.compute_dt(n, t)
            assert f(C.byref(cfg), ptr, plane, pitch, n, t, out.data_ptr(), None) == 0
            torch.cuda.synchronize()
            assert out[0].item() == dt_ref, (n, t)
        assert out[0].item() == cfg.T - (cfg.T - 0.1 * full)  # the clamp fired


def test_noalloc_allocates_nothing():
    """After the first call, further calls leave the device's free memory
    unchanged."""
    import torch

    f = _noalloc_fn()
    cfg = G.recipe_config("water_shock_air_bubble", 256, 128)
    ic = G.recipe_ic(cfg, "water_shock_air_bubble")
    out = torch.zeros(5, dtype=torch.float64, device="cuda")
    with G.Solver(cfg) as s:
        s.upload(ic)
        ptr, plane, pitch = s.state_device()
        assert f(C.byref(cfg), ptr, plane, pitch, 0, 0.0, out.data_ptr(), None) == 0
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info()
        for k in range(5):
            assert f(C.byref(cfg), ptr, plane, pitch, k, 0.0, out.data_ptr(), None) == 0
        torch.cuda.synchronize()
        free1, _ = torch.cuda.mem_get_info()
        assert free1 == free0


def test_noalloc_rejects_grids_beyond_its_scratch():
    f = _noalloc_fn()
    rows = G.lib().cfd_noalloc_max_rows()
    cfg = G.recipe_config("shock_bubbles", 64, rows + 1)
    fake = C.c_void_p(0x1000)  # never dereferenced: the size check comes first
    rc = f(C.byref(cfg), fake, 64 * (rows + 1), 64, 0, 0.0, fake, None)
    assert rc == -1
    assert "exceeds the fixed scratch" in G.last_error()


def test_noalloc_rejects_a_bad_configuration():
    """The configuration checks of cfd_create, before any device work."""
    f = _noalloc_fn()
    fake = C.c_void_p(0x1000)  # never dereferenced: the checks come first
    for field, bad in (("cfl", 0.0), ("dx", -1.0), ("gamma1", 1.0)):
        cfg = G.recipe_config("shock_bubbles", 64, 64)
        setattr(cfg, field, bad)
        assert f(C.byref(cfg), fake, 64 * 64, 64, 0, 0.0, fake, None) == -1, field
