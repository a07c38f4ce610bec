"""cfd_compute_dt_noalloc: compute_dt for callers that may not allocate
device memory (inside someone else's graph capture, fixed-memory real-time
loops, applications that own every allocation).  It must give what the
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
        for call in range(2):
            st = s.status()  # synchronises the solver's stream
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
            s.advance(3)


def test_noalloc_rejects_grids_beyond_its_scratch():
    f = _noalloc_fn()
    rows = G.lib().cfd_noalloc_max_rows()
    cfg = G.recipe_config("shock_bubbles", 64, rows + 1)
    fake = C.c_void_p(0x1000)  # never dereferenced: the size check comes first
    rc = f(C.byref(cfg), fake, 64 * (rows + 1), 64, 0, 0.0, fake, None)
    assert rc == -1
    assert "exceeds the fixed scratch" in G.last_error()
