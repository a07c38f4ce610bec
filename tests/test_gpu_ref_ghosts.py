"""Reference ghost values (cfd_set_reference_ghosts): the downloaded grid,
ghost cells and corners included, equals the grid the CPU oracle holds after
the same steps, which keeps the reference's buffer semantics (ghosts from
set_ICs, then the boundary fill made before the last sweep that read the
buffer; corners never refilled)."""
import numpy as np
import pytest

import cfdgpu as G
import oracle_py as O
from cfdtest import params_from_config

pytestmark = pytest.mark.gpu

CASES = [
    (G.EULER, "cross", 40, 36, {}, 37),
    (G.EULER, "circular_explosion", 36, 30, {"splitting": "strang"}, 23),
    (G.EULER, "totem_pole_1", 24, 22, {"flux_solver": "Godunov"}, 11),
    (G.EULER, "totem_pole_3", 30, 61, {"limiter": "vanleer"}, 17),
    (G.ALLAIRE, "ST2_x", 60, 8, {}, 20),
    (G.ALLAIRE, "shocked_helium_bubble", 40, 14, {"splitting": "strang"}, 15),
]


def _config(model, case, nx, ny, opt):
    cfg = G.case_config(model, case, nx, ny, flux_solver=opt.get("flux_solver", "MUSCL"))
    if "splitting" in opt:
        cfg.splitting = G.SPLIT[opt["splitting"]]
    if "limiter" in opt:
        cfg.limiter = G.LIMITERS[opt["limiter"]]
    return cfg


def _oracle(cfg, ic, steps):
    p, model = params_from_config(cfg)
    ref = ic.copy()
    O.port_run(model, p, ref, steps)
    return ref


@pytest.mark.parametrize("model,case,nx,ny,opt,steps", CASES)
@pytest.mark.parametrize("loop", ["device", "host"])
def test_reference_ghosts_match_oracle(model, case, nx, ny, opt, steps, loop):
    cfg = _config(model, case, nx, ny, opt)
    ic = G.case_ic(cfg, case)
    ref = _oracle(cfg, ic, steps)
    with G.Solver(cfg) as s:
        s.set_reference_ghosts(True)
        s.upload(ic)
        assert np.array_equal(s.download(G.GHOSTED_AOS_AS_REFERENCE), ic)
        if loop == "device":
            s.advance(steps)
        else:
            n, t = 0, 0.0
            for _ in range(steps):
                dt = s.compute_dt(n, t)
                s.step(dt)
                n, t = n + 1, t + dt
        out = s.download(G.GHOSTED_AOS_AS_REFERENCE)
        interior = s.download(G.GHOSTED_AOS)
    assert np.array_equal(out, ref)
    g = 1 if opt.get("flux_solver") == "Godunov" else 2
    assert np.array_equal(out[g:-g, g:-g], interior[g:-g, g:-g])


def test_reference_ghosts_of_device_built_case():
    cfg = G.case_config(G.EULER, "cross", 44, 40)
    ic = G.case_ic(cfg, "cross")
    ref = _oracle(cfg, ic, 9)
    with G.Solver(cfg) as s:
        s.set_reference_ghosts(True)
        s.upload_case("cross")
        assert np.array_equal(s.download(G.GHOSTED_AOS_AS_REFERENCE), ic)
        s.advance(9)
        assert np.array_equal(s.download(G.GHOSTED_AOS_AS_REFERENCE), ref)


def test_reference_ghosts_enabled_after_steps_and_disabled():
    cfg = G.case_config(G.EULER, "cross", 32, 32)
    ic = G.case_ic(cfg, "cross")
    ref = _oracle(cfg, ic, 20)
    with G.Solver(cfg) as s:
        s.upload(ic)
        s.advance(19)  # graph of 16 steps + 3 direct steps without the frame
        s.set_reference_ghosts(True)
        s.advance(1)
        out = s.download(G.GHOSTED_AOS_AS_REFERENCE)
        # corners: the frame started from this state's boundary fill, not
        # from the initial grid, so only the edges can match
        edge = np.ones(out.shape[:2], bool)
        for r in (slice(0, 2), slice(-2, None)):
            for c in (slice(0, 2), slice(-2, None)):
                edge[r, c] = False
        assert np.array_equal(out[edge], ref[edge])
        s.set_reference_ghosts(False)
        with pytest.raises(G.CfdError):
            s.download(G.GHOSTED_AOS_AS_REFERENCE)
        s.advance(16)  # recaptured graph without the frame still runs


def _schlieren_host(grid, model, dx, dy, g):
    """|grad rho| of the interior cells of a ghosted AoS grid, formed as the
    host writer forms it."""
    rho = grid[..., 0] if model == G.EULER else grid[..., 0] + grid[..., 1]
    gx = (rho[g:-g, g + 1:rho.shape[1] - g + 1] - rho[g:-g, g - 1:-g - 1]) / (2.0 * dx)
    gy = (rho[g + 1:rho.shape[0] - g + 1, g:-g] - rho[g - 1:-g - 1, g:-g]) / (2.0 * dy)
    return np.sqrt(gx * gx + gy * gy)


@pytest.mark.parametrize("model,case,nx,ny,opt,steps", CASES)
def test_device_schlieren_equals_host(model, case, nx, ny, opt, steps):
    """The schlieren field computed on the device equals the one formed from
    the downloaded grid, bit for bit, with either kind of ghost values."""
    cfg = _config(model, case, nx, ny, opt)
    ic = G.case_ic(cfg, case)
    g = 1 if opt.get("flux_solver") == "Godunov" else 2
    with G.Solver(cfg) as s:
        s.set_reference_ghosts(True)
        s.upload(ic)
        s.advance(steps)
        for layout in (G.GHOSTED_AOS, G.GHOSTED_AOS_AS_REFERENCE):
            host = _schlieren_host(s.download(layout), model, cfg.dx, cfg.dy, g)
            dev = s.schlieren(layout)
            assert dev.shape == host.shape
            assert np.array_equal(dev, host), layout
        with pytest.raises(G.CfdError):
            s.schlieren(G.SOA)
