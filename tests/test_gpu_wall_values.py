"""Time- and space-dependent wall values of b through the C ABI
(tb_set_wall_values) against the oracle's per-stage ALG_F refresh."""
import numpy as np
import pytest

from oracle.tarang_oracle import (RBC2D, RBC3D, TABLEAUS, RBC3Params, RBCParams, forward_2d, forward_3d,
                                  fourier_grid, rbc3_initial_b, rbc_initial_b, rel_l2)

pytestmark = pytest.mark.gpu

TS = {"RK222": 0, "RK443": 1, "SBDF1": 2, "SBDF2": 3}


def _walls_2d(p):
    x = fourier_grid(p.Nx, p.Lx)
    k = 2 * np.pi / p.Lx
    b0 = np.fft.rfft(1.0 + 0.1 * np.cos(k * x))
    b1 = np.fft.rfft(0.5 * np.cos(k * x) + 0.2 * np.sin(3 * k * x))
    t0 = np.fft.rfft(0.05 * np.sin(2 * k * x))
    return b0, b1, t0


@pytest.mark.parametrize("scheme,dt", [("RK443", 0.01), ("SBDF2", 0.01), ("RK222", 0.05)])
def test_wall_values_2d_match_oracle(tb, scheme, dt):
    p = RBCParams(Nx=32, Nz=16, Lx=4.0, Lz=1.0, Ra=1e6)
    b0, b1, t0 = _walls_2d(p)
    sim = RBC2D(p)
    sim.set_b_grid(rbc_initial_b(p, 42))
    sim.wall_b = lambda t: (b0 + b1 * t, t0)
    dom = tb.ChannelDomain(p.Nx, p.Nz, Lx=p.Lx, Lz=p.Lz)
    plan = tb.Plan(dom, p.kappa, p.nu, 1.0, 0.0, TS[scheme])
    plan.set_state(0, forward_2d(rbc_initial_b(p, 42)))
    plan.set_wall_values(0, b0, b1)
    plan.set_wall_values(1, t0)
    for _ in range(4):
        sim.step(dt, scheme)
    plan.step(dt, 4)
    for f, want in ((0, sim.b), (1, sim.ux), (2, sim.uz)):
        assert rel_l2(plan.get_state(f), want) < 1e-10


def test_wall_values_set_between_steps_are_rereferenced(tb):
    # bottom ramps from t = 0; the top is set at t = 2 dt: the bottom ramp must
    # continue from where it was, not restart
    p = RBCParams(Nx=32, Nz=16, Lx=4.0, Lz=1.0, Ra=1e6)
    b0, b1, t0 = _walls_2d(p)
    dt = 0.02
    sim = RBC2D(p)
    sim.set_b_grid(rbc_initial_b(p, 7))
    sim.wall_b = lambda t: (b0 + b1 * t, np.zeros_like(t0) if t <= 2 * dt + 1e-12 else t0)
    dom = tb.ChannelDomain(p.Nx, p.Nz, Lx=p.Lx, Lz=p.Lz)
    plan = tb.Plan(dom, p.kappa, p.nu, 1.0, 0.0, TS["SBDF1"])
    plan.set_state(0, forward_2d(rbc_initial_b(p, 7)))
    plan.set_wall_values(0, b0, b1)
    plan.set_wall_values(1, np.zeros_like(t0))
    for _ in range(2):
        sim.step(dt, "SBDF1")
    plan.step(dt, 2)
    plan.set_wall_values(1, t0)
    for _ in range(2):
        sim.step(dt, "SBDF1")
    plan.step(dt, 2)
    assert rel_l2(plan.get_state(0), sim.b) < 1e-10


def test_wall_values_3d_match_oracle(tb):
    p = RBC3Params(Nx=16, Ny=12, Nz=12, Lx=4.0, Ly=3.0, Ra=1e5)
    g = np.zeros((1, p.Ny, p.Nx))
    x = fourier_grid(p.Nx, p.Lx)[None, :]
    y = fourier_grid(p.Ny, p.Ly)[:, None]
    prof = 1.0 + 0.1 * np.cos(2 * np.pi * x / p.Lx) * np.sin(2 * np.pi * y / p.Ly)
    bot = np.fft.fft(np.fft.rfft(prof, axis=1), axis=0)  # (Ny, Nx/2+1)
    rate = 0.3 * bot
    sim = RBC3D(p)
    sim.set_b_grid(rbc3_initial_b(p, 42, amp=1e-2))
    sim.wall_b = lambda t: (bot + rate * t, np.zeros_like(bot))
    plan = tb.Plan3D(p.Nx, p.Ny, p.Nz, p.kappa, p.nu, 0, p.Lx, p.Ly, p.Lz)
    plan.set_state(0, plan.forward(rbc3_initial_b(p, 42, amp=1e-2)))
    plan.set_wall_values(0, bot, rate)
    plan.set_wall_values(1, np.zeros_like(bot))
    for _ in range(3):
        sim.step_rk(0.05, TABLEAUS["RK222"])
    plan.step(0.05, 3)
    for name, f in (("b", 0), ("ux", 1), ("uy", 5), ("uz", 2)):
        assert rel_l2(plan.get_state(f), getattr(sim, name)) < 1e-10, name
