"""CPU checks of the oracle's dynamic wall values of b (per-stage ALG_F
refresh, step_subproblem_rk.jl:547-560): a wall profile equal to the constant
BCs reproduces the constant run, and an x- and t-dependent profile is held at
the walls at the stage time of the solve."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

from oracle.tarang_oracle import RBC2D, RBCParams, backward_2d, fourier_grid, rbc_initial_b, rel_l2  # noqa: E402


def _profile(p, f):
    x = fourier_grid(p.Nx, p.Lx)
    return np.fft.rfft(f(x))  # the wall values' coefficients (unnormalised rfft)


def test_constant_profile_reproduces_constant_bcs():
    p = RBCParams(Nx=16, Nz=12, Ra=1e5)
    a, b = RBC2D(p), RBC2D(p)
    for s in (a, b):
        s.set_b_grid(rbc_initial_b(p, 3, amp=1e-2))
    bot = _profile(p, lambda x: np.full_like(x, p.bottom()))
    top = _profile(p, lambda x: np.full_like(x, p.b_top))
    b.wall_b = lambda t: (bot, top)
    for _ in range(3):
        a.step(0.05, "RK443")
        b.step(0.05, "RK443")
    assert rel_l2(b.b, a.b) < 1e-13 and rel_l2(b.uz, a.uz) < 1e-12


def test_varying_profile_is_held_at_the_walls_at_the_solve_time():
    p = RBCParams(Nx=16, Nz=16, Ra=1e5)
    s = RBC2D(p)
    s.set_b_grid(rbc_initial_b(p, 3, amp=1e-2))
    k = 2 * np.pi / p.Lx

    def wall(t):
        return (_profile(p, lambda x: 1.0 + 0.1 * (1 + 5 * t) * np.cos(k * x)),
                _profile(p, lambda x: 0.05 * np.sin(2 * k * x) * t))

    s.wall_b = wall
    dt = 0.05
    s.step(dt, "SBDF1")
    g = backward_2d(s.b, p.Nx)  # row 0 is z = 0, the last row z = Lz
    x = fourier_grid(p.Nx, p.Lx)
    assert np.abs(g[0] - (1.0 + 0.1 * (1 + 5 * dt) * np.cos(k * x))).max() < 1e-10
    assert np.abs(g[-1] - 0.05 * np.sin(2 * k * x) * dt).max() < 1e-10
