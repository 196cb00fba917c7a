"""FP32 turbulence program on the GPU against the FP64 oracle restatement of
the reference's DiagonalIMEX_SBDF2 vorticity step.  Bar: 1e-4 relative L2
after a few steps (FP32 arithmetic, chaotic dynamics kept short)."""
import numpy as np
import pytest

from oracle.tarang_oracle import rel_l2, run_turb, turb_forward, turb_initial_spec

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("Nx,Ny", [(32, 32), (48, 32), (64, 96)])
def test_turbulence_matches_oracle(tb, Nx, Ny):
    q0 = turb_initial_spec(Nx, Ny, seed=11)
    nu, dt, n = 1e-3, 2e-3, 6
    want = run_turb(q0, Nx, 2 * np.pi, 2 * np.pi, nu, dt, n)
    t = tb.Turb2D(Nx, Ny, nu, q0)
    t.step(dt, n)
    assert rel_l2(t.vorticity(), want) < 1e-4


def test_turbulence_nyquist_content(tb):
    # white noise reaches the Nyquist rows and columns: exercises the
    # projection, split and fold paths
    Nx, Ny = 32, 24
    rng = np.random.default_rng(5)
    q0 = turb_forward(rng.standard_normal((Ny, Nx)))
    nu, dt, n = 1e-2, 1e-3, 4
    want = run_turb(q0, Nx, 2 * np.pi, 2 * np.pi, nu, dt, n)
    t = tb.Turb2D(Nx, Ny, nu, q0)
    t.step(dt, n)
    assert rel_l2(t.vorticity(), want) < 1e-4


def test_turbulence_single_mode_decays_exactly(tb):
    Nx = Ny = 16
    x = np.arange(Nx) * 2 * np.pi / Nx
    X, Y = np.meshgrid(x, x)
    q0 = turb_forward(np.cos(2 * X + Y))
    nu, dt = 0.05, 0.1
    t = tb.Turb2D(Nx, Ny, nu, q0)
    t.step(dt, 1)
    assert np.abs(t.vorticity() - q0 / (1 + dt * nu * 5.0)).max() < 1e-5 * np.abs(q0).max()


@pytest.mark.parametrize("scheme", ["RK222", "RK443"])
@pytest.mark.parametrize("Nx,Ny", [(32, 32), (48, 32)])
def test_diagonal_rk_matches_oracle(tb, scheme, Nx, Ny):
    from oracle.tarang_oracle import run_turb_rk

    ts = {"RK222": tb._lib.TB_RK222, "RK443": tb._lib.TB_RK443}[scheme]
    q0 = turb_initial_spec(Nx, Ny, seed=13)
    nu, dt, n = 1e-3, 2e-3, 6
    want = run_turb_rk(q0, Nx, 2 * np.pi, 2 * np.pi, nu, dt, n, scheme)
    t = tb.Turb2D(Nx, Ny, nu, q0, timestepper=ts)
    t.step(dt, n)
    assert rel_l2(t.vorticity(), want) < 1e-4


def test_diagonal_rk_stiff_single_mode(tb):
    # dt nu k^2 = 50: the oracle's L-stable RK443 damps the mode; FP32 follows
    from oracle.tarang_oracle import run_turb_rk

    Nx = Ny = 16
    x = np.arange(Nx) * 2 * np.pi / Nx
    X, Y = np.meshgrid(x, x)
    q0 = turb_forward(np.cos(2 * X + Y))
    nu, dt = 10.0, 1.0
    want = run_turb_rk(q0, Nx, 2 * np.pi, 2 * np.pi, nu, dt, 2, "RK443")
    t = tb.Turb2D(Nx, Ny, nu, q0, timestepper=tb._lib.TB_RK443)
    t.step(dt, 2)
    got = t.vorticity()
    assert np.abs(got - want).max() < 1e-5 * np.abs(q0).max()
    assert np.abs(got).max() < 1e-2 * np.abs(q0).max()


@pytest.mark.parametrize("scheme", ["RK222", "RK443", "SBDF2"])
def test_reference_pin_viscous_rate(tb, scheme):
    # the reference's known answer (test/test_diagonal_imex.jl:208-275): cos(2x),
    # nu = 0.5, dt = 0.005, 200 steps decays to exp(-2) (its bar: rtol 0.05)
    ts = {"RK222": tb._lib.TB_RK222, "RK443": tb._lib.TB_RK443, "SBDF2": tb._lib.TB_SBDF2}[scheme]
    N = 16
    x = np.arange(N) * 2 * np.pi / N
    X, _ = np.meshgrid(x, x)
    q0 = turb_forward(np.cos(2 * X))
    t = tb.Turb2D(N, N, 0.5, q0, timestepper=ts)
    t.step(0.005, 200)
    ratio = np.abs(t.vorticity()).max() / np.abs(q0).max()
    assert abs(ratio - np.exp(-2.0)) < 1e-3 * np.exp(-2.0)


@pytest.mark.parametrize("scheme", ["RK222", "RK443"])
def test_reference_pin_stiff_mode_is_damped(tb, scheme):
    # test/test_diagonal_imex.jl:278-308: cos(6x), nu = 1, dt = 0.25, 20 steps
    ts = {"RK222": tb._lib.TB_RK222, "RK443": tb._lib.TB_RK443}[scheme]
    N = 16
    x = np.arange(N) * 2 * np.pi / N
    X, _ = np.meshgrid(x, x)
    q0 = turb_forward(np.cos(6 * X))
    t = tb.Turb2D(N, N, 1.0, q0, timestepper=ts)
    t.step(0.25, 20)
    g = np.abs(t.vorticity()).max() / np.abs(q0).max()
    assert np.isfinite(g) and g < 1e-2
