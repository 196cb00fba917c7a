"""Known answers of the oracle's doubly periodic turbulence restatement
(examples/2d_decaying_turbulence_gpu.jl; nonlinear_padding.jl;
step_diagonal_imex.jl).  CPU only."""
import numpy as np
import pytest

from oracle.tarang_oracle import (
    padded_multiply_2d,
    rel_l2,
    run_turb,
    turb_backward,
    turb_forward,
    turb_initial_spec,
    turb_rhs,
    turb_wavenumbers,
)


def grid(Nx, Ny):
    x = np.arange(Nx) * 2 * np.pi / Nx
    y = np.arange(Ny) * 2 * np.pi / Ny
    return np.meshgrid(x, y)


def test_transform_round_trip():
    rng = np.random.default_rng(0)
    g = rng.standard_normal((12, 16))
    assert np.abs(turb_backward(turb_forward(g), 16) - g).max() < 1e-13


def test_resolved_product_is_pointwise():
    X, Y = grid(16, 12)
    a = np.cos(2 * X) * np.sin(Y)
    b = np.sin(3 * X + 1) * np.cos(2 * Y)
    assert np.abs(padded_multiply_2d(a, b) - a * b).max() < 1e-13


def test_nyquist_modes_keep_full_amplitude():
    # the reason for the symmetric split/fold (nonlinear_padding.jl:182-190):
    # a Nyquist mode times 1 comes back at full amplitude along either axis
    X, Y = grid(16, 12)
    for a in (np.cos(8 * X) * np.cos(2 * Y), np.cos(2 * X) * np.cos(6 * Y), np.cos(8 * X) * np.cos(6 * Y)):
        assert np.abs(padded_multiply_2d(a, np.ones_like(a)) - a).max() < 1e-13


def test_single_mode_is_steady_under_advection():
    # psi ~ q for a single wavenumber shell: u.grad q = 0
    Nx, Ny = 32, 32
    X, Y = grid(Nx, Ny)
    q = turb_forward(np.cos(3 * X + 4 * Y))
    F = turb_rhs(q, Nx, 2 * np.pi, 2 * np.pi)
    assert np.abs(F).max() < 1e-10 * np.abs(q).max()


def test_sbdf_startup_and_viscous_decay():
    Nx, Ny, nu, dt = 16, 16, 0.05, 0.1
    X, Y = grid(Nx, Ny)
    q0 = turb_forward(np.cos(2 * X + Y))
    k2 = 5.0
    q1 = run_turb(q0, Nx, 2 * np.pi, 2 * np.pi, nu, dt, 1)
    assert np.abs(q1 - q0 / (1 + dt * nu * k2)).max() < 1e-12 * np.abs(q0).max()
    # SBDF2: q_{n+1} (3/2 + dt L) = 2 q_n - q_{n-1}/2 for a steady mode
    q2 = run_turb(q0, Nx, 2 * np.pi, 2 * np.pi, nu, dt, 2)
    want = (2 * q1 - 0.5 * q0) / (1.5 + dt * nu * k2)
    assert np.abs(q2 - want).max() < 1e-12 * np.abs(q0).max()


def test_initial_spectrum_is_seeded_and_scaled():
    a = turb_initial_spec(32, 32, 3)
    b = turb_initial_spec(32, 32, 3)
    assert np.array_equal(a, b)
    assert abs(np.abs(turb_backward(a, 32)).max() - 10.0) < 1e-12
    kx, ky = turb_wavenumbers(32, 32, 2 * np.pi, 2 * np.pi)
    assert np.abs(a[np.sqrt(kx ** 2 + ky ** 2) > 32 / 3.0 + 1e-9]).max() < 1e-9


@pytest.mark.parametrize("scheme,order", [("RK222", 2), ("RK443", 3)])
def test_diagonal_rk_order_on_viscous_decay(scheme, order):
    # a single mode is steady under advection, so q(t) = q0 exp(-nu k^2 t)
    # exactly: the step error falls as dt^order
    from oracle.tarang_oracle import run_turb_rk

    Nx = Ny = 16
    x = np.arange(Nx) * 2 * np.pi / Nx
    X, Y = np.meshgrid(x, x)
    q0 = turb_forward(np.cos(2 * X + Y))
    nu, T = 0.2, 0.5
    exact = q0 * np.exp(-nu * 5.0 * T)
    errs = []
    for n in (8, 16, 32):
        q = run_turb_rk(q0, Nx, 2 * np.pi, 2 * np.pi, nu, T / n, n, scheme)
        errs.append(np.abs(q - exact).max())
    rates = [np.log2(errs[i] / errs[i + 1]) for i in range(2)]
    assert min(rates) > order - 0.3, (errs, rates)


def test_diagonal_rk_is_l_stable_in_the_stiff_limit():
    # dt nu k^2 = 1e4: an L-stable step damps the mode (the ESDIRK tableau with
    # its off-diagonal terms; without them |R| -> |1 - 1/gamma| > 1)
    from oracle.tarang_oracle import turb_step_rk, TABLEAUS

    Nx = Ny = 16
    x = np.arange(Nx) * 2 * np.pi / Nx
    X, Y = np.meshgrid(x, x)
    q0 = turb_forward(np.cos(2 * X + Y))
    for scheme in ("RK222", "RK443"):
        q = turb_step_rk(q0, Nx, 2 * np.pi, 2 * np.pi, 1e4 / 5.0, 1.0, TABLEAUS[scheme])
        assert np.abs(q).max() < 1e-2 * np.abs(q0).max(), scheme


def test_diagonal_rk_and_sbdf2_agree_as_dt_shrinks():
    from oracle.tarang_oracle import run_turb_rk

    Nx = Ny = 32
    q0 = turb_initial_spec(Nx, Ny, seed=3)
    nu, T = 1e-3, 0.02
    a = run_turb_rk(q0, Nx, 2 * np.pi, 2 * np.pi, nu, T / 8, 8, "RK443")
    b = run_turb(q0, Nx, 2 * np.pi, 2 * np.pi, nu, T / 64, 64)
    assert rel_l2(a, b) < 1e-4


# The reference's own known answers for the diagonal IMEX steppers
# (test/test_diagonal_imex.jl:208-308).  A single Fourier mode is steady under
# the advection, so the vorticity problem reduces to their viscous decay.
def _mode(N, k):
    x = np.arange(N) * 2 * np.pi / N
    X, _ = np.meshgrid(x, x)
    return turb_forward(np.cos(k * X))


@pytest.mark.parametrize("scheme", ["RK222", "RK443", "SBDF2"])
def test_reference_pin_viscous_rate(scheme):
    # cos(2x), nu = 0.5, dt = 0.005, 200 steps: amplitude exp(-nu k^2 T) =
    # exp(-2) within the reference's rtol 0.05 (and far closer here)
    from oracle.tarang_oracle import run_turb_rk

    N = 16
    q0 = _mode(N, 2)
    if scheme == "SBDF2":
        q = run_turb(q0, N, 2 * np.pi, 2 * np.pi, 0.5, 0.005, 200)
    else:
        q = run_turb_rk(q0, N, 2 * np.pi, 2 * np.pi, 0.5, 0.005, 200, scheme)
    ratio = np.abs(turb_backward(q, N)).max() / np.abs(turb_backward(q0, N)).max()
    assert abs(ratio - np.exp(-2.0)) < 0.05 * np.exp(-2.0)
    assert abs(ratio - np.exp(-2.0)) < 1e-3 * np.exp(-2.0)


@pytest.mark.parametrize("scheme", ["RK222", "RK443"])
def test_reference_pin_stiff_mode_is_damped(scheme):
    # cos(6x), nu = 1, dt = 0.25 (dt nu k^2 = 9), 20 steps: finite, below the
    # start and below 1e-2 (the full ESDIRK tableau; a diagonal-only update
    # would grow ~2000x)
    from oracle.tarang_oracle import run_turb_rk

    N = 16
    q0 = _mode(N, 6)
    q = run_turb_rk(q0, N, 2 * np.pi, 2 * np.pi, 1.0, 0.25, 20, scheme)
    g, g0 = np.abs(turb_backward(q, N)).max(), np.abs(turb_backward(q0, N)).max()
    assert np.isfinite(g) and g < g0 and g < 1e-2
