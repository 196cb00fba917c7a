"""PeriodicDomain and the vorticity problem through the Python mirror of the
reference API, written as examples/2d_decaying_turbulence_gpu.jl writes it:
fields on a doubly periodic domain, the q/psi/u system with its gauge, a
DiagonalIMEX solver, q["g"] set after the solver is built, run with a
callback.  Checked against the FP64 oracle."""
import numpy as np
import pytest

from oracle.tarang_oracle import (
    rel_l2,
    run_turb,
    run_turb_rk,
    turb_backward,
    turb_forward,
    turb_initial_spec,
    turb_wavenumbers,
)

pytestmark = pytest.mark.gpu


def test_periodic_transforms_match_the_oracle(tb):
    rng = np.random.default_rng(4)
    for Nx, Ny in ((32, 24), (96, 64)):
        T = tb.PeriodicTransform(Nx, Ny)
        g = rng.standard_normal((Ny, Nx))
        c = T.forward(g)
        assert rel_l2(c, turb_forward(g)) < 1e-13
        c2 = turb_forward(rng.standard_normal((Ny, Nx)))
        assert rel_l2(T.backward(c2), turb_backward(c2, Nx)) < 1e-13
        assert rel_l2(T.backward(c), g) < 1e-13


def build(tb, N, nu, dt, ts):
    domain = tb.PeriodicDomain(N, N)
    q = tb.ScalarField(domain, "q")
    psi = tb.ScalarField(domain, "psi")
    u = tb.VectorField(domain, "u")
    tau_psi = tb.ScalarField(domain, "tau_psi", bases=())
    problem = tb.IVP([q, psi, u, tau_psi])
    tb.add_parameters(problem, nu=nu)
    tb.add_equation(problem, "∂t(q) - nu*Δ(q) = -u⋅∇(q)")
    tb.add_equation(problem, "Δ(psi) + tau_psi - q = 0")
    tb.add_equation(problem, "u - skew(grad(psi)) = 0")
    tb.add_bc(problem, "integ(psi) = 0")
    solver = tb.InitialValueSolver(problem, ts, dt=dt)
    return domain, q, psi, u, solver


@pytest.mark.parametrize("scheme", ["SBDF2", "RK222", "RK443"])
def test_reference_style_turbulence_script(tb, scheme):
    N, nu, dt, n = 32, 1e-3, 2e-3, 6
    ts = {"SBDF2": tb.DiagonalIMEX_SBDF2(), "RK222": tb.DiagonalIMEX_RK222(), "RK443": tb.DiagonalIMEX_RK443()}
    domain, q, psi, u, solver = build(tb, N, nu, dt, ts[scheme])
    q0 = turb_backward(turb_initial_spec(N, N, seed=21), N)
    q["g"] = q0  # set after the solver exists, as the example does
    seen = []
    tb.run(solver, stop_iteration=n, callbacks=[(2, lambda s: seen.append(s.iteration))])
    assert seen == [2, 4, 6] and solver.iteration == n and abs(solver.sim_time - n * dt) < 1e-12
    c0 = turb_forward(q0)
    want = (run_turb(c0, N, 2 * np.pi, 2 * np.pi, nu, dt, n) if scheme == "SBDF2"
            else run_turb_rk(c0, N, 2 * np.pi, 2 * np.pi, nu, dt, n, scheme))
    got = q["c"]
    assert rel_l2(got, want) < 1e-4
    # psi and u follow from q: psi^ = -q^/k^2, u = (-d_y psi, d_x psi)
    kx, ky = turb_wavenumbers(N, N, 2 * np.pi, 2 * np.pi)
    k2 = kx ** 2 + ky ** 2
    psi_want = np.where(k2 > 0, -got / np.where(k2 > 0, k2, 1.0), 0.0)
    assert rel_l2(psi["c"], psi_want) < 1e-12
    assert rel_l2(u.components[0]["g"], turb_backward(-1j * ky * psi_want, N)) < 1e-12
    assert rel_l2(u.components[1]["g"], turb_backward(1j * kx * psi_want, N)) < 1e-12
    assert rel_l2(q["g"], turb_backward(got, N)) < 1e-12
    with pytest.raises(NotImplementedError):
        psi["g"] = np.zeros((N, N))


def test_enstrophy_decays_and_energy_is_nearly_kept(tb):
    # the example's diagnostics: enstrophy Z cascades and decays, energy E
    # (inverse cascade) decays far less over the same time
    N, nu, dt = 64, 1e-3, 2e-3
    domain, q, psi, u, solver = build(tb, N, nu, dt, tb.DiagonalIMEX_SBDF2())
    q["g"] = turb_backward(turb_initial_spec(N, N, seed=5), N)

    def EZ():
        ux, uy, qg = u.components[0]["g"], u.components[1]["g"], q["g"]
        return 0.5 * np.mean(ux ** 2 + uy ** 2), 0.5 * np.mean(qg ** 2)

    E0, Z0 = EZ()
    tb.run(solver, stop_iteration=200)
    E1, Z1 = EZ()
    assert Z1 < Z0 and E1 < E0
    assert (E0 - E1) / E0 < (Z0 - Z1) / Z0
