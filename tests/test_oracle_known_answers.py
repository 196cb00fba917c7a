"""The CPU oracle against the reference's own known-answer tests.

Each case restates an analytic check from the reference test suite or docs:
  - transform round trip / known Chebyshev coefficients  test/test_gpu_fc_2d_complete.jl:66-190
  - spectral derivatives vs analytic                    test/test_gpu_fc_2d_complete.jl:195-260
  - 3/2-dealiased products (incl. the Nyquist case)     test/test_gpu_fc_2d_complete.jl:262-330
  - Chebyshev D, BC rows, integration weights           test/test_chebyshev.jl:126-400
  - tau-method Poisson quick start u = z(1-z)           docs/src/pages/tau_method.md:35-85
  - walls enforced after nonlinear steps                test/test_gpu_fc_2d_complete.jl:395-420
  - RBC builds and steps finitely                        test/test_subproblem_rk.jl:19-110
  - min-norm mass solve = least squares                  test/test_batched_mass_solve.jl:169-220
  - time-stepper order on an exact linear solution      test/test_timestepper_boundaries.jl:78-176
  - variable-step SBDF2 / SBDF1 coefficient values       test/test_timestepper_boundaries.jl:78-176
  - DCT-I convention and the RF x Cheb forward chain     test/test_gpu_dct1_kernels_cpu.jl:35-214
  - T-basis derivative recurrence (orders 1 and 2)       test/test_gpu_dct1_kernels_cpu.jl:164-180
  - rfft / fft wavenumber orders and length scaling      test/test_basis_wavenumbers.jl:36-69
and writes the periodic and 3D transform conventions out as DFT sums
(src/core/transforms/transform_fourier.jl:473-590).
"""
import numpy as np
import numpy.polynomial.chebyshev as npc
import pytest

from oracle.tarang_oracle import (
    RBC2D,
    RBCParams,
    backward_2d,
    cheb_diff_matrix,
    cheb_eval_row,
    cheb_forward,
    cheb_grid,
    cheb_integ_row,
    fourier_grid,
    forward_2d,
    padded_length,
    padded_multiply,
    rbc_initial_b,
    rel_l2,
    run_rbc,
    wavenumbers_rfft,
)


def test_grids_and_wavenumbers():
    z = cheb_grid(9, 0.0, 1.0)
    assert z[0] == pytest.approx(0.0, abs=1e-15) and z[-1] == pytest.approx(1.0)
    assert np.all(np.diff(z) > 0)
    assert np.allclose(fourier_grid(8, 2 * np.pi), np.arange(8) * np.pi / 4)
    assert np.allclose(wavenumbers_rfft(8, 4.0), 2 * np.pi / 4 * np.arange(5))
    assert padded_length(12) == 18 and padded_length(256) == 384 and padded_length(1024) == 1536
    assert padded_length(6) == 10  # ceil(9) bumped to even


def test_transform_roundtrip_and_known_coefficients():
    Nx, Nz = 8, 9
    x = fourier_grid(Nx, 2 * np.pi)
    z = cheb_grid(Nz, 0.0, 1.0)
    prof = 1 + z + 0.25 * (2 * z**2 - 1)
    g = prof[:, None] * np.sin(2 * x)[None, :]
    c = forward_2d(g)
    assert np.abs(backward_2d(c, Nx) - g).max() < 1e-14
    # sin(2x) -> rfft bin 2 = -i Nx/2 ; profile's Chebyshev-T coefficients on [0,1]
    X = 2 * z - 1
    want = npc.chebfit(X, prof, Nz - 1)
    assert np.allclose(c[:, 2], -1j * Nx / 2 * want, atol=1e-13)
    assert np.abs(np.delete(c, 2, axis=1)).max() < 1e-13


def test_spectral_derivatives_match_analytic():
    Nx, Nz = 16, 11
    x = fourier_grid(Nx, 2 * np.pi)
    z = cheb_grid(Nz, 0.0, 1.0)
    prof, dprof = z**2 * (1 - z), 2 * z - 3 * z**2
    g = prof[:, None] * np.sin(2 * x)[None, :]
    c = forward_2d(g)
    k = wavenumbers_rfft(Nx, 2 * np.pi)
    D = cheb_diff_matrix(Nz, 1.0)
    gx = backward_2d(1j * k[None, :] * c, Nx)
    gz = backward_2d(D @ c, Nx)
    assert np.abs(gx - prof[:, None] * 2 * np.cos(2 * x)[None, :]).max() < 2e-10
    assert np.abs(gz - dprof[:, None] * np.sin(2 * x)[None, :]).max() < 2e-10


def test_dealiased_product_resolved_case_is_pointwise():
    Nx, Nz = 12, 9
    x = fourier_grid(Nx, 2 * np.pi)
    z = cheb_grid(Nz, 0.0, 1.0)
    a = (1 + z)[:, None] * np.cos(2 * x)[None, :]
    b = (1 - z)[:, None] * np.sin(3 * x)[None, :]
    assert np.abs(padded_multiply(a, b) - a * b).max() < 3e-9


def test_dealiased_product_nyquist_case():
    # cos(6x)(1+z) * cos(6x)(1-z) on 12 points: the Nyquist bin is split X/2 at
    # +-6 on the 18-point grid, cos(12x) aliases onto +-6 there, and truncation
    # folds both images back into the Nyquist bin.  Worked by hand from
    # nonlinear_padding.jl:182-226, 294-346, 359-443:
    #   result = (1 - z^2) (1 + cos(6x)) / 2
    Nx, Nz = 12, 9
    x = fourier_grid(Nx, 2 * np.pi)
    z = cheb_grid(Nz, 0.0, 1.0)
    a = (1 + z)[:, None] * np.cos(6 * x)[None, :]
    b = (1 - z)[:, None] * np.cos(6 * x)[None, :]
    want = (1 - z**2)[:, None] * (1 + np.cos(6 * x))[None, :] / 2
    assert np.abs(padded_multiply(a, b) - want).max() < 1e-14


def test_chebyshev_operator_rows():
    N = 12
    D = cheb_diff_matrix(N, 2.0)  # [-1, 1]
    for n in range(N):
        e = np.zeros(N)
        e[n] = 1
        want = npc.chebder(e) if n > 0 else np.zeros(1)
        got = D @ e
        assert np.allclose(got[: len(want)], want) and np.allclose(got[len(want):], 0)
    assert np.allclose(cheb_eval_row(N, 1.0), 1) and np.allclose(cheb_eval_row(N, -1.0), (-1.0) ** np.arange(N))
    w = cheb_integ_row(N, 1.0)
    for n in range(N):
        e = np.zeros(N)
        e[n] = 1
        I = npc.chebint(e, lbnd=-1)
        assert w[n] == pytest.approx(0.5 * npc.chebval(1.0, I), abs=1e-14)


def test_tau_poisson_quick_start():
    # D^2 u + tau1 e_{N-1} + tau2 e_{N-2} = -2 e_0, u(0) = u(1) = 0  ->  u = z(1-z)
    N = 16
    D = cheb_diff_matrix(N, 1.0)
    A = np.zeros((N + 2, N + 2))
    A[:N, :N] = D @ D
    A[N - 1, N] = 1.0
    A[N - 2, N + 1] = 1.0
    A[N, :N] = cheb_eval_row(N, -1.0)
    A[N + 1, :N] = cheb_eval_row(N, 1.0)
    rhs = np.zeros(N + 2)
    rhs[0] = -2.0
    sol = np.linalg.solve(A, rhs)
    z = cheb_grid(N, 0.0, 1.0)
    u = cheb_forward(np.eye(N))  # unused columns; evaluate through the backward map
    from oracle.tarang_oracle import cheb_backward

    ug = cheb_backward(sol[:N])
    assert np.abs(ug - z * (1 - z)).max() < 1e-14
    assert abs(sol[N]) < 1e-12 and abs(sol[N + 1]) < 1e-12


def test_rbc_builds_and_enforces_walls():
    p = RBCParams(Nx=16, Nz=8, Lx=4.0, Lz=1.0, Ra=1e4)
    sim = RBC2D(p)
    for m in (0, 3):
        M, L, bc, af = sim.mode_matrices(m)
        assert M.shape == L.shape == (sim.n_unknowns(m),) * 2
        assert len(bc) == (7 if m == 0 else 6)
    sim.set_b_grid(rbc_initial_b(p))
    for _ in range(5):
        sim.step(0.01, "RK222")
    bg = backward_2d(sim.b, p.Nx)
    uz = backward_2d(sim.uz, p.Nx)
    assert np.isfinite(bg).all() and np.isfinite(uz).all()
    assert np.abs(bg[0] - p.Lz).max() < 1e-8 and np.abs(bg[-1]).max() < 1e-8
    assert np.abs(uz[0]).max() < 1e-8 and np.abs(uz[-1]).max() < 1e-8


def test_mass_solve_is_min_norm_least_squares():
    p = RBCParams(Nx=8, Nz=8)
    sim = RBC2D(p)
    M = sim.dense_mode_matrices(2)[0]
    rhs = np.random.default_rng(0).standard_normal(M.shape[0]) + 0j
    want = np.linalg.lstsq(M, rhs, rcond=None)[0]
    assert np.allclose(sim.mass_solve(2, rhs), want, atol=1e-14)


def test_sparse_and_dense_tau_solves_agree():
    # batched-vs-per-mode parity analogue (test_mode_batch_parity.jl:411-455): 1e-12
    p = RBCParams(Nx=16, Nz=12, Ra=1e6)
    sim = RBC2D(p)
    rng = np.random.default_rng(1)
    for m in (0, 1, 8):
        M, L, _, _ = sim.dense_mode_matrices(m)
        A = M + 0.05 * L
        r = rng.standard_normal(A.shape[0]) + 1j * rng.standard_normal(A.shape[0])
        x_sparse = sim._lhs_lu(m, 1.0, 0.05).solve(r)
        x_dense = np.linalg.solve(A, r)
        assert rel_l2(x_sparse, x_dense) < 1e-12


def _diffusion_error(scheme, dt, T=0.4):
    # Horizontally uniform b: no flow develops and b diffuses exactly,
    # b = Lz - z + A exp(-kappa pi^2 t) sin(pi z), Lz = 1.
    p = RBCParams(Nx=8, Nz=24, Lx=4.0, Lz=1.0, Ra=25.0, Pr=1.0)
    sim = RBC2D(p)
    z = cheb_grid(p.Nz, 0.0, 1.0)
    A = 0.3
    g = np.repeat(((1 - z) + A * np.sin(np.pi * z))[:, None], p.Nx, axis=1)
    sim.set_b_grid(g)
    n = int(round(T / dt))
    for _ in range(n):
        sim.step(dt, scheme)
    exact = (1 - z) + A * np.exp(-p.kappa * np.pi**2 * n * dt) * np.sin(np.pi * z)
    return np.abs(backward_2d(sim.b, p.Nx)[:, 0] - exact).max()


@pytest.mark.parametrize("scheme,order", [("RK222", 2), ("RK443", 3), ("SBDF2", 2)])
def test_timestepper_order_on_exact_diffusion(scheme, order):
    e1 = _diffusion_error(scheme, 0.1)
    e2 = _diffusion_error(scheme, 0.05)
    rate = np.log2(e1 / e2)
    assert rate > order - 0.3, (scheme, e1, e2, rate)


def test_reference_pin_variable_step_sbdf_coefficients():
    # test/test_timestepper_boundaries.jl "Variable timestep coefficient
    # builders": dt = 0.02 after dt_prev = 0.01 (w1 = 2)
    from oracle.tarang_oracle import sbdf_coefs

    dt, dt_prev = 0.02, 0.01
    w1 = dt / dt_prev
    a, b, c = sbdf_coefs(2, dt, dt_prev)
    assert abs(a[0] - (1.0 + 2.0 * w1) / ((1.0 + w1) * dt)) < 1e-14
    assert abs(a[1] - (-(1.0 + w1) / dt)) < 1e-14
    assert abs(a[2] - w1 ** 2 / ((1.0 + w1) * dt)) < 1e-14
    assert tuple(b) == (1.0,) and tuple(c) == (0.0, 1.0 + w1, -w1)
    # the SBDF1 startup: (1/dt, -1/dt), (1,), (0, 1)
    a1, b1, c1 = sbdf_coefs(1, dt)
    assert tuple(a1) == (1.0 / dt, -1.0 / dt) and tuple(b1) == (1.0,) and tuple(c1) == (0.0, 1.0)


def _redft00(x):
    # FFTW's REDFT00 written out: Y_k = x_0 + (-1)^k x_{n-1}
    #                                   + 2 sum_{j=1}^{n-2} x_j cos(pi j k/(n-1))
    n = x.shape[0]
    j = np.arange(n)
    C = 2.0 * np.cos(np.pi * np.outer(j, j) / (n - 1))
    C[:, 0] = 1.0
    C[:, -1] = (-1.0) ** j
    return C @ x


@pytest.mark.parametrize("n", [9, 16])
def test_reference_pin_dct1_convention(n):
    # test/test_gpu_dct1_kernels_cpu.jl:35-50,88-106: forward = REDFT00/(n-1),
    # endpoints halved, odd coefficients negated; backward undoes it
    from oracle.tarang_oracle import cheb_backward, cheb_forward

    rng = np.random.default_rng(n)
    mat = rng.standard_normal((n, 5))
    sign = np.where(np.arange(n) % 2 == 0, 1.0, -1.0)[:, None]
    want = _redft00(mat) / (n - 1)
    want[0] /= 2
    want[-1] /= 2
    want *= sign
    fwd = cheb_forward(mat)
    assert np.abs(fwd - want).max() < 1e-13
    y = fwd * sign
    y[0] *= 2
    y[-1] *= 2
    assert np.abs(cheb_backward(fwd) - _redft00(y) / 2).max() < 1e-12
    assert np.abs(cheb_backward(fwd) - mat).max() < 1e-12


def test_reference_pin_fourier_chebyshev_forward_chain():
    # test/test_gpu_dct1_kernels_cpu.jl:187-214: the 2D RealFourier x
    # ChebyshevT forward is the unnormalised rfft along x, then the DCT-I
    # convention along z (16 x 9 grid); both stages written out as matrices
    from oracle.tarang_oracle import forward_2d

    Nx, Nz = 16, 9
    g = np.random.default_rng(9).standard_normal((Nz, Nx))
    k = np.arange(Nx // 2 + 1)
    F = np.exp(-2j * np.pi * np.outer(np.arange(Nx), k) / Nx)
    spec = g @ F
    sign = np.where(np.arange(Nz) % 2 == 0, 1.0, -1.0)[:, None]
    want = _redft00(spec) / (Nz - 1)
    want[0] /= 2
    want[-1] /= 2
    want *= sign
    assert np.abs(forward_2d(g) - want).max() < 1e-12


def _c2r(h, Nx):
    # FFTW's c2r along the last axis, written out: the imaginary parts of the
    # kx = 0 and Nyquist bins do not enter (transform_fourier.jl:553-575)
    x = np.arange(Nx)
    k = np.arange(1, Nx // 2)
    E = np.exp(2j * np.pi * np.outer(k, x) / Nx)
    g = h[..., :1].real + h[..., Nx // 2:Nx // 2 + 1].real * (-1.0) ** x
    return (g + 2.0 * np.real(h[..., 1:Nx // 2] @ E)) / Nx


def test_periodic_and_3d_transforms_written_out():
    # the doubly periodic (rfft x, fft y) and the 3D channel (rfft x, fft y,
    # DCT-I z) conventions as explicit DFT sums (transform_fourier.jl:473-590)
    from oracle.tarang_oracle import backward_3d, cheb_backward, forward_3d, turb_backward, turb_forward

    rng = np.random.default_rng(11)
    Nx, Ny, Nz = 12, 8, 9
    Fx = np.exp(-2j * np.pi * np.outer(np.arange(Nx), np.arange(Nx // 2 + 1)) / Nx)
    Fy = np.exp(-2j * np.pi * np.outer(np.arange(Ny), np.arange(Ny)) / Ny)
    g2 = rng.standard_normal((Ny, Nx))
    assert np.abs(turb_forward(g2) - Fy.T @ (g2 @ Fx)).max() < 1e-12
    c2 = rng.standard_normal((Ny, Nx // 2 + 1)) + 1j * rng.standard_normal((Ny, Nx // 2 + 1))
    assert np.abs(turb_backward(c2, Nx) - _c2r(np.conj(Fy) @ c2 / Ny, Nx)).max() < 1e-12

    g3 = rng.standard_normal((Nz, Ny, Nx))
    spec = np.einsum("yq,zqk->zyk", Fy.T, g3 @ Fx)
    sign = np.where(np.arange(Nz) % 2 == 0, 1.0, -1.0)[:, None, None]
    want = np.tensordot(_redft00(np.eye(Nz)), spec, axes=(1, 0)) / (Nz - 1)
    want[0] /= 2
    want[-1] /= 2
    want *= sign
    assert np.abs(forward_3d(g3) - want).max() < 1e-11
    assert np.abs(backward_3d(forward_3d(g3), Nx) - g3).max() < 1e-12
    c3 = rng.standard_normal(want.shape) + 1j * rng.standard_normal(want.shape)
    h = np.einsum("yq,zqk->zyk", np.conj(Fy) / Ny, cheb_backward(c3, axis=0))
    assert np.abs(backward_3d(c3, Nx) - _c2r(h, Nx)).max() < 1e-12


@pytest.mark.parametrize("n", [9, 17])
def test_reference_pin_chebyshev_derivative_recurrence(n):
    # test/test_gpu_dct1_kernels_cpu.jl:164-180: the T-basis derivative with
    # scale 2/3.7, and order 2 as the first-derivative pass applied twice.
    # Backward recurrence d_{k-1} = d_{k+1} + 2 k c_k, d_0 halved.
    scale = 2.0 / 3.7
    c = np.random.default_rng(n).standard_normal((n, 4))
    d = np.zeros_like(c)
    for k in range(n - 1, 0, -1):
        d[k - 1] = (d[k + 1] if k + 1 < n else 0.0) + 2.0 * k * c[k]
    d[0] /= 2.0
    d *= scale
    D = cheb_diff_matrix(n, 3.7)
    assert np.abs(D @ c - d).max() < 1e-11
    assert np.abs(D @ (D @ c) - D @ d).max() < 1e-9
    assert np.abs(npc.chebder(c, scl=scale) - (D @ c)[:-1]).max() < 1e-11


def test_reference_pin_wavenumbers():
    # test/test_basis_wavenumbers.jl:36-69: rfft layout 0..N/2 (N = 7 gives
    # 0..3), the length scaling 2 pi / L, and the full fft order of the y axis
    # with -N/2 at the Nyquist index
    from oracle.tarang_oracle import turb_wavenumbers, wavenumbers_rfft

    assert np.allclose(wavenumbers_rfft(8, 2 * np.pi), [0, 1, 2, 3, 4])
    assert np.allclose(wavenumbers_rfft(7, 2 * np.pi), [0, 1, 2, 3])
    assert np.allclose(wavenumbers_rfft(8, 4 * np.pi), 0.5 * np.arange(5))
    kx, ky = turb_wavenumbers(16, 8, 2 * np.pi, 2 * np.pi)
    assert np.allclose(ky.ravel(), [0, 1, 2, 3, -4, -3, -2, -1])
    assert np.allclose(kx.ravel(), np.arange(9)) and kx.ravel()[-1] == 8.0
