"""3D Rayleigh-Benard (RealFourier x, RealFourier y, ChebyshevT z) through the
C ABI against the 3D oracle: the FP64 plan to 1e-10 relative L2 of every
field, the mixed plan (FP32 transforms and products, FP64 tau solves) to 1e-6."""
import numpy as np
import pytest

from oracle.tarang_oracle import RBC3D, TABLEAUS, RBC3Params, backward_3d, forward_3d, rbc3_initial_b, rel_l2

pytestmark = pytest.mark.gpu

TS = {"RK222": 0, "RK443": 1}

CASES = [
    # Nx, Ny, Nz, Lx, Ly, Ra, scheme, dt, steps
    (16, 12, 16, 4.0, 3.0, 1e5, "RK222", 0.05, 4),
    (12, 16, 12, 3.0, 4.0, 1e6, "RK443", 0.02, 3),
    (24, 24, 20, 4.0, 4.0, 1e7, "RK222", 0.005, 3),
    # 2376 modes: enough mode groups that the tau solves run one warp per group
    (64, 72, 8, 4.0, 4.0, 1e6, "RK222", 0.02, 2),
    # 384-point padded x / y transforms (the compiled plans of the 256-point grids)
    (256, 8, 8, 4.0, 4.0, 1e6, "RK222", 0.01, 2),
    (8, 256, 8, 4.0, 4.0, 1e6, "RK222", 0.01, 2),
]


def _run(tb, case, precision, seed=42, tensor_cores=False):
    Nx, Ny, Nz, Lx, Ly, Ra, scheme, dt, n = case
    p = RBC3Params(Nx=Nx, Ny=Ny, Nz=Nz, Lx=Lx, Ly=Ly, Lz=1.0, Ra=Ra)
    plan = tb.Plan3D(Nx, Ny, Nz, p.kappa, p.nu, TS[scheme], Lx, Ly, 1.0, precision=precision)
    plan.set_gemm_path(tensor_cores)
    plan.set_state(tb._lib.TB_FIELD_B, plan.forward(rbc3_initial_b(p, seed, amp=1e-2)))
    plan.step(dt, n)
    sim = RBC3D(p)
    sim.set_b_grid(rbc3_initial_b(p, seed, amp=1e-2))
    for _ in range(n):
        sim.step_rk(dt, TABLEAUS[scheme])
    return plan, sim


FIELDS = [("b", 0), ("ux", 1), ("uy", 5), ("uz", 2)]


@pytest.mark.parametrize("case", CASES)
def test_rbc3d_f64_matches_oracle(tb, case):
    plan, sim = _run(tb, case, tb._lib.TB_PREC_F64)
    for name, f in FIELDS:
        got, want = plan.get_state(f), getattr(sim, name)
        assert np.abs(want).max() > 0
        assert rel_l2(got, want) < 1e-10, name
    assert np.abs(plan.get_state(tb._lib.TB_FIELD_P)).max() == 0.0  # zeroed by the final mass solve


@pytest.mark.parametrize("case", CASES[:2] + CASES[-2:])
def test_rbc3d_mixed_matches_oracle(tb, case):
    plan, sim = _run(tb, case, tb._lib.TB_PREC_MIXED)
    for name, f in FIELDS:
        assert rel_l2(plan.get_state(f), getattr(sim, name)) < 1e-6, name


@pytest.mark.parametrize("case", CASES[:2] + CASES[-3:])
def test_rbc3d_mixed_tensor_cores_match_oracle(tb, case):
    # the z transforms on the streaming tcgen05 kernel (TF32, three products
    # per term): partial 32-column tiles (216 and 224 columns), 2 to 150
    # tiles per field
    plan, sim = _run(tb, case, tb._lib.TB_PREC_MIXED, tensor_cores=True)
    assert plan.gemm_path()
    for name, f in FIELDS:
        assert rel_l2(plan.get_state(f), getattr(sim, name)) < 1e-6, name


def test_rbc3d_state_io_round_trip(tb):
    Nx, Ny, Nz = 12, 24, 10
    plan = tb.Plan3D(Nx, Ny, Nz, 1e-3, 1e-3)
    rng = np.random.default_rng(3)
    shape = (Nz, Ny, Nx // 2 + 1)
    fields = {f: rng.standard_normal(shape) + 1j * rng.standard_normal(shape) for f in (0, 1, 2, 3, 5)}
    for f, v in fields.items():
        plan.set_state(f, v)
    for f, v in fields.items():
        assert np.abs(plan.get_state(f) - v).max() < 1e-13 * np.abs(v).max()
    taus = rng.standard_normal((9, Ny, Nx // 2 + 1)) + 0j
    plan.set_state(tb._lib.TB_FIELD_TAU, taus)
    assert np.abs(plan.get_state(tb._lib.TB_FIELD_TAU) - taus).max() < 1e-13


def test_rbc3d_rejects_unsupported(tb):
    with pytest.raises(tb.TarangError):
        tb.Plan3D(16, 12, 15, 1e-3, 1e-3)  # odd Nz
    with pytest.raises(tb.TarangError):
        tb.Plan3D(16, 18, 16, 1e-3, 1e-3)  # padded Ny = 28 is not 2^a 3^b


def test_rbc3d_transforms_match_oracle(tb):
    Nx, Ny, Nz = 24, 16, 12
    plan = tb.Plan3D(Nx, Ny, Nz, 1e-3, 1e-3, Lx=3.0, Ly=2.0)
    g = np.random.default_rng(4).standard_normal((Nz, Ny, Nx))
    c = plan.forward(g)
    assert rel_l2(c, forward_3d(g)) < 1e-13
    assert rel_l2(plan.backward(c), g) < 1e-13
    c2 = forward_3d(g)
    c2[:, :, -1] += 0.5j  # non-Hermitian Nyquist content is dropped like FFTW's c2r
    assert rel_l2(plan.backward(c2), backward_3d(c2, Nx)) < 1e-13


@pytest.mark.parametrize("precision,tol", [(0, 1e-10), (1, 1e-6)])
def test_rbc3d_sbdf2_matches_oracle(tb, precision, tol):
    p = RBC3Params(Nx=16, Ny=12, Nz=12, Lx=4.0, Ly=3.0, Ra=1e6)
    sim = RBC3D(p)
    sim.set_b_grid(rbc3_initial_b(p, 42, amp=1e-2))
    for _ in range(4):
        sim.step(0.02, "SBDF2")
    plan = tb.Plan3D(16, 12, 12, p.kappa, p.nu, 3, 4.0, 3.0, 1.0, precision=precision)
    plan.set_state(0, plan.forward(rbc3_initial_b(p, 42, amp=1e-2)))
    plan.step(0.02, 4)
    for name, f in FIELDS:
        assert rel_l2(plan.get_state(f), getattr(sim, name)) < tol, name


def test_reference_style_3d_script(tb):
    # the 3D channel written against the mirror API as in the reference's
    # examples/ivp/rotating_rayleigh_benard_3d.jl (without rotation), against the oracle
    Lx, Ly, Lz, Nx, Ny, Nz, Ra = 4.0, 3.0, 1.0, 16, 12, 12, 1e5
    kappa, nu = Ra ** -0.5, Ra ** -0.5
    domain = tb.ChannelDomain3D(Nx, Ny, Nz, Lx=Lx, Ly=Ly, Lz=Lz, zbounds=(0.0, Lz))
    p = tb.ScalarField(domain, "p")
    b = tb.ScalarField(domain, "b")
    u = tb.VectorField(domain, "u")
    xy = (domain.xbasis, domain.ybasis)
    taus = [tb.ScalarField(domain, "tau_p", ()), tb.ScalarField(domain, "tau_b1", xy),
            tb.ScalarField(domain, "tau_b2", xy), tb.VectorField(domain, "tau_u1", xy),
            tb.VectorField(domain, "tau_u2", xy)]
    assert taus[1]["c"].shape == (Ny, Nx // 2 + 1) and len(u.components) == 3
    problem = tb.IVP([p, b, u] + taus)
    tb.add_parameters(problem, kappa=kappa, nu=nu, Lz=Lz)
    tb.add_equation(problem, "trace(grad_u) + tau_p = 0")
    tb.add_equation(problem, "∂t(b) - kappa*div(grad_b) + τ_lift(tau_b2) = -u⋅∇(b)")
    tb.add_equation(problem, "∂t(u) - nu*div(grad_u) + ∇(p) - b*ez + τ_lift(tau_u2) = -u⋅∇(u)")
    tb.add_bc(problem, "b(z=0) = Lz")
    tb.add_bc(problem, "u(z=0) = 0")
    tb.add_bc(problem, "b(z=Lz) = 0")
    tb.add_bc(problem, "u(z=Lz) = 0")
    tb.add_bc(problem, "integ(p) = 0")
    solver = tb.InitialValueSolver(problem, tb.RK222(), dt=0.02)
    rp = RBC3Params(Nx=Nx, Ny=Ny, Nz=Nz, Lx=Lx, Ly=Ly, Lz=Lz, Ra=Ra)
    b["g"] = rbc3_initial_b(rp, 42, amp=1e-2)
    tb.run(solver, stop_iteration=3)
    sim = RBC3D(rp)
    sim.set_b_grid(rbc3_initial_b(rp, 42, amp=1e-2))
    for _ in range(3):
        sim.step_rk(0.02, TABLEAUS["RK222"])
    assert solver.iteration == 3
    assert rel_l2(b["c"], sim.b) < 1e-10
    for comp, want in zip(u.components, (sim.ux, sim.uy, sim.uz)):
        assert rel_l2(comp["c"], want) < 1e-10
    assert b["g"].shape == (Nz, Ny, Nx)
