"""Host-side checks that need no GPU: the C ABI library loads and exports every
symbol include/tarang_b200.h declares, the plan compiler's banded layout, the
API mirror's equation recogniser and the benchmark byte model."""
import ctypes
import os
import re

import pytest

from __graft_entry__ import ROOT


def header_functions():
    src = open(os.path.join(ROOT, "include", "tarang_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(tb_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_header_symbol(tb):
    names = header_functions()
    assert len(names) >= 20
    lib = ctypes.CDLL(os.path.join(ROOT, "tarang.jl_b200", "libtarang_b200.so"))
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # and the Python binding declares a signature for each
    assert sorted(tb._lib.SIGNATURES) == names


def test_status_strings_and_version(tb):
    lib = tb.lib
    assert lib.tb_version() >= 1
    assert lib.tb_status_string(0) == b"ok"
    assert lib.tb_status_string(3) == b"singular tau system"
    assert lib.tb_status_string(99) == b"unknown status"


def test_no_gpu_is_an_error_not_a_crash(tb):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    ctx = ctypes.c_void_p()
    assert tb.lib.tb_context_create(0, ctypes.byref(ctx)) == tb._lib.TB_ECUDA
    assert tb.lib.tb_last_error(None)


@pytest.mark.parametrize("Nz", [8, 9, 16, 17, 64, 256])
def test_tau_layout_is_bordered_banded(tb, Nz):
    for cls in (0, 1):
        info = (ctypes.c_int * 4)()
        assert tb.lib.tb_tau_layout_query(Nz, 4.0, 1.0, cls, info) == 0
        n, nb, kl, ku = list(info)
        assert n == 2 * Nz  # bulk rows of the parity class
        assert nb == (3 if cls == 0 else 4)  # boundary rows incl. integ(p)/tau_p pin
        assert kl <= 4 and ku <= 8


def test_tau_layout_rejects_bad_sizes(tb):
    info = (ctypes.c_int * 4)()
    assert tb.lib.tb_tau_layout_query(4, 4.0, 1.0, 0, info) == tb._lib.TB_EINVAL
    assert tb.lib.tb_tau_layout_query(64, -1.0, 1.0, 0, info) == tb._lib.TB_EINVAL
    assert tb.lib.tb_tau_layout_query(64, 4.0, 1.0, 2, info) == tb._lib.TB_EINVAL


def _rbc_problem(tb, extra_eq=None):
    dom = tb.api.Domain((tb.RealFourier("x", 16, (0, 4.0), 1.5), tb.ChebyshevT("z", 8, (0, 1.0), 1.5)))
    p, b = tb.ScalarField(dom, "p"), tb.ScalarField(dom, "b")
    u = tb.VectorField(dom, "u")
    problem = tb.IVP([p, b, u])
    tb.add_parameters(problem, kappa=1e-3, nu=2e-3, Lz=1.0)
    tb.add_equation(problem, "trace(grad_u) + tau_p = 0")
    tb.add_equation(problem, "∂t(b) - kappa*div(grad_b) + τ_lift(tau_b2) = -u⋅∇(b)")
    tb.add_equation(problem, "∂t(u) - nu*div(grad_u) + ∇(p) - b*ez + τ_lift(tau_u2) = -u⋅∇(u)")
    if extra_eq:
        tb.add_equation(problem, extra_eq)
    for bc in ("b(z=0) = Lz", "u(z=0) = 0", "b(z=Lz) = 0", "u(z=Lz) = 0", "integ(p) = 0"):
        tb.add_bc(problem, bc)
    return problem


def test_equation_recogniser_reads_the_reference_rbc_strings(tb):
    spec = tb.api._match_boussinesq(_rbc_problem(tb))
    assert spec["kappa"] == 1e-3 and spec["nu"] == 2e-3
    assert spec["b_bottom"] == 1.0 and spec["b_top"] == 0.0
    assert spec["names"] == {"b": "b", "u": "u", "p": "p"}


def test_equation_recogniser_refuses_other_systems(tb):
    with pytest.raises(NotImplementedError):
        tb.api._match_boussinesq(_rbc_problem(tb, extra_eq="∂t(c) - kappa*lap(c) = 0"))
    problem = _rbc_problem(tb)
    problem.bcs[1] = "u(z=0) = 1"
    with pytest.raises(NotImplementedError):
        tb.api._match_boussinesq(problem)


def _vorticity_problem(tb, nu_eq="∂t(q) - nu*Δ(q) = -u⋅∇(q)", bcs=("integ(psi) = 0",)):
    dom = tb.PeriodicDomain(16, 16)
    q, psi = tb.ScalarField(dom, "q"), tb.ScalarField(dom, "psi")
    u = tb.VectorField(dom, "u")
    tau = tb.ScalarField(dom, "tau_psi", bases=())
    problem = tb.IVP([q, psi, u, tau])
    tb.add_parameters(problem, nu=1e-4)
    tb.add_equation(problem, nu_eq)
    tb.add_equation(problem, "Δ(psi) + tau_psi - q = 0")
    tb.add_equation(problem, "u - skew(grad(psi)) = 0")
    for bc in bcs:
        tb.add_bc(problem, bc)
    return problem, dom, u, tau


def test_vorticity_recogniser_reads_the_reference_example_strings(tb):
    # the equations of examples/2d_decaying_turbulence_gpu.jl, on a domain
    # whose field shapes follow the periodic coefficient layout
    problem, dom, u, tau = _vorticity_problem(tb)
    spec = tb.api._match_vorticity(problem)
    assert spec["nu"] == 1e-4
    assert spec["names"] == {"q": "q", "psi": "psi", "u": "u", "tau": "tau_psi"}
    assert dom.periodic and dom.coeff_shape() == (16, 9) and dom.grid_shape() == (16, 16)
    assert [c.name for c in u.components] == ["u_x", "u_y"] and tau._coeff.shape == ()


def test_vorticity_recogniser_refuses_other_systems(tb):
    with pytest.raises(NotImplementedError):
        tb.api._match_vorticity(_vorticity_problem(tb, nu_eq="∂t(q) - nu*Δ(Δ(q)) = -u⋅∇(q)")[0])
    with pytest.raises(NotImplementedError):
        tb.api._match_vorticity(_vorticity_problem(tb, bcs=())[0])


def test_periodic_solver_needs_a_diagonal_stepper(tb):
    # a ChebyshevT stepper on a periodic problem is refused before any GPU work
    problem = _vorticity_problem(tb)[0]
    with pytest.raises(NotImplementedError):
        tb.InitialValueSolver(problem, tb.RK222(), dt=1e-3)


def test_cpu_architecture_is_refused(tb):
    with pytest.raises(NotImplementedError):
        tb.ChannelDomain(16, 8, arch=tb.CPU())


def test_byte_model_matches_the_measurement_plan(tb):
    from tarang_b200 import workloads as W

    assert W.step_model_bytes(W.C1, "RK222") / 1e6 == pytest.approx(129.9, rel=2e-3)
    assert W.step_model_bytes(W.C2, "RK443") / 1e9 == pytest.approx(3.03, rel=2e-3)
    assert W.step_model_bytes(W.C2, "RK222") / 1e9 == pytest.approx(2.03, rel=2e-3)
    assert W.step_model_bytes(W.C2, "SBDF2") / 1e9 == pytest.approx(1.01, rel=2e-3)


def test_initial_condition_matches_the_oracle(tb):
    import numpy as np

    from oracle.tarang_oracle import RBCParams, rbc_initial_b
    from tarang_b200 import workloads as W

    cfg = W.RBCConfig(Nx=32, Nz=16, Ra=2e6)
    p = RBCParams(Nx=32, Nz=16, Ra=2e6)
    assert np.array_equal(W.rbc_initial_grid(cfg), rbc_initial_b(p, 42))
