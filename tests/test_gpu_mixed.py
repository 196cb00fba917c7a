"""Mixed precision (TB_PREC_MIXED): FP32 transforms and products, FP64 tau LU,
solves and stage algebra.  The bar is the mixed form's: 1e-6 relative L2 of
every field against the FP64 oracle."""
import numpy as np
import pytest

from oracle.tarang_oracle import RBCParams, forward_2d, rbc_initial_b, rel_l2, run_rbc

pytestmark = pytest.mark.gpu

TS = {"RK222": 0, "RK443": 1, "SBDF1": 2, "SBDF2": 3}


@pytest.mark.parametrize("Nx,Nz,Ra,scheme,dt,n", [
    (48, 24, 1e8, "RK443", 0.01, 10),
    (64, 32, 2e6, "RK222", 0.05, 10),
    (32, 16, 1e8, "SBDF2", 0.01, 10),
])
def test_mixed_matches_oracle(tb, Nx, Nz, Ra, scheme, dt, n):
    p = RBCParams(Nx=Nx, Nz=Nz, Lx=4.0, Lz=1.0, Ra=Ra)
    dom = tb.ChannelDomain(Nx, Nz, Lx=4.0, Lz=1.0)
    plan = tb.Plan(dom, p.kappa, p.nu, 1.0, 0.0, TS[scheme], precision=tb._lib.TB_PREC_MIXED)
    plan.set_state(0, forward_2d(rbc_initial_b(p, 42)))
    plan.step(dt, n)
    sim = run_rbc(p, scheme, dt, n, seed=42)
    for f, want in zip(range(3), (sim.b, sim.ux, sim.uz)):
        assert rel_l2(plan.get_state(f), want) < 1e-6


def test_mixed_rhs_close_to_f64(tb):
    Nx, Nz = 96, 24
    p = RBCParams(Nx=Nx, Nz=Nz)
    dom = tb.ChannelDomain(Nx, Nz)
    a = tb.Plan(dom, p.kappa, p.nu, 1.0, 0.0, 0)
    b = tb.Plan(dom, p.kappa, p.nu, 1.0, 0.0, 0, precision=tb._lib.TB_PREC_MIXED)
    rng = np.random.default_rng(1)
    ins = [forward_2d(rng.standard_normal((Nz, Nx))) for _ in range(3)]
    ra, rb = a.rhs_advection(*ins), b.rhs_advection(*ins)
    for x, y in zip(ra, rb):
        assert rel_l2(y, x) < 1e-5  # single-precision products of O(1) random fields
