"""Mixed precision on the tcgen05 tensor cores: the FP32 Chebyshev transform
GEMMs in TF32 with three products per term.  The tensor-core path and the SIMT
FP32 path agree to FP32 rounding, both match the FP64 oracle at the mixed
form's 1e-6 bar over several steps, and shapes beyond the tensor-core tile
(Nz > 256) fall back to the SIMT kernel with the same results."""
import numpy as np
import pytest

from oracle.tarang_oracle import RBCParams, RBC2D, forward_2d, rbc_initial_b, rel_l2, run_rbc

pytestmark = pytest.mark.gpu

TS = {"RK222": 0, "RK443": 1, "SBDF2": 3}


def _mixed_plan(tb, Nx, Nz, Ra, scheme, tensor_cores):
    p = RBCParams(Nx=Nx, Nz=Nz, Lx=4.0, Lz=1.0, Ra=Ra)
    dom = tb.ChannelDomain(Nx, Nz, Lx=4.0, Lz=1.0)
    plan = tb.Plan(dom, p.kappa, p.nu, 1.0, 0.0, TS[scheme], precision=tb._lib.TB_PREC_MIXED)
    plan.set_gemm_path(tensor_cores)
    assert plan.gemm_path() == tensor_cores
    return p, plan


@pytest.mark.parametrize("Nx,Nz", [(96, 24), (64, 17), (1024, 256), (48, 9)])
def test_tensor_core_rhs_matches_simt_and_oracle(tb, Nx, Nz):
    rng = np.random.default_rng(4)
    ins = [forward_2d(rng.standard_normal((Nz, Nx))) for _ in range(3)]
    outs = {}
    for tc in (True, False):
        _, plan = _mixed_plan(tb, Nx, Nz, 1e6, "RK222", tc)
        outs[tc] = plan.rhs_advection(*ins)
    ref = RBC2D(RBCParams(Nx=Nx, Nz=Nz, Lx=4.0, Lz=1.0)).rhs(*ins)
    for a, b, r in zip(outs[True], outs[False], ref):
        assert rel_l2(a, b) < 1e-5  # both FP32-accurate; different summation orders
        assert rel_l2(a, r) < 1e-5
        assert rel_l2(b, r) < 1e-5


@pytest.mark.parametrize("Nx,Nz,Ra,scheme,dt,n", [
    (48, 24, 1e8, "RK443", 0.01, 10),
    (64, 32, 2e6, "RK222", 0.05, 10),
    (32, 16, 1e8, "SBDF2", 0.01, 10),
    (256, 64, 2e6, "RK222", 0.125, 20),
])
def test_tensor_core_steps_match_oracle(tb, Nx, Nz, Ra, scheme, dt, n):
    p, plan = _mixed_plan(tb, Nx, Nz, Ra, scheme, True)
    plan.set_state(0, forward_2d(rbc_initial_b(p, 42)))
    plan.step(dt, n)
    sim = run_rbc(p, scheme, dt, n, seed=42)
    for f, want in zip(range(3), (sim.b, sim.ux, sim.uz)):
        assert rel_l2(plan.get_state(f), want) < 1e-6


def test_beyond_the_tensor_core_tile_falls_back(tb):
    # Nz = 288: 144 rows per parity half, more than the 128-row MMA tile
    Nx, Nz = 32, 288
    rng = np.random.default_rng(8)
    ins = [forward_2d(rng.standard_normal((Nz, Nx))) for _ in range(3)]
    outs = {}
    for tc in (True, False):
        _, plan = _mixed_plan(tb, Nx, Nz, 1e6, "RK222", tc)
        outs[tc] = plan.rhs_advection(*ins)
    for a, b in zip(outs[True], outs[False]):
        assert np.array_equal(a, b)  # the same SIMT kernel ran


def _plan3(tb, Nx, Ny, Nz, tensor_cores):
    from oracle.tarang_oracle import RBC3Params, rbc3_initial_b

    p = RBC3Params(Nx=Nx, Ny=Ny, Nz=Nz, Lx=4.0, Ly=4.0, Lz=1.0, Ra=1e7)
    plan = tb.Plan3D(Nx, Ny, Nz, p.kappa, p.nu, TS["RK222"], 4.0, 4.0, 1.0, precision=tb._lib.TB_PREC_MIXED)
    plan.set_gemm_path(tensor_cores)
    plan.set_state(tb._lib.TB_FIELD_B, plan.forward(rbc3_initial_b(p, 42, amp=1e-2)))
    return plan


@pytest.mark.parametrize("Nx,Ny,Nz", [(128, 96, 64), (64, 64, 128)])
def test_3d_streaming_tensor_cores_match_simt(tb, Nx, Ny, Nz):
    # many (field, 32-column tile) tasks per persistent CTA (12480 and 4224
    # columns), the largest supported Nz; both paths are FP32-accurate
    plans = {tc: _plan3(tb, Nx, Ny, Nz, tc) for tc in (True, False)}
    for pl in plans.values():
        pl.step(0.005, 3)
    for f in (0, 1, 2, 5):
        a, b = plans[True].get_state(f), plans[False].get_state(f)
        assert np.isfinite(a).all()
        assert rel_l2(a, b) < 1e-6, f


def test_3d_beyond_the_streaming_tile_falls_back(tb):
    # Nz = 136 > 128 rows per tile: the SIMT kernel runs
    plans = {tc: _plan3(tb, 8, 8, 136, tc) for tc in (True, False)}
    for pl in plans.values():
        pl.step(0.001, 2)
    for f in (0, 1, 2, 5):
        assert np.array_equal(plans[True].get_state(f), plans[False].get_state(f))
