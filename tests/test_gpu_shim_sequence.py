"""The Julia extension's call sequence, made through the C ABI with ctypes.

Julia is not installed here, so the ABI calls of ext/TarangB200Ext.jl (as
written out in INTEGRATION.md) are replayed in the same order, with CUDA
buffers in the field's coefficient layout standing in for the CuArrays:

  build:     tb_context_create, tb_plan_create (the Boussinesq descriptor)
  per step:  tb_set_states(b, u_x, u_z, p, taus; TB_DEVICE | TB_KEEP_HISTORY)
             tb_step(dt, 1)
             tb_get_states(b, u_x, u_z, p, taus; TB_DEVICE)

The state after the steps must equal the oracle's (1e-10) and, bit for bit,
the state of a plan stepped the same number of steps without the per-step
round trips; SBDF2 checks that the write-back keeps the multistep history.
"""
import ctypes

import numpy as np
import pytest

from oracle.tarang_oracle import RBCParams, forward_2d, rbc_initial_b, rel_l2, run_rbc

pytestmark = pytest.mark.gpu


def _desc(L, p, ts):
    d = L.tb_problem_desc()
    d.ndim, d.Nx, d.Ny, d.Nz = 2, p.Nx, 1, p.Nz
    d.Lx, d.Ly, d.Lz, d.dealias = p.Lx, 1.0, p.Lz, 1.5
    d.precision, d.timestepper, d.program = L.TB_PREC_F64, ts, L.TB_PROGRAM_RBC
    d.kappa, d.nu, d.b_bottom, d.b_top = p.kappa, p.nu, p.Lz, 0.0
    return d


@pytest.mark.parametrize("scheme,ts", [("RK443", 1), ("SBDF2", 3)])
def test_shim_call_sequence_matches_oracle_and_plain_stepping(tb, scheme, ts):
    import torch

    L, lib = tb._lib, tb.lib
    p = RBCParams(Nx=64, Nz=32, Lx=4.0, Lz=1.0, Ra=1e7)
    dt, nsteps = 0.01, 6
    ctx = ctypes.c_void_p()
    assert lib.tb_context_create(0, ctypes.byref(ctx)) == 0
    plan, plain = ctypes.c_void_p(), ctypes.c_void_p()
    d = _desc(L, p, ts)
    assert lib.tb_plan_create(ctx, ctypes.byref(d), ctypes.byref(plan)) == 0, lib.tb_last_error(ctx)
    assert lib.tb_plan_create(ctx, ctypes.byref(d), ctypes.byref(plain)) == 0, lib.tb_last_error(ctx)
    try:
        nk = p.Nx // 2 + 1
        # the fields' coefficient arrays on the device (one allocation each, as CuArrays are)
        b0 = forward_2d(rbc_initial_b(p, 42))
        dev = {f: torch.zeros((p.Nz, nk), dtype=torch.complex128, device="cuda")
               for f in (L.TB_FIELD_B, L.TB_FIELD_UX, L.TB_FIELD_UZ, L.TB_FIELD_P)}
        dev[L.TB_FIELD_B].copy_(torch.from_numpy(b0))
        dev[L.TB_FIELD_TAU] = torch.zeros((7, nk), dtype=torch.complex128, device="cuda")
        sel = (ctypes.c_int * 5)(L.TB_FIELD_B, L.TB_FIELD_UX, L.TB_FIELD_UZ, L.TB_FIELD_P, L.TB_FIELD_TAU)
        ptrs = (ctypes.c_void_p * 5)(*[dev[f].data_ptr() for f in sel])
        for _ in range(nsteps):
            torch.cuda.synchronize()  # the shim's CUDA.synchronize(): the task stream wrote the fields
            assert lib.tb_set_states(plan, 5, sel, ptrs, L.TB_DEVICE | L.TB_KEEP_HISTORY) == 0, lib.tb_last_error(ctx)
            assert lib.tb_step(plan, dt, 1) == 0, lib.tb_last_error(ctx)
            assert lib.tb_get_states(plan, 5, sel, ptrs, L.TB_DEVICE) == 0, lib.tb_last_error(ctx)
        # the same steps without the round trips
        assert lib.tb_set_state(plain, L.TB_FIELD_B, b0.ctypes.data_as(ctypes.c_void_p), L.TB_HOST) == 0
        assert lib.tb_step(plain, dt, nsteps) == 0, lib.tb_last_error(ctx)
        ref = run_rbc(p, scheme, dt, nsteps, seed=42)
        for f, want in ((L.TB_FIELD_B, ref.b), (L.TB_FIELD_UX, ref.ux), (L.TB_FIELD_UZ, ref.uz)):
            got = dev[f].cpu().numpy()
            alone = np.empty_like(got)
            assert lib.tb_get_state(plain, f, alone.ctypes.data_as(ctypes.c_void_p), L.TB_HOST) == 0
            assert np.array_equal(got, alone), (f, np.abs(got - alone).max())
            assert rel_l2(got, want) < 1e-10, f
    finally:
        lib.tb_plan_destroy(plan)
        lib.tb_plan_destroy(plain)
        lib.tb_context_destroy(ctx)


def test_plain_state_write_restarts_sbdf_history(tb):
    # without TB_KEEP_HISTORY a write restarts SBDF2 at SBDF1 (documented);
    # the sequence above relies on the flag to keep it
    L = tb._lib
    p = RBCParams(Nx=32, Nz=16, Lx=4.0, Lz=1.0, Ra=1e7)
    plans = []
    for keep in (True, False):
        dom = tb.ChannelDomain(p.Nx, p.Nz, Lx=p.Lx, Lz=p.Lz)
        pl = tb.Plan(dom, p.kappa, p.nu, p.Lz, 0.0, 3)
        pl.set_state(0, forward_2d(rbc_initial_b(p, 42)))
        pl.step(0.01, 2)
        b = pl.get_state(0)
        where = L.TB_HOST | (L.TB_KEEP_HISTORY if keep else 0)
        assert tb.lib.tb_set_state(pl.ptr, 0, b.ctypes.data_as(ctypes.c_void_p), where) == 0
        pl.step(0.01, 2)
        plans.append(pl.get_state(2))
    ref = run_rbc(p, "SBDF2", 0.01, 4, seed=42)
    assert rel_l2(plans[0], ref.uz) < 1e-10
    assert rel_l2(plans[1], ref.uz) > 1e-6  # the restarted run took an SBDF1 step
