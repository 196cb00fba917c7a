"""Checkpoints through the C ABI: a run restarted from a saved file continues
like the uninterrupted run whose state went through the same grid round trip
(the saved grid fields drop the non-Hermitian part of the Nyquist modes, as
the reference's grid-space save_state does; RK steppers carry no history),
the clock is restored, and staging overlaps further steps without seeing
them."""
import numpy as np
import pytest

from oracle.tarang_oracle import (RBC3Params, RBCParams, backward_2d, backward_3d, forward_2d, forward_3d,
                                  rbc3_initial_b, rbc_initial_b, rel_l2)

pytestmark = pytest.mark.gpu


def test_restart_2d_continues_the_run(tb, tmp_path):
    p = RBCParams(Nx=48, Nz=24, Lx=4.0, Lz=1.0, Ra=1e8)
    dom = tb.ChannelDomain(48, 24, Lx=4.0, Lz=1.0)
    a = tb.Plan(dom, p.kappa, p.nu, 1.0, 0.0, 1)
    a.set_state(0, forward_2d(rbc_initial_b(p, 42)))
    a.step(0.01, 3)
    path = str(tmp_path / "rbc.nc")
    a.save_state(path)
    b = tb.Plan(dom, p.kappa, p.nu, 1.0, 0.0, 1)
    b.load_state(path)
    assert abs(b.sim_time() - a.sim_time()) < 1e-15
    # the saved grid is the state's grid
    from tarang_b200.checkpoint import read_checkpoint

    data, clock = read_checkpoint(path, ("b", "ux", "uz", "p"))
    assert clock[1] == 3 and abs(clock[2] - 0.01) < 1e-15
    assert rel_l2(data[0], backward_2d(a.get_state(0), 48)) < 1e-13
    for f in (0, 1, 2, 3):  # the uninterrupted run, through the same grid round trip
        a.set_state(f, forward_2d(backward_2d(a.get_state(f), 48)))
    a.step(0.01, 3)
    b.step(0.01, 3)
    for f in (0, 1, 2):
        assert rel_l2(b.get_state(f), a.get_state(f)) < 1e-11


def test_restart_3d_continues_the_run(tb, tmp_path):
    p = RBC3Params(Nx=16, Ny=12, Nz=12, Lx=4.0, Ly=3.0, Ra=1e6)
    a = tb.Plan3D(16, 12, 12, p.kappa, p.nu, 0, 4.0, 3.0, 1.0)
    a.set_state(0, a.forward(rbc3_initial_b(p, 42, amp=1e-2)))
    a.step(0.02, 2)
    path = str(tmp_path / "rbc3.nc")
    a.save_state(path)
    b = tb.Plan3D(16, 12, 12, p.kappa, p.nu, 0, 4.0, 3.0, 1.0)
    b.load_state(path)
    for f in (0, 1, 5, 2, 3):
        a.set_state(f, forward_3d(backward_3d(a.get_state(f), 16)))
    a.step(0.02, 2)
    b.step(0.02, 2)
    for f in (0, 1, 5, 2):
        assert rel_l2(b.get_state(f), a.get_state(f)) < 1e-11


def test_staging_overlaps_later_steps(tb):
    import ctypes

    p = RBCParams(Nx=64, Nz=32, Ra=1e6)
    dom = tb.ChannelDomain(64, 32, Lx=4.0, Lz=1.0)
    a = tb.Plan(dom, p.kappa, p.nu, 1.0, 0.0, 0)
    a.set_state(0, forward_2d(rbc_initial_b(p, 1)))
    a.step(0.05, 2)
    want = backward_2d(a.get_state(0), 64)
    host = np.empty((4, 32, 64))
    clock = np.zeros(3)
    tb._lib.check(tb.lib.tb_checkpoint_stage(a.ptr, host.ctypes.data_as(ctypes.c_void_p), host.size,
                                             clock.ctypes.data_as(ctypes.c_void_p)), a.ctx)
    a.step(0.05, 3)  # steps on while the copy drains
    tb._lib.check(tb.lib.tb_checkpoint_wait(a.ptr), a.ctx)
    assert rel_l2(host[0], want) < 1e-13 and clock[1] == 2
