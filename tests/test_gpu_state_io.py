"""Multi-field state I/O (tb_set_states / tb_get_states): the same data and the
same steps as the per-field calls, one wait per call."""
import ctypes

import numpy as np
import pytest

from oracle.tarang_oracle import RBCParams, forward_2d, rbc_initial_b

pytestmark = pytest.mark.gpu

FIELDS = (0, 1, 2, 3, 4)  # b, ux, uz, p, taus


def _plan(tb, p):
    dom = tb.ChannelDomain(p.Nx, p.Nz, Lx=4.0, Lz=1.0)
    plan = tb.Plan(dom, p.kappa, p.nu, 1.0, 0.0, 1)
    plan.set_state(0, forward_2d(rbc_initial_b(p, 42)))
    plan.step(0.01, 3)
    return plan


def test_states_round_trip_and_step_like_single_fields(tb):
    p = RBCParams(Nx=64, Nz=32, Lx=4.0, Lz=1.0, Ra=1e7)
    a, b = _plan(tb, p), _plan(tb, p)
    got = {f: np.empty(a._field_shape(f), np.complex128) for f in FIELDS}
    a.get_states(got)
    for f in FIELDS:
        assert np.array_equal(got[f], a.get_state(f))
    # perturb, load through both routes, step both: bitwise the same states
    rng = np.random.default_rng(3)
    new = {f: got[f] * (1 + 1e-3 * rng.standard_normal(got[f].shape)) for f in FIELDS}
    a.set_states(new)
    for f in FIELDS:
        b.set_state(f, new[f])
    a.step(0.01, 2)
    b.step(0.01, 2)
    out = {f: np.empty(a._field_shape(f), np.complex128) for f in FIELDS}
    a.get_states(out)
    for f in FIELDS:
        assert np.array_equal(out[f], b.get_state(f))


def test_states_reject_bad_selectors_and_shapes(tb):
    p = RBCParams(Nx=32, Nz=16, Lx=4.0, Lz=1.0, Ra=1e6)
    plan = _plan(tb, p)
    before = plan.get_state(0)
    buf = np.zeros_like(before)
    fields = (ctypes.c_int * 2)(0, 9)
    ptrs = (ctypes.c_void_p * 2)(buf.ctypes.data, buf.ctypes.data)
    st = tb.lib.tb_set_states(plan.ptr, 2, fields, ptrs, 0)
    assert st == tb._lib.TB_EINVAL
    assert np.array_equal(plan.get_state(0), before)  # nothing was copied
    with pytest.raises(ValueError):
        plan.set_states({0: np.zeros((3, 3), np.complex128)})
    with pytest.raises(ValueError):
        plan.set_state(0, np.zeros((3, 3), np.complex128))  # would read past the array
    assert np.array_equal(plan.get_state(0), before)
    with pytest.raises(ValueError):
        plan.get_states({0: np.zeros(before.shape, np.complex64)})


def test_states_through_one_contiguous_buffer(tb):
    # adjacent host views in the device order go as one copy per direction
    p = RBCParams(Nx=64, Nz=32, Lx=4.0, Lz=1.0, Ra=1e7)
    a, b = _plan(tb, p), _plan(tb, p)
    Nz, nk = p.Nz, p.Nx // 2 + 1
    buf = np.empty((4 * Nz + 7) * nk, np.complex128)
    views = {f: buf[f * Nz * nk:(f + 1) * Nz * nk].reshape(Nz, nk) for f in (0, 1, 2, 3)}
    views[4] = buf[4 * Nz * nk:].reshape(7, nk)
    a.get_states(views)
    for f in FIELDS:
        assert np.array_equal(views[f], a.get_state(f))
    buf *= 1.0 + 1e-3 * np.cos(np.arange(buf.size))
    a.set_states(views)
    for f in FIELDS:
        b.set_state(f, views[f])
    a.step(0.01, 2)
    b.step(0.01, 2)
    a.get_states(views)
    for f in FIELDS:
        assert np.array_equal(views[f], b.get_state(f))


@pytest.mark.parametrize("scheme", [0, 1])  # RK222, RK443
def test_rk_step_does_not_read_p_or_taus(tb, scheme):
    # the IMEX RK tableaus never apply L to the step's initial state (their
    # first implicit column and bI[0] are zero) and M has no p or tau columns,
    # so a step's p and taus are outputs only: the end-to-end bench uploads
    # b, u_x, u_z alone
    p = RBCParams(Nx=64, Nz=32, Lx=4.0, Lz=1.0, Ra=1e7)
    plans = []
    for seed in (None, 5):
        dom = tb.ChannelDomain(p.Nx, p.Nz, Lx=4.0, Lz=1.0)
        pl = tb.Plan(dom, p.kappa, p.nu, 1.0, 0.0, scheme)
        pl.set_state(0, forward_2d(rbc_initial_b(p, 42)))
        pl.step(0.01, 2)
        if seed is not None:
            rng = np.random.default_rng(seed)
            for f in (3, 4):
                shape = pl._field_shape(f)
                pl.set_state(f, rng.standard_normal(shape) + 1j * rng.standard_normal(shape))
        plans.append(pl)
    for pl in plans:
        pl.step(0.01, 2)
    for f in FIELDS:
        assert np.array_equal(plans[0].get_state(f), plans[1].get_state(f)), f


def test_async_step_then_states_read_back_like_the_synchronous_step(tb):
    # tb_set_states (TB_NO_WAIT), tb_step_async, tb_get_states per step (the
    # end-to-end bench's loop): the step queues behind the upload and the
    # read-back behind the step on the plan's stream, so the one wait sees
    # the finished step, bitwise as after waiting copies and tb_step
    p = RBCParams(Nx=64, Nz=32, Lx=4.0, Lz=1.0, Ra=1e7)
    a, b = _plan(tb, p), _plan(tb, p)
    Nz, nk = p.Nz, p.Nx // 2 + 1
    buf = np.empty((4 * Nz + 7) * nk, np.complex128)
    views = {f: buf[f * Nz * nk:(f + 1) * Nz * nk].reshape(Nz, nk) for f in (0, 1, 2, 3)}
    views[4] = buf[4 * Nz * nk:].reshape(7, nk)
    a.get_states(views)
    for _ in range(3):
        step_in = {f: views[f].copy() for f in (0, 1, 2)}
        a.set_states(step_in, keep_history=True, wait=False)
        a.step_async(0.01, 1)
        a.get_states(views)
        b.set_states(step_in, keep_history=True)
        b.step(0.01, 1)
        for f in FIELDS:
            assert np.array_equal(views[f], b.get_state(f)), f
    # a read-back cannot skip its wait (the caller reads the data on return)
    fields = (ctypes.c_int * 1)(0)
    ptrs = (ctypes.c_void_p * 1)(views[0].ctypes.data)
    before = views[0].copy()
    assert tb.lib.tb_get_states(a.ptr, 1, fields, ptrs, tb._lib.TB_HOST | tb._lib.TB_NO_WAIT) == tb._lib.TB_EINVAL
    assert np.array_equal(views[0], before)
