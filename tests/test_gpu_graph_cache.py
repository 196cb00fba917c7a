"""Cached step graphs stay consistent with the factor sets they read.

A plan keeps at most two tau factor sets; a third dt takes over the oldest
set's device buffers.  Captured step graphs hold those buffers' addresses, so
a multi-step graph captured at dt1 must not be replayed after its set was
rebuilt for another dt.  The sequence below evicts the dt1 set while the dt1
multi-step graph is cached, then asks for dt1 multi-steps again; it must give
exactly what plain single steps at the same dts give.
"""
import numpy as np
import pytest

from oracle.tarang_oracle import RBCParams, forward_2d, rbc_initial_b

pytestmark = pytest.mark.gpu


def _plan(tb, p, scheme):
    dom = tb.ChannelDomain(p.Nx, p.Nz, Lx=p.Lx, Lz=p.Lz)
    plan = tb.Plan(dom, p.kappa, p.nu, p.Lz, 0.0, scheme)
    plan.set_state(0, forward_2d(rbc_initial_b(p)))
    return plan


@pytest.mark.parametrize("scheme", [1, 0])  # RK443, RK222
def test_multistep_graph_after_factor_set_eviction(tb, scheme):
    p = RBCParams(Nx=64, Nz=32, Lx=4.0, Lz=1.0, Ra=1e6)
    dt1, dt2, dt3 = 0.01, 0.0125, 0.015
    graphed = _plan(tb, p, scheme)
    plain = _plan(tb, p, scheme)
    graphed.step_async(dt1, 8, 8)  # multi-step graph captured against the dt1 set
    graphed.wait()
    graphed.step(dt2, 1)  # second factor set
    graphed.step(dt3, 1)  # evicts the dt1 set, reusing its buffers for dt3
    graphed.step_async(dt1, 8, 8)  # dt1 rebuilt in other buffers: the graph must follow
    graphed.wait()
    for dt, n in ((dt1, 8), (dt2, 1), (dt3, 1), (dt1, 8)):
        for _ in range(n):
            plain.step(dt, 1)
    for f in (0, 1, 2):
        a, b = graphed.get_state(f), plain.get_state(f)
        assert np.array_equal(a, b), (f, np.abs(a - b).max())
