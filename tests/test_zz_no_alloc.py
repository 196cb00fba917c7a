"""The allocation-free dealiased product, checked against the plan entry point
and the oracle's padded product.

tb_dealiased_multiply_noalloc serves callers that cannot let a library call
cudaMalloc (a host runtime that owns the device memory pool, or a process with
a fixed device footprint): it takes the caller's device buffers and keeps its
FFT twiddles in a static device array.  This file is collected last so a run
that stops at the first failure has already run every other test; it also
passes on its own in a fresh process (the first call does the per-device
set-up)."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _plan_product(tb, Nx, Nz, a, b):
    dom = tb.ChannelDomain(Nx, Nz, Lx=4.0, Lz=1.0)
    plan = tb.Plan(dom, 1e-3, 1e-3, 1.0, 0.0, 0)
    return plan.dealiased_multiply(a, b)


def _noalloc_product(tb, Nx, Nz, a, b):
    import torch

    ta = torch.as_tensor(np.ascontiguousarray(a), device="cuda")
    tbb = torch.as_tensor(np.ascontiguousarray(b), device="cuda")
    out = torch.full_like(ta, float("nan"))
    torch.cuda.synchronize()
    st = tb.lib.tb_dealiased_multiply_noalloc(0, Nx, Nz, ctypes.c_void_p(ta.data_ptr()),
                                              ctypes.c_void_p(tbb.data_ptr()), ctypes.c_void_p(out.data_ptr()))
    assert st == 0, tb.lib.tb_last_error(None)
    return out.cpu().numpy()


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_noalloc_product_matches_plan_entry_point_on_two_calls(tb):
    from oracle.tarang_oracle import padded_multiply

    rng = np.random.default_rng(11)
    # calls in a row with different sizes: each rewrites the shared twiddles.
    # Nx = 2048 (padded length 3072) fills the static array exactly.
    for Nx, Nz in ((256, 64), (96, 17), (2048, 8), (256, 64)):
        a = rng.standard_normal((Nz, Nx))
        b = rng.standard_normal((Nz, Nx))
        want = _plan_product(tb, Nx, Nz, a, b)
        got = _noalloc_product(tb, Nx, Nz, a, b)
        assert _rel(got, want) < 1e-12, (Nx, Nz)
        assert _rel(got, padded_multiply(a, b)) < 1e-12, (Nx, Nz)


def test_noalloc_product_rejects_sizes_beyond_its_array(tb):
    import torch

    buf = torch.zeros(4096 * 2, dtype=torch.float64, device="cuda")
    p = ctypes.c_void_p(buf.data_ptr())
    assert tb.lib.tb_dealiased_multiply_noalloc(0, 4096, 2, p, p, p) == 6  # TB_ENOTSUPPORTED
    assert b"2048" in tb.lib.tb_last_error(None)
    assert tb.lib.tb_dealiased_multiply_noalloc(0, 14, 2, p, p, p) == 6  # 14 = 2 x 7: no radix-2/3 FFT
    assert tb.lib.tb_dealiased_multiply_noalloc(0, 15, 2, p, p, p) == 1  # odd Nx
    assert tb.lib.tb_dealiased_multiply_noalloc(0, 64, 2, p, None, p) == 1  # null buffer
    assert b"null" in tb.lib.tb_last_error(None)
