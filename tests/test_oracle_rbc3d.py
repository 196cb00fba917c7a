"""CPU checks of the 3D Rayleigh-Benard oracle (no GPU).

The 3D restatement is pinned to the 2D one (which the known-answer tests and
golden fixtures pin): a y-invariant 3D state must evolve exactly as the 2D
problem, with the ky = 0 plane equal to Ny times the 2D coefficients (the
unnormalised y transform of a constant).  Two symmetry checks cover what the
2D case cannot: x <-> y exchange and the reality of the evolved fields.
"""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

from oracle.tarang_oracle import (  # noqa: E402
    RBC2D,
    RBC3D,
    TABLEAUS,
    RBC3Params,
    RBCParams,
    backward_3d,
    forward_3d,
    padded_multiply,
    padded_multiply_3d,
    rbc3_initial_b,
    rbc_initial_b,
    rel_l2,
)


def test_y_invariant_state_follows_the_2d_problem():
    p2 = RBCParams(Nx=16, Nz=12, Lx=4.0, Lz=1.0, Ra=1e6)
    p3 = RBC3Params(Nx=16, Ny=6, Nz=12, Lx=4.0, Ly=3.0, Lz=1.0, Ra=1e6)
    b2 = rbc_initial_b(p2, 3)
    s2 = RBC2D(p2)
    s2.set_b_grid(b2)
    s3 = RBC3D(p3)
    s3.set_b_grid(np.repeat(b2[:, None, :], p3.Ny, axis=1))
    for _ in range(3):
        s2.step(0.05, "RK222")
        s3.step_rk(0.05, TABLEAUS["RK222"])
    for a2, a3 in ((s2.b, s3.b), (s2.ux, s3.ux), (s2.uz, s3.uz)):
        assert rel_l2(a3[:, 0, :] / p3.Ny, a2) < 1e-11
        assert np.abs(a3[:, 1:, :]).max() < 1e-18 * max(1.0, np.abs(a2).max())
    assert np.abs(s3.uy).max() < 1e-20


def test_product_matches_2d_product_for_y_invariant_fields():
    rng = np.random.default_rng(5)
    a = rng.standard_normal((4, 1, 12))
    b = rng.standard_normal((4, 1, 12))
    A, B = np.repeat(a, 8, axis=1), np.repeat(b, 8, axis=1)
    out = padded_multiply_3d(A, B)
    ref = padded_multiply(a[:, 0, :], b[:, 0, :])
    assert np.abs(out - ref[:, None, :]).max() < 1e-13


def test_x_y_exchange_symmetry():
    # The exchange is exact except at the Nyquist modes: x carries its Nyquist
    # as +Nx/2 (rfft layout) and y as -Ny/2 (fft order), so the two directions
    # differ at the level of the Nyquist content the products create (~1e-5
    # in u after two steps from a Nyquist-free start); a transposition or sign error in the y handling is O(1).
    p = RBC3Params(Nx=12, Ny=12, Nz=10, Lx=3.0, Ly=3.0, Ra=3e5)
    c = forward_3d(rbc3_initial_b(p, 9, amp=1e-2))
    c[:, :, -1] = 0.0  # no Nyquist content at the start
    c[:, p.Ny // 2, :] = 0.0
    g = backward_3d(c, p.Nx)
    sa, sb = RBC3D(p), RBC3D(p)
    sa.set_b_grid(g)
    sb.set_b_grid(np.ascontiguousarray(g.transpose(0, 2, 1)))
    for _ in range(2):
        sa.step_rk(0.05, TABLEAUS["RK222"])
        sb.step_rk(0.05, TABLEAUS["RK222"])
    G = lambda c: backward_3d(c, p.Nx)  # noqa: E731
    sw = lambda x: x.transpose(0, 2, 1)  # noqa: E731
    assert rel_l2(sw(G(sb.b)), G(sa.b)) < 1e-9
    assert rel_l2(sw(G(sb.uy)), G(sa.ux)) < 1e-4
    assert rel_l2(sw(G(sb.ux)), G(sa.uy)) < 1e-4
    assert rel_l2(sw(G(sb.uz)), G(sa.uz)) < 1e-4
    assert np.abs(G(sa.ux)).max() > 1e-9  # the flow is genuinely 3D


def test_nyquist_planes_carry_non_hermitian_content():
    # The kx = Nx/2 plane (and the ky = -Ny/2 row) solve complex systems whose
    # partner modes are not their conjugates, so the stored state leaves the
    # real subspace there; this is why every grid round trip of a state field
    # (and the L X_j terms of the stages) sees the Hermitian projection.
    p = RBC3Params(Nx=8, Ny=6, Nz=10, Ra=1e5)
    s = RBC3D(p)
    s.set_b_grid(rbc3_initial_b(p, 1, amp=1e-2))
    for _ in range(2):
        s.step_rk(0.05, TABLEAUS["RK443"])
    c = s.ux
    d = forward_3d(backward_3d(c, p.Nx)) - c
    assert np.abs(d[:, :, 1:-1]).max() < 1e-13 * np.abs(c).max()
    assert np.abs(d[:, :, -1]).max() > 1e-6 * np.abs(c[:, :, -1]).max()


def test_stage_solution_satisfies_walls():
    p = RBC3Params(Nx=8, Ny=6, Nz=12, Ra=1e5)
    s = RBC3D(p)
    s.set_b_grid(rbc3_initial_b(p, 2, amp=1e-2))
    M, L, bc, algf = s.mode_matrices(1, 2)
    rhs = np.random.default_rng(0).standard_normal(M.shape[0]) + 0j
    rhs[bc] = 0.1 * algf[bc]
    x = s._lhs_lu(1, 2, 1.0, 0.1).solve(rhs)
    r = (M + 0.1 * L) @ x - rhs
    assert np.abs(r).max() < 1e-9 * np.abs(rhs).max()
    N = p.Nz
    for f in range(1, 5):  # b, ux, uy, uz vanish at both walls at kx != 0
        c = x[f * N : (f + 1) * N]
        assert abs(np.sum(c)) < 1e-9 and abs(np.sum(c * (-1.0) ** np.arange(N))) < 1e-9


def test_y_invariant_sbdf2_follows_the_2d_problem():
    p2 = RBCParams(Nx=16, Nz=12, Lx=4.0, Lz=1.0, Ra=1e6)
    p3 = RBC3Params(Nx=16, Ny=6, Nz=12, Lx=4.0, Ly=3.0, Lz=1.0, Ra=1e6)
    b2 = rbc_initial_b(p2, 3)
    s2 = RBC2D(p2)
    s2.set_b_grid(b2)
    s3 = RBC3D(p3)
    s3.set_b_grid(np.repeat(b2[:, None, :], p3.Ny, axis=1))
    for _ in range(4):
        s2.step(0.02, "SBDF2")
        s3.step(0.02, "SBDF2")
    for a2, a3 in ((s2.b, s3.b), (s2.ux, s3.ux), (s2.uz, s3.uz)):
        assert rel_l2(a3[:, 0, :] / p3.Ny, a2) < 1e-11
