"""Tunable kernel shapes (tau-solve partitions, 3D x-pass rows per CTA) and
the tuners that choose them: every shape gives the same solution, and tuning
leaves the state where it was."""
import numpy as np
import pytest

from oracle.tarang_oracle import RBCParams, forward_2d, rbc_initial_b, rel_l2, run_rbc
from oracle.tarang_oracle import RBC3D, TABLEAUS, RBC3Params, rbc3_initial_b

pytestmark = pytest.mark.gpu


def test_tau_partitions_give_the_oracle_solution(tb):
    p = RBCParams(Nx=48, Nz=24, Lx=4.0, Lz=1.0, Ra=1e8)
    sim = run_rbc(p, "RK443", 0.01, 4, seed=42)
    # Nz = 24: 48 band rows, 4 windows of 12, so 8 partitions do not fit (refused)
    for parts in (4, 1):
        dom = tb.ChannelDomain(48, 24, Lx=4.0, Lz=1.0)
        plan = tb.Plan(dom, p.kappa, p.nu, 1.0, 0.0, 1)
        plan.set_variant(tau_parts=parts)
        assert plan.variant()[0] == parts
        plan.set_state(0, forward_2d(rbc_initial_b(p, 42)))
        plan.step(0.01, 4)
        for f, want in ((0, sim.b), (1, sim.ux), (2, sim.uz)):
            assert rel_l2(plan.get_state(f), want) < 1e-10
    dom = tb.ChannelDomain(48, 24, Lx=4.0, Lz=1.0)
    plan = tb.Plan(dom, p.kappa, p.nu, 1.0, 0.0, 1)
    with pytest.raises(tb.TarangError):
        plan.set_variant(tau_parts=8)


@pytest.mark.parametrize("scheme,ts", [("RK443", 1), ("SBDF2", 3)])
def test_uneven_eight_partitions_give_the_oracle_solution(tb, scheme, ts):
    # Nz = 64: 132 band rows per class, padded to 144 = 12 windows of 12 rows,
    # so eight partitions take 1 or 2 windows each
    p = RBCParams(Nx=64, Nz=64, Lx=4.0, Lz=1.0, Ra=1e8)
    sim = run_rbc(p, scheme, 0.01, 5, seed=42)
    states = {}
    for parts in (8, 4, 1):
        dom = tb.ChannelDomain(64, 64, Lx=4.0, Lz=1.0)
        plan = tb.Plan(dom, p.kappa, p.nu, 1.0, 0.0, ts)
        plan.set_variant(tau_parts=parts)
        assert plan.variant()[0] == parts
        plan.set_state(0, forward_2d(rbc_initial_b(p, 42)))
        plan.step(0.01, 5)
        for f, want in ((0, sim.b), (1, sim.ux), (2, sim.uz)):
            assert rel_l2(plan.get_state(f), want) < 1e-10, (parts, f)
        states[parts] = [plan.get_state(f) for f in (0, 1, 2, 3)]
    for parts in (8, 4):
        for a, b in zip(states[parts], states[1]):
            # partitions change the rounding of the sweeps (responses), not the solution
            assert rel_l2(a, b) < 1e-11 or np.abs(b).max() == 0.0


@pytest.mark.parametrize("scheme,ts", [("RK443", 1), ("SBDF2", 3)])
def test_uneven_sixteen_partitions_give_the_oracle_solution(tb, scheme, ts):
    # Nz = 96: 196 band rows per class, padded to 240 = 20 windows of 12 rows
    # (10 window pairs over 8 warps), so the sixteen partitions take 1 or 2
    # windows each; the records stream in 3-row stages, y and the particular
    # unknowns through global scratch, the starting windows carried down
    p = RBCParams(Nx=64, Nz=96, Lx=4.0, Lz=1.0, Ra=1e8)
    sim = run_rbc(p, scheme, 0.01, 5, seed=42)
    states = {}
    for parts in (16, 1):
        dom = tb.ChannelDomain(64, 96, Lx=4.0, Lz=1.0)
        plan = tb.Plan(dom, p.kappa, p.nu, 1.0, 0.0, ts)
        plan.set_variant(tau_parts=parts)
        assert plan.variant()[0] == parts
        plan.set_state(0, forward_2d(rbc_initial_b(p, 42)))
        plan.step(0.01, 5)
        for f, want in ((0, sim.b), (1, sim.ux), (2, sim.uz)):
            assert rel_l2(plan.get_state(f), want) < 1e-10, (parts, f)
        states[parts] = [plan.get_state(f) for f in (0, 1, 2, 3)]
    for a, b in zip(states[16], states[1]):
        assert rel_l2(a, b) < 1e-11 or np.abs(b).max() == 0.0


def test_sixteen_partitions_need_sixteen_windows(tb):
    # Nz = 64: 144 padded band rows = 12 windows, fewer than 16 partitions
    dom = tb.ChannelDomain(64, 64, Lx=4.0, Lz=1.0)
    p = RBCParams(Nx=64, Nz=64, Lx=4.0, Lz=1.0, Ra=1e8)
    plan = tb.Plan(dom, p.kappa, p.nu, 1.0, 0.0, 1)
    with pytest.raises(tb.TarangError):
        plan.set_variant(tau_parts=16)


@pytest.mark.parametrize("key", ["16x11", "24x16", "96x24"])
def test_batched_x_products_match_golden_rhs(tb, golden_dir, key):
    import os

    d = np.load(os.path.join(golden_dir, "transforms.npz"))
    Nx, Nz = map(int, key.split("x"))
    p = RBCParams(Nx=Nx, Nz=Nz)  # the fixture's parameters (Lx 4, Lz 1)
    dom = tb.ChannelDomain(Nx, Nz, Lx=p.Lx, Lz=p.Lz)
    outs = {}
    for form in (1, 2, 3):
        plan = tb.Plan(dom, p.kappa, p.nu, 1.0, 0.0, 0)
        plan.set_variant(xrows=form)
        assert plan.variant()[1] == form
        outs[form] = plan.rhs_advection(*(d[f"rhs_in{i}_{key}"] for i in range(3)))
        for i in range(3):
            assert rel_l2(outs[form][i], d[f"rhs_out{i}_{key}"]) < 1e-12
    for form in (2, 3):
        for a, b in zip(outs[1], outs[form]):
            assert rel_l2(a, b) < 1e-14


@pytest.mark.parametrize("form", [2, 3])
@pytest.mark.parametrize("scheme,ts", [("RK443", 1), ("SBDF2", 3)])
def test_batched_x_products_steps_match_oracle(tb, scheme, ts, form):
    p = RBCParams(Nx=256, Nz=64, Lx=4.0, Lz=1.0, Ra=1e8)
    sim = run_rbc(p, scheme, 0.01, 4, seed=42)
    dom = tb.ChannelDomain(256, 64, Lx=4.0, Lz=1.0)
    plan = tb.Plan(dom, p.kappa, p.nu, 1.0, 0.0, ts)
    plan.set_variant(xrows=form)
    plan.set_state(0, forward_2d(rbc_initial_b(p, 42)))
    plan.step(0.01, 4)
    for f, want in ((0, sim.b), (1, sim.ux), (2, sim.uz)):
        assert rel_l2(plan.get_state(f), want) < 1e-10


def test_batched_x_products_mixed_precision(tb):
    # the FP32 batched kernel against the FP32 per-field kernel and the FP64 oracle RHS
    from oracle.tarang_oracle import RBC2D

    Nx, Nz = 96, 24
    rng = np.random.default_rng(6)
    ins = [forward_2d(rng.standard_normal((Nz, Nx))) for _ in range(3)]
    p = RBCParams(Nx=Nx, Nz=Nz)
    dom = tb.ChannelDomain(Nx, Nz, Lx=p.Lx, Lz=p.Lz)
    outs = {}
    for form in (1, 2, 3):
        plan = tb.Plan(dom, p.kappa, p.nu, 1.0, 0.0, 0, precision=tb._lib.TB_PREC_MIXED)
        plan.set_variant(xrows=form)
        outs[form] = plan.rhs_advection(*ins)
    ref = RBC2D(p).rhs(*ins)
    for form in (2, 3):
        for a, b, r in zip(outs[1], outs[form], ref):
            assert rel_l2(b, a) < 1e-6 and rel_l2(b, r) < 1e-5


def test_xpass_rows_and_tau_partitions_agree_in_3d(tb):
    p = RBC3Params(Nx=24, Ny=24, Nz=12, Lx=4.0, Ly=4.0, Ra=1e6)
    sim = RBC3D(p)
    sim.set_b_grid(rbc3_initial_b(p, 42, amp=1e-2))
    for _ in range(2):
        sim.step_rk(0.01, TABLEAUS["RK222"])
    ref = None
    for parts, rows in ((4, 2), (1, 1), (1, 4), (4, 1)):
        plan = tb.Plan3D(24, 24, 12, p.kappa, p.nu, 0, 4.0, 4.0, 1.0, precision=tb._lib.TB_PREC_MIXED)
        plan.set_variant(tau_parts=parts, xrows=rows)
        assert plan.variant() == (parts, rows)
        plan.set_state(0, plan.forward(rbc3_initial_b(p, 42, amp=1e-2)))
        plan.step(0.01, 2)
        ux = plan.get_state(1)
        assert rel_l2(ux, sim.ux) < 1e-6
        if ref is None:
            ref = ux
        else:
            assert rel_l2(ux, ref) < 1e-12  # the same arithmetic in every shape


def test_plan_tune_keeps_state_and_picks_a_feasible_shape(tb):
    p = RBCParams(Nx=64, Nz=32, Lx=4.0, Lz=1.0, Ra=1e6)
    dom = tb.ChannelDomain(64, 32, Lx=4.0, Lz=1.0)
    plan = tb.Plan(dom, p.kappa, p.nu, 1.0, 0.0, 0)
    plan.set_state(0, forward_2d(rbc_initial_b(p, 42)))
    plan.step(0.02, 2)
    before = [plan.get_state(f) for f in (0, 1, 2)]
    parts, rows = plan.tune(0.02, trial_steps=3)
    assert parts in (1, 4, 8, 16) and rows in (1, 2, 3) and plan.variant() == (parts, rows)
    for f, b in zip((0, 1, 2), before):
        assert np.array_equal(plan.get_state(f), b)
    plan.step(0.02, 2)  # steps on with the chosen shape
    assert np.isfinite(plan.get_state(2)).all()


def test_ensemble_tune_applies_one_partitioning_to_all_members(tb):
    plans = []
    for Nx, Nz in ((64, 16), (96, 24), (128, 32)):
        p = RBCParams(Nx=Nx, Nz=Nz, Ra=1e6)
        dom = tb.ChannelDomain(Nx, Nz, Lx=4.0, Lz=1.0)
        pl = tb.Plan(dom, p.kappa, p.nu, 1.0, 0.0, 0)
        pl.set_state(0, forward_2d(rbc_initial_b(p, 7)))
        plans.append(pl)
    ens = tb.Ensemble(plans)
    before = [pl.get_state(0) for pl in plans]
    ens.tune(0.02, trial_steps=2)
    parts = {pl.variant()[0] for pl in plans}
    assert len(parts) == 1 and parts <= {1, 4, 8}
    for pl, b in zip(plans, before):
        assert np.array_equal(pl.get_state(0), b)
