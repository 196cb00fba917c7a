"""Ensembles and asynchronous stepping through the C ABI.

The ensemble runner steps independent plans concurrently on worker streams;
each member must end exactly where the same plan stepped alone ends (the same
graphs run, only their interleaving on the device changes), tuning must leave
every member's state untouched, and asynchronous steps must equal synchronous
ones.  Members are also checked against the CPU oracle at 1e-10.
"""
import numpy as np
import pytest

from oracle.tarang_oracle import RBCParams, forward_2d, rbc_initial_b, rel_l2, run_rbc

pytestmark = pytest.mark.gpu

TS = {"RK222": 0, "RK443": 1, "SBDF1": 2, "SBDF2": 3}
# (Nx, Nz, Ra, scheme, dt): uneven sizes, parameters and schemes
MEMBERS = [
    (32, 16, 2e6, "RK222", 0.125),
    (48, 24, 1e8, "RK443", 0.01),
    (64, 17, 1e6, "SBDF2", 0.05),
    (96, 24, 1e7, "RK222", 0.02),
    (32, 16, 1e5, "RK443", 0.1),
]


def build(tb, spec, seed, precision=None):
    Nx, Nz, Ra, scheme, _ = spec
    p = RBCParams(Nx=Nx, Nz=Nz, Lx=4.0, Lz=1.0, Ra=Ra)
    dom = tb.ChannelDomain(Nx, Nz, Lx=4.0, Lz=1.0)
    prec = tb._lib.TB_PREC_F64 if precision is None else precision
    plan = tb.Plan(dom, p.kappa, p.nu, 1.0, 0.0, TS[scheme], precision=prec)
    plan.set_state(0, forward_2d(rbc_initial_b(p, seed)))
    return p, plan


def states(plan):
    return [plan.get_state(f) for f in range(3)]


def test_ensemble_members_equal_solo_runs(tb):
    nsteps = 7
    solo = []
    for k, spec in enumerate(MEMBERS):
        _, plan = build(tb, spec, 40 + k)
        plan.step(spec[4], nsteps)
        solo.append(states(plan))
    plans = [build(tb, spec, 40 + k)[1] for k, spec in enumerate(MEMBERS)]
    ens = tb.Ensemble(plans)
    ens.set_config(3, 4)  # 3 worker streams, graphs of 4 steps (7 = 4 + 3)
    ms, total = ens.run([s[4] for s in MEMBERS], nsteps)
    assert total > 0 and np.all(ms > 0) and np.all(ms <= total + 1e-3)
    for k, plan in enumerate(plans):
        for a, b in zip(states(plan), solo[k]):
            assert np.array_equal(a, b), f"member {k} differs from its solo run"


def test_ensemble_members_match_oracle(tb):
    nsteps = 4
    plans, params = [], []
    for k, spec in enumerate(MEMBERS[:3]):
        p, plan = build(tb, spec, 42)
        plans.append(plan)
        params.append(p)
    ens = tb.Ensemble(plans)
    ens.set_config(2, 2)
    ens.run([s[4] for s in MEMBERS[:3]], nsteps)
    for spec, p, plan in zip(MEMBERS[:3], params, plans):
        sim = run_rbc(p, spec[3], spec[4], nsteps, seed=42)
        for got, want in zip(states(plan), (sim.b, sim.ux, sim.uz)):
            assert rel_l2(got, want) < 1e-10


def test_tune_restores_state(tb):
    plans = [build(tb, spec, 7 + k)[1] for k, spec in enumerate(MEMBERS)]
    before = [states(p) for p in plans]
    t_before = [p.sim_time() for p in plans]
    ens = tb.Ensemble(plans)
    s, g = ens.tune([spec[4] for spec in MEMBERS], trial_steps=4)
    assert 1 <= s <= len(plans) and g in (1, 4)
    assert ens.config() == (s, g)
    for p, st, t in zip(plans, before, t_before):
        for a, b in zip(states(p), st):
            assert np.array_equal(a, b)
        assert p.sim_time() == t


def test_async_steps_equal_sync_steps(tb):
    spec = MEMBERS[1]
    _, a = build(tb, spec, 3)
    _, b = build(tb, spec, 3)
    a.step(spec[4], 6)
    b.step_async(spec[4], 6, graph_steps=4)
    b.wait()
    assert b.idle()
    for x, y in zip(states(a), states(b)):
        assert np.array_equal(x, y)
    assert b.device_bytes() > 0


# same shapes with different Ra / Pr (fusible groups), plus lone shapes
FUSED = [
    (32, 16, 2e6, "RK222", 0.05),
    (64, 24, 1e7, "RK443", 0.01),
    (32, 16, 1e5, "RK222", 0.05),
    (64, 24, 3e6, "RK443", 0.01),
    (32, 16, 5e6, "RK222", 0.05),
    (48, 17, 1e6, "RK222", 0.05),   # lone shape: steps per member
    (64, 24, 1e8, "RK443", 0.01),
]


def test_fused_form_matches_solo_runs_and_oracle(tb):
    nsteps = 5
    solo = []
    for k, spec in enumerate(FUSED):
        _, plan = build(tb, spec, 70 + k)
        plan.step(spec[4], nsteps)
        solo.append(states(plan))
    pairs = [build(tb, spec, 70 + k) for k, spec in enumerate(FUSED)]
    plans = [pl for _, pl in pairs]
    ens = tb.Ensemble(plans)
    ens.set_form(True)
    ens.set_config(2, 2)
    ms, total = ens.run([s[4] for s in FUSED], nsteps)
    fused, groups = ens.form()
    assert fused and groups == 2
    for k, plan in enumerate(plans):
        for a, b in zip(states(plan), solo[k]):
            assert rel_l2(a, b) < 1e-12, f"member {k}"
        assert abs(plan.sim_time() - nsteps * FUSED[k][4]) < 1e-12
    # and the stacked plans hold each member's own kappa / nu
    for k in (0, 1, 3):
        p, _ = pairs[k]
        ref = run_rbc(p, FUSED[k][3], FUSED[k][4], nsteps, seed=70 + k)
        assert rel_l2(plans[k].get_state(0), ref.b) < 1e-10
        assert rel_l2(plans[k].get_state(2), ref.uz) < 1e-10
    # a second run continues from the scattered states
    ens.run([s[4] for s in FUSED], 2)
    _, again = build(tb, FUSED[2], 72)
    again.step(FUSED[2][4], nsteps + 2)
    assert rel_l2(plans[2].get_state(0), again.get_state(0)) < 1e-12


@pytest.mark.parametrize("form", [1, 2])
def test_fused_form_with_mixed_precision_members(tb, form):
    # mixed members stack like Float64 ones; each matches its solo mixed run
    # to FP32 rounding and the FP64 oracle at the mixed bar (1e-6)
    nsteps = 5
    mixed = tb._lib.TB_PREC_MIXED
    solo = []
    for k, spec in enumerate(FUSED):
        _, plan = build(tb, spec, 70 + k, mixed)
        plan.set_variant(xrows=form)
        plan.step(spec[4], nsteps)
        solo.append(states(plan))
    pairs = [build(tb, spec, 70 + k, mixed) for k, spec in enumerate(FUSED)]
    plans = [pl for _, pl in pairs]
    for pl in plans:
        pl.set_variant(xrows=form)
    ens = tb.Ensemble(plans)
    ens.set_form(True)
    ens.set_config(2, 2)
    ens.run([s[4] for s in FUSED], nsteps)
    fused, groups = ens.form()
    assert fused and groups == 2
    for k, plan in enumerate(plans):
        for a, b in zip(states(plan), solo[k]):
            assert rel_l2(a, b) < 1e-6, f"member {k}"
    for k in (0, 1, 3):
        p, _ = pairs[k]
        ref = run_rbc(p, FUSED[k][3], FUSED[k][4], nsteps, seed=70 + k)
        assert rel_l2(plans[k].get_state(0), ref.b) < 1e-6
        assert rel_l2(plans[k].get_state(2), ref.uz) < 1e-6


FUSED_SBDF = [
    (48, 24, 1e7, "SBDF2", 0.01),
    (32, 16, 1e6, "SBDF2", 0.02),
    (48, 24, 1e8, "SBDF2", 0.01),
    (32, 16, 1e5, "SBDF2", 0.02),
]


def test_fused_form_with_multistep_members(tb):
    # SBDF2 members stack with their history (F and M X of the previous step):
    # the first fused run starts at SBDF1 and carries the history out; the
    # second continues at SBDF2 from the scattered history
    nsteps = 4
    solo = []
    for k, spec in enumerate(FUSED_SBDF):
        _, plan = build(tb, spec, 110 + k)
        plan.step(spec[4], nsteps + 3)
        solo.append(states(plan))
    pairs = [build(tb, spec, 110 + k) for k, spec in enumerate(FUSED_SBDF)]
    plans = [pl for _, pl in pairs]
    ens = tb.Ensemble(plans)
    ens.set_form(True)
    ens.set_config(2, 2)
    ens.run([s[4] for s in FUSED_SBDF], nsteps)
    fused, groups = ens.form()
    assert fused and groups == 2
    for k in (0, 3):
        p, _ = pairs[k]
        ref = run_rbc(p, "SBDF2", FUSED_SBDF[k][4], nsteps, seed=110 + k)
        for got, want in zip(states(plans[k]), (ref.b, ref.ux, ref.uz)):
            assert rel_l2(got, want) < 1e-10
    ens.run([s[4] for s in FUSED_SBDF], 3)
    for k, plan in enumerate(plans):
        for a, b in zip(states(plan), solo[k]):
            assert rel_l2(a, b) < 1e-12, f"member {k}"
        assert abs(plan.sim_time() - (nsteps + 3) * FUSED_SBDF[k][4]) < 1e-12


def test_tuner_may_choose_the_fused_form(tb):
    plans = [build(tb, spec, 90 + k)[1] for k, spec in enumerate(FUSED)]
    before = [pl.get_state(0) for pl in plans]
    ens = tb.Ensemble(plans)
    ens.tune([s[4] for s in FUSED], trial_steps=2)
    fused, groups = ens.form()
    assert groups in (0, 2)
    for pl, b in zip(plans, before):
        assert np.array_equal(pl.get_state(0), b)
    ens.run([s[4] for s in FUSED], 2)
    assert all(np.isfinite(pl.get_state(0)).all() for pl in plans)
