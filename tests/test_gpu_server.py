"""Request server: continuous batching of RBC and turbulence requests.

Each result must be the same alone and in the mix: bitwise for a request on
its own plan and graphs (only the interleaving on the device differs), to
rounding (1e-12) for a member of a cohort stepped as one stacked plan;
admission must respect the device-memory budget, and the statistics report
time to solution."""
import numpy as np
import pytest

from oracle.tarang_oracle import RBCParams, rbc_initial_b, rel_l2, run_rbc, turb_initial_spec

pytestmark = pytest.mark.gpu


def rbc_req(tb, Nx, Nz, Ra, seed):
    p = RBCParams(Nx=Nx, Nz=Nz, Lx=4.0, Lz=1.0, Ra=Ra)
    return p, tb.rbc_desc(Nx, Nz, p.kappa, p.nu, 0), rbc_initial_b(p, seed)


def test_results_same_alone_and_in_mix(tb):
    reqs = []
    for k, (Nx, Nz, Ra) in enumerate([(32, 16, 2e6), (64, 24, 1e7), (48, 16, 1e5)]):
        p, d, b0 = rbc_req(tb, Nx, Nz, Ra, 100 + k)
        reqs.append(("rbc", d, 0.02, 12 + 3 * k, b0))
    for k, (N, M) in enumerate([(32, 32), (64, 48)]):
        reqs.append(("turb", tb.turb_desc(N, M, 1e-3), 2e-3, 10 + k, turb_initial_spec(N, M, seed=200 + k)))
    # a DiagonalIMEX RK443 turbulence request beside the SBDF2 ones
    reqs.append(("turb", tb.turb_desc(32, 32, 1e-3, timestepper=tb._lib.TB_RK443), 2e-3, 7,
                 turb_initial_spec(32, 32, seed=210)))
    alone = []
    for _, d, dt, n, init in reqs:
        s = tb.Server(budget_bytes=1 << 30, max_running=1, chunk_steps=4)
        rid = s.submit(d, dt, n, init)
        s.wait_all()
        assert s.poll(rid)[0] == tb._lib.TB_REQ_DONE
        alone.append(s.result(rid))
        s.close()
    s = tb.Server(budget_bytes=1 << 30, max_running=8, chunk_steps=3)
    ids = [s.submit(d, dt, n, init) for _, d, dt, n, init in reqs]
    s.wait_all()
    for rid, want in zip(ids, alone):
        st, tts = s.poll(rid)
        assert st == tb._lib.TB_REQ_DONE and tts > 0
        for a, b in zip(s.result(rid), want):
            assert np.array_equal(a, b)
    stats = s.stats()
    assert stats["completed"] == len(reqs) and stats["failed"] == 0
    assert stats["peak_running"] >= 2
    assert stats["p99_ms"] >= stats["p50_ms"] > 0
    s.close()


def test_cohort_results_match_solo_runs_and_oracle(tb):
    # five RBC requests of one shape at one dt (their own Ra, seeds and step
    # counts within 25 % of each other) run as one stacked plan, each leaving
    # at its own count; a request of the same shape with a far step count, one
    # of another shape and a turbulence request run alone
    specs = [(1e6, 9), (1e7, 8), (2e6, 10), (1e5, 9), (5e6, 8), (3e6, 30)]
    reqs = []
    for k, (Ra, n) in enumerate(specs):
        p, d, b0 = rbc_req(tb, 48, 24, Ra, 400 + k)
        reqs.append((p, d, 0.02, n, b0))
    alone = []
    for p, d, dt, n, b0 in reqs:
        s = tb.Server(budget_bytes=1 << 30, max_running=1, chunk_steps=4)
        rid = s.submit(d, dt, n, b0)
        s.wait_all()
        alone.append(s.result(rid))
        s.close()
    s = tb.Server(budget_bytes=1 << 30, max_running=8, chunk_steps=4)
    s.set_cohort(16)
    ids = [s.submit(d, dt, n, b0) for _, d, dt, n, b0 in reqs]
    _, od, ob = rbc_req(tb, 32, 16, 1e6, 450)
    oid = s.submit(od, 0.02, 5, ob)
    tid = s.submit(tb.turb_desc(32, 32, 1e-3), 2e-3, 6, turb_initial_spec(32, 32, seed=460))
    s.wait_all()
    for rid, want in zip(ids + [oid, tid], alone + [None, None]):
        assert s.poll(rid)[0] == tb._lib.TB_REQ_DONE
        if want is not None:
            for a, b in zip(s.result(rid), want):
                # the stacked kernels change only the rounding
                assert rel_l2(a, b) < 1e-12
    for k in (0, 2):
        p, _, dt, n, _ = reqs[k]
        sim = run_rbc(p, "RK222", dt, n, seed=400 + k)
        b, ux, uz = s.result(ids[k])
        assert rel_l2(b, sim.b) < 1e-10 and rel_l2(uz, sim.uz) < 1e-10
    st = s.stats()
    assert st["completed"] == 8 and st["failed"] == 0
    assert st["peak_cohort"] >= 2 and st["cohort_requests"] >= 2
    s.close()


def test_cohorts_off_gives_solo_results_bitwise(tb):
    reqs = [rbc_req(tb, 48, 24, Ra, 500 + k) for k, Ra in enumerate((1e6, 3e6, 1e7))]
    alone = []
    for p, d, b0 in reqs:
        s = tb.Server(budget_bytes=1 << 30, max_running=1, chunk_steps=3)
        rid = s.submit(d, 0.02, 6, b0)
        s.wait_all()
        alone.append(s.result(rid))
        s.close()
    s = tb.Server(budget_bytes=1 << 30, max_running=8, chunk_steps=3)
    s.set_cohort(1)
    ids = [s.submit(d, 0.02, 6, b0) for _, d, b0 in reqs]
    s.wait_all()
    for rid, want in zip(ids, alone):
        for a, b in zip(s.result(rid), want):
            assert np.array_equal(a, b)
    assert s.stats()["peak_cohort"] == 1
    s.close()


def test_rbc_request_matches_oracle(tb):
    p, d, b0 = rbc_req(tb, 32, 16, 2e6, 42)
    s = tb.Server(budget_bytes=1 << 30, max_running=4, chunk_steps=2)
    rid = s.submit(d, 0.125, 5, b0)
    s.wait_all()
    b, ux, uz = s.result(rid)
    sim = run_rbc(p, "RK222", 0.125, 5, seed=42)
    assert rel_l2(b, sim.b) < 1e-10 and rel_l2(uz, sim.uz) < 1e-10
    s.close()


def test_admission_respects_budget(tb):
    p, d, b0 = rbc_req(tb, 64, 24, 1e6, 1)
    s = tb.Server(budget_bytes=1 << 30, max_running=16, chunk_steps=2)
    rid = s.submit(d, 0.02, 2, b0)
    s.wait_all()
    one = s.stats()["peak_bytes"]
    s.close()
    # a budget that holds two such runs at a time: never more than two run together
    s = tb.Server(budget_bytes=2 * one + one // 2, max_running=16, chunk_steps=2)
    ids = [s.submit(d, 0.02, 6, b0) for _ in range(5)]
    s.wait_all()
    st = s.stats()
    assert st["completed"] == 5 and st["peak_bytes"] <= st["budget_bytes"] and st["peak_running"] <= 2
    # a request that can never fit fails instead of blocking the queue
    big = tb.rbc_desc(512, 128, 1e-4, 1e-4, 0)
    bid = s.submit(big, 0.01, 1, np.zeros((128, 512)))
    s.wait_all()
    assert s.poll(bid)[0] == tb._lib.TB_REQ_FAILED
    s.close()
    del rid, ids


def test_failing_requests_do_not_disturb_the_others(tb):
    # kappa = 0 passes submission and fails in the plan build on a setup
    # thread; those requests end FAILED with the build's message while the
    # valid ones, built concurrently on other setup threads, complete
    good, bad = [], []
    s = tb.Server(budget_bytes=1 << 30, max_running=8, chunk_steps=3)
    for k in range(6):
        p, d, b0 = rbc_req(tb, 32, 16, 1e6, 300 + k)
        if k % 2:
            d.kappa = 0.0
            bad.append(s.submit(d, 0.02, 6, b0))
        else:
            good.append(s.submit(d, 0.02, 6, b0))
    s.wait_all()
    for rid in good:
        assert s.poll(rid)[0] == tb._lib.TB_REQ_DONE
    for rid in bad:
        assert s.poll(rid)[0] == tb._lib.TB_REQ_FAILED
        assert b"kappa and nu must be positive" in tb.lib.tb_last_error(s.ctx)
    st = s.stats()
    assert st["completed"] == len(good) and st["failed"] == len(bad)
    s.close()
