"""Host logic of the instance sharding used for N > 1 (independent solves,
no data-path collective): the longest-processing-time partition and the
whole-job statistics combined from per-rank parts."""
import numpy as np

from __graft_entry__ import load_package

load_package()
from tarang_b200 import workloads as W  # noqa: E402


def test_partition_covers_every_instance_once_and_balances():
    costs = [W.instance_cost(c) for c in W.ensemble_members(64)]
    for world in (1, 2, 3, 8):
        parts = W.shard_instances(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        # LPT bound: no rank exceeds the mean by more than the largest item
        assert max(loads) <= sum(costs) / world + max(costs) + 1e-9
        assert parts == W.shard_instances(costs, world)  # deterministic


def test_serving_requests_have_costs_of_both_kinds():
    reqs = W.serving_requests(60)
    c = [W.instance_cost(r) for r in reqs]
    assert all(v > 0 for v in c)
    assert {r.kind for r in reqs} == {"rbc", "turb"}


def test_combined_ensemble_and_serving_statistics():
    a = {"steps": 300, "total_ms": 100.0, "ms": [10.0, 50.0, 100.0], "plain_s": 0.5, "plain_done_ms": [100, 300, 500]}
    b = {"steps": 200, "total_ms": 80.0, "ms": [20.0, 80.0], "plain_s": 0.4, "plain_done_ms": [150, 400]}
    e = W.combine_ensemble([a, b])
    assert e["value"] == 500 / 0.1 and e["plain_value"] == 500 / 0.5
    assert e["members"] == 5 and e["p50_ms"] == 50.0 and e["total_ms"] == 100.0
    s = W.combine_serving([{"completed": 3, "steps": 300, "wall_s": 2.0, "tts_ms": [1.0, 2.0, 3.0]},
                           {"completed": 2, "steps": 100, "wall_s": 4.0, "tts_ms": [4.0, 5.0]}])
    assert s["solves_per_s"] == 5 / 4.0 and s["steps_per_s"] == 100.0 and s["p50_ms"] == 3.0
    assert np.isclose(s["p99_ms"], np.percentile([1, 2, 3, 4, 5], 99))
