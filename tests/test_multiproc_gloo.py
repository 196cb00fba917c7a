"""The N>1 plumbing of bench.py on CPU: two gloo ranks, replicas only.

Each rank runs the reference arm on a tiny slice of work; rank 0 alone prints
the JSON line, both ranks exit 0, and the barrier / max-over-ranks helpers
agree across ranks."""
import json
import os
import subprocess
import sys

from __graft_entry__ import ROOT


def _run_two_ranks(code: str, port: int):
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), TB_DIST_BACKEND="gloo", PYTHONPATH=ROOT)
        procs.append(subprocess.Popen([sys.executable, "-c", code], env=env, cwd=ROOT, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = [p.communicate(timeout=180) for p in procs]
    return [(p.returncode, o, e) for p, (o, e) in zip(procs, outs)]


def test_dist_barrier_and_max_over_ranks():
    code = (
        "import bench\n"
        "d = bench.Dist()\n"
        "d.barrier()\n"
        "print(d.max(float(d.rank) * 10 + 1))\n"
        "d.close()\n"
    )
    res = _run_two_ranks(code, 29611)
    for rc, out, err in res:
        assert rc == 0, err
        assert float(out.strip().splitlines()[-1]) == 11.0


def test_reference_arm_prints_once_under_two_ranks():
    # rank 0 alone runs the CPU leg; the other rank leaves at once (no process
    # group, so it never waits in a barrier for rank 0's minutes of host work)
    code = (
        "import sys, time\n"
        "sys.argv = ['bench.py', '--impl', 'reference', '--config', 'c1', '--steps', '1', '--warmup', '3']\n"
        "import bench\n"
        "t0 = time.perf_counter()\n"
        "bench.main()\n"
        "print('ELAPSED', time.perf_counter() - t0)\n"
    )
    res = _run_two_ranks(code, 29623)
    assert all(rc == 0 for rc, _, _ in res), [e[-2000:] for _, _, e in res]
    lines0 = [l for l in res[0][1].splitlines() if l.startswith("{")]
    lines1 = [l for l in res[1][1].splitlines() if l.startswith("{")]
    assert len(lines0) == 1 and not lines1
    el = [float(next(l for l in out.splitlines() if l.startswith("ELAPSED")).split()[1]) for _, out, _ in res]
    assert el[1] < 0.5 * el[0], el
    d = json.loads(lines0[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["e2e"]["h2d_bytes_per_step"] == 0
    assert d["warmup"] == 3 and d["steps"] == 1 and d["cpu_baseline"]["kind"] == "port"


def test_instance_sharding_is_complete_disjoint_and_agreed_by_two_ranks():
    # Each rank derives its share of the ensemble members and of the serving
    # requests on its own (no communication), as bench.py does under torchrun;
    # the gathered shares must cover every instance exactly once and every rank
    # must have computed the same partition.
    code = (
        "import json, bench\n"
        "from __graft_entry__ import load_package\n"
        "load_package()\n"
        "from tarang_b200 import workloads as W\n"
        "d = bench.Dist()\n"
        "mem = W.ensemble_members(64)\n"
        "req = W.serving_requests(60)\n"
        "sm = W.shard_instances([W.instance_cost(c) for c in mem], d.world)\n"
        "sr = W.shard_instances([W.instance_cost(r) for r in req], d.world)\n"
        "got = d.gather({'rank': d.rank, 'members': sm[d.rank], 'requests': sr[d.rank], 'plan': [sm, sr]})\n"
        "print(json.dumps(got))\n"
        "d.close()\n"
    )
    res = _run_two_ranks(code, 29637)
    for rc, out, err in res:
        assert rc == 0, err[-2000:]
    got = json.loads(res[0][1].strip().splitlines()[-1])
    assert got == json.loads(res[1][1].strip().splitlines()[-1])
    assert [g["rank"] for g in got] == [0, 1]
    assert got[0]["plan"] == got[1]["plan"]
    for key, n in (("members", 64), ("requests", 60)):
        allidx = sorted(got[0][key] + got[1][key])
        assert allidx == list(range(n))
        assert got[0][key] and got[1][key]
