"""Phase clocks of the partitioned tau solve on the 2D benchmark grid.

Runs the 1024x256 RK443 plan (Ra 1e8, dt 0.01, the benchmark's seeded initial
state) on the phase-clock build of the library (``make -C tarang.jl_b200/csrc
clocks``, which records the SM cycle counter at the phase boundaries of every
partition of every mode group) and prints, per partition count, the cycles of
each phase: F1 forward sweep, F2 starting windows and border, B1 backward
sweep, B2 window carry, B3 response pass.  Usage (one GPU):

    make -C tarang.jl_b200/csrc clocks
    python tarang.jl_b200/solve_clocks.py 4 8 16
"""
from __future__ import annotations

import ctypes
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CLOCKS_LIB = os.path.join(HERE, "libtarang_b200_clocks.so")
PHASES = ["F1", "F2", "B1", "B2", "B3"]


def main(parts):
    import numpy as np

    if not os.path.exists(CLOCKS_LIB):
        raise SystemExit(f"{CLOCKS_LIB} is missing: make -C tarang.jl_b200/csrc clocks")
    os.environ["TARANG_B200_LIB"] = CLOCKS_LIB
    sys.path.insert(0, os.path.dirname(HERE))
    from __graft_entry__ import load_package

    tb = load_package()
    from tarang_b200 import workloads as W
    from tarang_b200._lib import TB_FIELD_B, lib

    import torch

    lib.tb_solve_clocks.restype = ctypes.c_int
    lib.tb_solve_clocks.argtypes = [ctypes.POINTER(ctypes.c_longlong), ctypes.c_int]
    cfg = W.C2
    dom = tb.ChannelDomain(cfg.Nx, cfg.Nz, Lx=cfg.Lx, Lz=cfg.Lz, arch=tb.GPU(0))
    plan = tb.Plan(dom, cfg.kappa, cfg.nu, cfg.Lz, 0.0, 1)
    plan.set_state(TB_FIELD_B, plan.forward(W.rbc_initial_grid(cfg)))
    groups = (cfg.Nx // 2 + 1 + 3) // 4
    out = {}
    for P in parts:
        plan.set_variant(tau_parts=P, xrows=3)
        plan.step(cfg.dt, 3)
        torch.cuda.synchronize()
        n = groups * P * 8
        buf = (ctypes.c_longlong * n)()
        if lib.tb_solve_clocks(buf, n) != 0:
            raise SystemExit("tb_solve_clocks failed")
        a = np.frombuffer(buf, dtype=np.int64).reshape(groups, P, 8).astype(np.float64)
        d = np.diff(a[:, :, :6], axis=2)  # [group][partition][phase]
        total = a[:, :, 5].max(axis=1) - a[:, :, 0].min(axis=1)
        out[P] = {
            "cycles_median_over_groups": float(np.median(total)),
            "phase_cycles_by_partition": {
                k: dict(zip(PHASES, (float(np.median(d[:, k, i])) for i in range(5)))) for k in range(P)
            },
        }
    print(json.dumps(out, indent=1))


if __name__ == "__main__":
    main([int(a) for a in sys.argv[1:]] or [8])
