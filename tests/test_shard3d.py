"""Mode-sharded 3D step on CPU: the partition, the two pencil exchanges and a
whole RK222 step on two gloo ranks, against the single-rank oracle.

Each rank owns a kx range (all ky, all z).  The per-rank kernels are stood in
for by the oracle's pencil-form RHS stages (rhs3_stage_modes / _rows / _back)
and its per-mode tau solves over the rank's modes; the exchanges are the
library's PencilExchange over torch.distributed (gloo here, NCCL on GPUs).
"""
import os
import subprocess
import sys

import numpy as np
import pytest

from __graft_entry__ import ROOT, load_package

load_package()
from tarang_b200 import shard3d as S  # noqa: E402

from oracle.tarang_oracle import (  # noqa: E402
    RBC3D,
    RBC3Params,
    forward_3d,
    padded_length,
    rel_l2,
    rhs3_stage_back,
    rhs3_stage_modes,
    rhs3_stage_rows,
)


def test_split_even_covers_every_index_once():
    for n, w in ((9, 2), (9, 4), (129, 8), (8, 8), (384, 3)):
        r = S.split_even(n, w)
        assert r[0][0] == 0 and r[-1][1] == n and len(r) == w
        assert all(a[1] == b[0] for a, b in zip(r, r[1:]))
        sizes = [h - l for l, h in r]
        assert max(sizes) - min(sizes) <= 1 and min(sizes) >= 1
    with pytest.raises(ValueError):
        S.split_even(3, 4)


def test_pencil_stages_equal_the_oracle_rhs():
    p = RBC3Params(Nx=16, Ny=12, Nz=8, Ra=1e6)
    sim = RBC3D(p)
    rng = np.random.default_rng(3)
    cs = [forward_3d(rng.standard_normal((p.Nz, p.Ny, p.Nx))) for _ in range(4)]
    ref = sim.rhs(*cs)
    got = rhs3_stage_back(sim, rhs3_stage_rows(sim, rhs3_stage_modes(sim, cs, 0)))
    for g, r in zip(got, ref):
        assert rel_l2(g, r) < 1e-13


def test_exchange_index_maps_with_uneven_ranges():
    import torch

    geom = S.PencilGeometry(Nz=3, My=10, Kx=7, world=3)
    full = torch.randn(2, geom.Nz, geom.My, geom.Kx, dtype=torch.complex128)
    rows = _route_all(geom, lambda ex, a: ex.to_rows(a), [full[..., kl:kh].contiguous() for (kl, kh) in geom.kx])
    for r, (yl, yh) in enumerate(geom.rows):
        assert torch.equal(rows[r], full[..., yl:yh, :])
    back = _route_all(geom, lambda ex, b: ex.to_modes(b), rows)
    for r, (kl, kh) in enumerate(geom.kx):
        assert torch.equal(back[r], full[..., kl:kh])
    real = torch.randn(4, geom.Nz, geom.My, geom.Kx, dtype=torch.float32)  # FP32 products (mixed plans)
    rows = _route_all(geom, lambda ex, a: ex.to_rows(a), [real[..., kl:kh].contiguous() for (kl, kh) in geom.kx])
    for r, (yl, yh) in enumerate(geom.rows):
        assert torch.equal(rows[r], real[..., yl:yh, :])
    b = geom.exchange_bytes(arrays=12, itemsize=8)
    assert b["total"] == 12 * 3 * 10 * 7 * 8
    own = sum(12 * 3 * (kh - kl) * (yh - yl) * 8 for (kl, kh), (yl, yh) in zip(geom.kx, geom.rows))
    assert b["between_ranks"] == b["total"] - own


def _route_all(geom, op, inputs):
    """Run `op(exchange, input)` for every rank of `geom` in one process.  A
    first pass records every rank's send buffer; the second pass serves each
    rank's all_to_all from those buffers, as the collective would."""
    import torch

    W = geom.world
    posted = {}
    for r in range(W):
        def record(out, inp, osp, isp, r=r):
            posted[r] = (inp.clone(), list(isp))
        op(S.PencilExchange(geom, r, all_to_all=record), inputs[r])
    outs = []
    for r in range(W):
        def serve(out, inp, osp, isp, r=r):
            pieces = [posted[s][0][sum(posted[s][1][:r]):sum(posted[s][1][:r + 1])] for s in range(W)]
            assert [len(x) for x in pieces] == list(osp)
            out.copy_(torch.cat(pieces))
        outs.append(op(S.PencilExchange(geom, r, all_to_all=serve), inputs[r]))
    return outs


_RANK_CODE = r"""
import os, sys, json
import numpy as np
import torch
import torch.distributed as dist
from __graft_entry__ import load_package
load_package()
from tarang_b200 import shard3d as S
from oracle.tarang_oracle import (RBC3D, RBC3Params, TABLEAUS, rbc3_initial_b, padded_length,
                                  rhs3_stage_modes, rhs3_stage_rows, rhs3_stage_back, cheb_backward, cheb_forward)
import scipy.fft as sfft

dist.init_process_group("gloo")
rank, world = dist.get_rank(), dist.get_world_size()
p = RBC3Params(Nx=16, Ny=12, Nz=8, Ra=1e6)
dt = 0.01
sim = RBC3D(p)
sim.set_b_grid(rbc3_initial_b(p, 42, amp=1e-2))
My = padded_length(p.Ny, p.dealias)
geom = S.PencilGeometry(Nz=p.Nz, My=My, Kx=sim.Kx, world=world)
kl, kh = geom.kx[rank]
ex = S.PencilExchange(geom, rank)
modes = [(iy, ix) for iy in range(p.Ny) for ix in range(kl, kh)]

def rhs_fn():
    loc = [c[..., kl:kh] for c in (sim.b, sim.ux, sim.uy, sim.uz)]
    mod = lambda cs: torch.from_numpy(rhs3_stage_modes(sim, cs, kl))
    rows = lambda t: torch.from_numpy(rhs3_stage_rows(sim, t.numpy()))
    back = lambda t: rhs3_stage_back(sim, t.numpy())
    F = S.sharded_rhs(ex, mod, rows, back, loc)
    out = []
    for f in F:
        full = np.zeros_like(sim.b)
        full[..., kl:kh] = f
        out.append(full)
    return out

def proj_fn(c):
    # the grid round trip of this rank's kx planes (Im dropped at kx = 0 and Nx/2)
    out = np.zeros_like(c)
    t = sfft.ifft(cheb_backward(c[..., kl:kh], axis=0), axis=1)
    ix = np.arange(kl, kh)
    edge = (ix == 0) | (ix == p.Nx // 2)
    t[..., edge] = np.real(t[..., edge])
    out[..., kl:kh] = cheb_forward(sfft.fft(t, axis=1), axis=0)
    return out

for _ in range(2):
    sim.step_rk(dt, TABLEAUS["RK222"], modes=modes, rhs_fn=rhs_fn, proj_fn=proj_fn)
parts = [None] * world
dist.all_gather_object(parts, {f: getattr(sim, f)[..., kl:kh] for f in ("b", "ux", "uy", "uz")})
if rank == 0:
    ref = RBC3D(p)
    ref.set_b_grid(rbc3_initial_b(p, 42, amp=1e-2))
    for _ in range(2):
        ref.step_rk(dt, TABLEAUS["RK222"])
    errs = {}
    for f in ("b", "ux", "uy", "uz"):
        got = np.concatenate([pt[f] for pt in parts], axis=-1)
        want = getattr(ref, f)
        errs[f] = float(np.linalg.norm(got - want) / np.linalg.norm(want))
    print("ERRS", json.dumps(errs))
dist.barrier()
dist.destroy_process_group()
"""


def test_two_gloo_ranks_step_matches_single_rank_oracle():
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1", MASTER_PORT="29651",
                   PYTHONPATH=ROOT)
        procs.append(subprocess.Popen([sys.executable, "-c", _RANK_CODE], env=env, cwd=ROOT,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = [pr.communicate(timeout=300) for pr in procs]
    for pr, (o, e) in zip(procs, outs):
        assert pr.returncode == 0, e[-3000:]
    import json

    line = next(l for l in outs[0][0].splitlines() if l.startswith("ERRS"))
    errs = json.loads(line.split(" ", 1)[1])
    for f, e in errs.items():
        assert e < 1e-12, (f, e)
