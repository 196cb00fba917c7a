"""Mode-sharded 3D Rayleigh-Benard: partition and pencil exchanges.

The reference's distributed subproblem path moves every field between its FFT
pencil and the Chebyshev-local solve pencil (``to_solve_layout!``,
src/core/subsystems/subproblem_io.jl:100-330); its CUDA extension does the
z <-> y <-> x transposes with grouped NCCL send/recv
(ext/cuda/nccl_transpose.jl:418 ``nccl_alltoall!``, :539-940).

Here rank r owns a contiguous range of kx (all ky, all z).  The tau systems
are per (kx, ky) mode, the Chebyshev transforms per (kx, ky) column and the
y FFTs per (kx, z) column, so the solves and those transforms are local.  Only
the x direction of the 3/2-dealiased products needs every kx, so one RHS
evaluation makes two exchanges (one all-to-all each):

  to_rows   after the y-inverse transforms: F arrays [f][z][y][kx in r]
            (y on the 3/2-padded grid, kx spectral) -> [f][z][y in s][kx all]
            for every destination rank s, whose padded y rows are a
            contiguous range;
  to_modes  after the x pass (products, forward x transform, truncation):
            the inverse, P product arrays [f][z][y in s][kx all] ->
            [f][z][y][kx in r].

Every block goes to this rank's own buffers first (``all_to_all_single`` on
torch tensors: NCCL for CUDA tensors, gloo for host tensors); no kernel reads
another GPU's memory.  Bytes per exchange (complex entries of `dtype`):
  to_rows  : F * Nz * My * Kx * itemsize over all ranks,
  to_modes : P * Nz * My * Kx * itemsize,
of which a fraction (world - 1) / world crosses between GPUs; the library's
3D RHS carries F = 12 (value, y and z derivative of b, u_x, u_y, u_z; the x
derivative comes from the x bins in the x pass) and P = 4 arrays in FP32 (mixed
precision) or FP64.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Callable, List, Optional, Sequence, Tuple


def split_even(n: int, world: int) -> List[Tuple[int, int]]:
    """Contiguous [lo, hi) ranges of range(n) over `world` ranks, the first
    n % world ranges one longer.  Every rank gets at least one index."""
    if world < 1 or n < world:
        raise ValueError(f"cannot split {n} indices over {world} ranks")
    base, extra = divmod(n, world)
    out, lo = [], 0
    for r in range(world):
        hi = lo + base + (1 if r < extra else 0)
        out.append((lo, hi))
        lo = hi
    return out


def kx_ranges(Kx: int, world: int) -> List[Tuple[int, int]]:
    """kx columns per rank.  Each kx column holds Ny tau systems of equal
    cost, so an even split of the columns balances the solves and the local
    transforms."""
    return split_even(Kx, world)


def y_ranges(My: int, world: int) -> List[Tuple[int, int]]:
    """Padded y rows of the x pass per rank."""
    return split_even(My, world)


@dataclass(frozen=True)
class PencilGeometry:
    """Sizes of the two pencils: Nz Chebyshev levels, My padded y rows, Kx =
    Nx/2 + 1 kx bins, split over `world` ranks."""

    Nz: int
    My: int
    Kx: int
    world: int

    @property
    def kx(self) -> List[Tuple[int, int]]:
        return kx_ranges(self.Kx, self.world)

    @property
    def rows(self) -> List[Tuple[int, int]]:
        return y_ranges(self.My, self.world)

    def exchange_bytes(self, arrays: int, itemsize: int) -> dict:
        """Total bytes of one exchange of `arrays` complex arrays of `itemsize`
        bytes per entry, and the part that crosses between ranks."""
        total = arrays * self.Nz * self.My * self.Kx * itemsize
        cross = sum(arrays * self.Nz * (kh - kl) * (yh - yl) * itemsize
                    for r, (kl, kh) in enumerate(self.kx) for s, (yl, yh) in enumerate(self.rows) if r != s)
        return {"total": total, "between_ranks": cross}


class PencilExchange:
    """The two all-to-alls of one RHS evaluation on this rank.

    Arrays are torch tensors, complex or real, with the pencil's last two
    axes (y, kx): ``to_rows`` takes [..., My, Kx_r] (this rank's kx range) and
    returns [..., My_r, Kx] (this rank's rows); ``to_modes`` is its inverse.
    The leading axes (fields, z) are carried as they are.  `all_to_all` is
    ``torch.distributed.all_to_all_single`` unless a stand-in is given (one
    process emulating several ranks passes a function that moves the blocks
    between its own buffers)."""

    def __init__(self, geom: PencilGeometry, rank: int, group=None,
                 all_to_all: Optional[Callable] = None):
        self.g, self.rank, self.group = geom, rank, group
        if all_to_all is None:
            import torch.distributed as dist

            def all_to_all(out, inp, out_splits, in_splits):
                dist.all_to_all_single(out, inp, out_splits, in_splits, group=group)

        self._a2a = all_to_all

    @staticmethod
    def _flat(t):
        import torch

        return torch.view_as_real(t).reshape(-1) if t.is_complex() else t.reshape(-1)

    def to_rows(self, a):
        """[..., My, Kx_r] -> [..., My_r, Kx] (blocks to every rank's rows)."""
        import torch

        g, r = self.g, self.rank
        kl, kh = g.kx[r]
        yl, yh = g.rows[r]
        lead = a.shape[:-2]
        assert a.shape[-2:] == (g.My, kh - kl), (a.shape, g.My, kh - kl)
        send = torch.cat([self._flat(a[..., sl:sh, :].contiguous()) for (sl, sh) in g.rows])
        per = 2 if a.is_complex() else 1
        nlead = 1
        for d in lead:
            nlead *= d
        in_splits = [nlead * (sh - sl) * (kh - kl) * per for (sl, sh) in g.rows]
        out_splits = [nlead * (yh - yl) * (ch - cl) * per for (cl, ch) in g.kx]
        recv = torch.empty(sum(out_splits), dtype=send.dtype, device=send.device)
        self._a2a(recv, send, out_splits, in_splits)
        out = torch.empty(lead + (yh - yl, g.Kx), dtype=a.dtype, device=a.device)
        off = 0
        for (cl, ch), n in zip(g.kx, out_splits):
            blk = recv[off:off + n]
            off += n
            shape = lead + (yh - yl, ch - cl)
            out[..., cl:ch] = torch.view_as_complex(blk.reshape(shape + (2,))) if a.is_complex() else blk.reshape(shape)
        return out

    def to_modes(self, b):
        """[..., My_r, Kx] -> [..., My, Kx_r] (the inverse of to_rows)."""
        import torch

        g, r = self.g, self.rank
        kl, kh = g.kx[r]
        yl, yh = g.rows[r]
        lead = b.shape[:-2]
        assert b.shape[-2:] == (yh - yl, g.Kx), (b.shape, yh - yl, g.Kx)
        send = torch.cat([self._flat(b[..., cl:ch].contiguous()) for (cl, ch) in g.kx])
        per = 2 if b.is_complex() else 1
        nlead = 1
        for d in lead:
            nlead *= d
        in_splits = [nlead * (yh - yl) * (ch - cl) * per for (cl, ch) in g.kx]
        out_splits = [nlead * (sh - sl) * (kh - kl) * per for (sl, sh) in g.rows]
        recv = torch.empty(sum(out_splits), dtype=send.dtype, device=send.device)
        self._a2a(recv, send, out_splits, in_splits)
        out = torch.empty(lead + (g.My, kh - kl), dtype=b.dtype, device=b.device)
        off = 0
        for (sl, sh), n in zip(g.rows, out_splits):
            blk = recv[off:off + n]
            off += n
            shape = lead + (sh - sl, kh - kl)
            out[..., sl:sh, :] = torch.view_as_complex(blk.reshape(shape + (2,))) if b.is_complex() else blk.reshape(shape)
        return out


def sharded_rhs(exchange: PencilExchange, stage_modes: Callable, stage_rows: Callable, stage_back: Callable,
                local_coeffs: Sequence):
    """One RHS evaluation of the mode-sharded step: this rank's kx columns go
    through `stage_modes` (Chebyshev backward, projections, y padding and
    inverse y transforms -> [F][z][My][Kx_r]), the rows exchange, `stage_rows`
    (x derivatives, x padding, products, forward x transform and truncation on
    this rank's padded y rows -> [P][z][My_r][Kx]), the modes exchange and
    `stage_back` (forward y transform, y fold and truncation, Chebyshev forward
    -> the F coefficients of this rank's modes).  The stage functions are the
    per-rank kernels (or a CPU stand-in); every collective is in the two
    exchanges, in the same order on every rank."""
    a = stage_modes(local_coeffs)
    rows = exchange.to_rows(a)
    prods = stage_rows(rows)
    back = exchange.to_modes(prods)
    return stage_back(back)
