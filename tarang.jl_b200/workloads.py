"""Seeded synthetic workloads for the benchmark configurations.

The reference seeds its initial noise with Julia's RNG
(src/core/field/field_layout/field_layout_operations.jl:34-60), which cannot be
reproduced here; these workloads draw the same kind of noise from NumPy's
PCG64 so that the CPU oracle and the library see identical arrays.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Optional

import numpy as np


@dataclass
class RBCConfig:
    """2D Rayleigh-Benard: ChannelDomain(Nx, Nz; Lx, Lz), Boussinesq with tau/lift BCs."""

    Nx: int = 1024
    Nz: int = 256
    Lx: float = 4.0
    Lz: float = 1.0
    Ra: float = 1e8
    Pr: float = 1.0
    dt: float = 0.01
    scheme: str = "RK443"
    seed: int = 42
    noise: float = 1e-3

    @property
    def kappa(self) -> float:  # free-fall scaling, test/test_subproblem_rk.jl:23-24
        return (self.Ra * self.Pr) ** -0.5

    @property
    def nu(self) -> float:
        return (self.Ra / self.Pr) ** -0.5


C1 = RBCConfig(Nx=256, Nz=64, Ra=2e6, dt=0.125, scheme="RK222")
C2 = RBCConfig(Nx=1024, Nz=256, Ra=1e8, dt=0.01, scheme="RK443")


def rbc_initial_grid(cfg: RBCConfig) -> np.ndarray:
    """b0 = Lz - z + noise * z (Lz - z) xi on the (Nz, Nx) grid, xi ~ N(0,1) from PCG64(seed)."""
    rng = np.random.default_rng(cfg.seed)
    xi = rng.standard_normal((cfg.Nx, cfg.Nz)).T
    z = (cfg.Lz / 2.0 * (1.0 - np.cos(np.pi * np.arange(cfg.Nz) / (cfg.Nz - 1))))[:, None]
    return (cfg.Lz - z) + cfg.noise * z * (cfg.Lz - z) * xi


def state_bytes(cfg: RBCConfig) -> int:
    """Bytes of the coefficient state (b, ux, uz, p and 7 taus), complex128."""
    nk = cfg.Nx // 2 + 1
    return 16 * (4 * cfg.Nz * nk + 7 * nk)


TABLEAU_PATTERNS = {
    # (AE nonzero pattern, AI nonzero pattern, bE, bI) of src/core/timesteppers/types.jl:49-167
    "RK222": (
        [[0, 0, 0], [1, 0, 0], [1, 1, 0]],
        [[0, 0, 0], [0, 1, 0], [0, 1, 1]],
        [0, 1, 1],
        [0, 1, 1],
    ),
    "RK443": (
        [[0, 0, 0, 0], [1, 0, 0, 0], [1, 1, 0, 0], [1, 1, 1, 0]],
        [[0, 0, 0, 0], [0, 1, 0, 0], [0, 1, 1, 0], [0, 1, 1, 1]],
        [0, 1, 1, 1],
        [0, 1, 1, 1],
    ),
}


def step_model_bytes(cfg: RBCConfig, scheme: str) -> float:
    """Algorithmic HBM bytes of one step under the hot-path byte model.

    C = one complex coefficient field, V = one equation-space vector over all
    modes, Phi = the per-mode bordered-banded LHS at nominal size (n*848 B).
    Per stage: read MX0, read every F_j / LX_j with a nonzero tableau entry,
    read Phi if a_ii != 0, write X_i, RHS reads the 3 advected fields and
    writes 3 F fields; if L X_i is used later: read X_i, read Phi, write LX_i.
    Plus the pre-stage M X_n (2V) and the final update.  SBDF2: one RHS,
    one solve and the history terms.
    """
    nk = cfg.Nx // 2 + 1
    n = 4 * cfg.Nz + 7
    C = nk * cfg.Nz * 16.0
    V = nk * n * 16.0
    Phi = nk * n * 848.0
    if scheme == "SBDF2":
        # nominal multistep count: the RHS (6C), the solve and the L X history term
        # each read Phi, plus the state / history / F vectors (12 V)
        return 2 * Phi + 12 * V + 6 * C
    AE, AI, bE, bI = TABLEAU_PATTERNS[scheme]
    s = len(bE)
    total = 2 * V
    for i in range(s):
        total += V
        for j in range(i):
            total += V * (AE[i][j] + AI[i][j])
        if AI[i][i]:
            total += Phi
        total += V + 6 * C
        used_later = any(AI[k][i] for k in range(i + 1, s)) or bI[i]
        if used_later:
            total += 2 * V + Phi
    total += V + sum(V * (bE[j] + bI[j]) for j in range(s)) + 2 * V
    return total


@dataclass
class RBC3Config:
    """3D Rayleigh-Benard: RealFourier x, y x ChebyshevT z (ChannelDomain3D-style, z in [0, Lz])."""

    Nx: int = 256
    Ny: int = 256
    Nz: int = 128
    Lx: float = 4.0
    Ly: float = 4.0
    Lz: float = 1.0
    Ra: float = 1e7
    Pr: float = 1.0
    dt: float = 5e-3
    scheme: str = "RK222"
    steps: int = 50
    seed: int = 42
    noise: float = 1e-3

    @property
    def kappa(self) -> float:
        return (self.Ra * self.Pr) ** -0.5

    @property
    def nu(self) -> float:
        return (self.Ra / self.Pr) ** -0.5


C3 = RBC3Config()


def rbc3_initial_grid(cfg: RBC3Config) -> np.ndarray:
    """b0 = Lz - z + noise * z (Lz - z) xi on the (Nz, Ny, Nx) grid, xi ~ N(0,1)
    from PCG64(seed) drawn in Julia (x, y, z) order."""
    rng = np.random.default_rng(cfg.seed)
    xi = rng.standard_normal((cfg.Nx, cfg.Ny, cfg.Nz)).transpose(2, 1, 0)
    z = (cfg.Lz / 2.0 * (1.0 - np.cos(np.pi * np.arange(cfg.Nz) / (cfg.Nz - 1))))[:, None, None]
    return (cfg.Lz - z) + cfg.noise * z * (cfg.Lz - z) * xi


def step_model_bytes3(cfg: RBC3Config) -> float:
    """The byte model of step_model_bytes for the 3D system: modes (Nx/2+1) Ny,
    n = 5 Nz + 9 per mode, and the RHS reads the 4 advected fields and writes
    4 F fields (8 C per stage)."""
    nk = (cfg.Nx // 2 + 1) * cfg.Ny
    n = 5 * cfg.Nz + 9
    C = nk * cfg.Nz * 16.0
    V = nk * n * 16.0
    Phi = nk * n * 848.0
    AE, AI, bE, bI = TABLEAU_PATTERNS[cfg.scheme]
    s = len(bE)
    total = 2 * V
    for i in range(s):
        total += V
        for j in range(i):
            total += V * (AE[i][j] + AI[i][j])
        if AI[i][i]:
            total += Phi
        total += V + 8 * C
        if any(AI[k][i] for k in range(i + 1, s)) or bI[i]:
            total += 2 * V + Phi
    total += V + sum(V * (bE[j] + bI[j]) for j in range(s)) + 2 * V
    return total


# ---------------------------------------------------------------------------
# Batched ensemble: independent 2D RBC instances of uneven size.
# ---------------------------------------------------------------------------
ENSEMBLE_SIZES = ((128, 32), (256, 64), (384, 96), (512, 128))


def ensemble_members(n: int = 64, seed: int = 7, dt: float = 0.02, scheme: str = "RK222"):
    """Ensemble configuration: (Nx, Nz) drawn by seed from ENSEMBLE_SIZES, Ra
    log-uniform in [1e5, 1e8], Pr uniform in [0.7, 7]; member k gets noise seed
    1000 + k.  One dt for all members (free-fall units, well inside the
    advective limit of the first 100 steps from rest)."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        Nx, Nz = ENSEMBLE_SIZES[int(rng.integers(len(ENSEMBLE_SIZES)))]
        Ra = float(10.0 ** rng.uniform(5.0, 8.0))
        Pr = float(rng.uniform(0.7, 7.0))
        out.append(RBCConfig(Nx=Nx, Nz=Nz, Ra=Ra, Pr=Pr, dt=dt, scheme=scheme, seed=1000 + k))
    return out


# ---------------------------------------------------------------------------
# Serving mix: Poisson arrivals of RBC channel runs and 2D decaying turbulence.
# ---------------------------------------------------------------------------
TURB_SIZES = (256, 512, 1024)


@dataclass
class ServeRequest:
    kind: str          # "rbc" or "turb"
    arrival_s: float   # arrival time from the start of the replay
    nsteps: int
    rbc: Optional[RBCConfig] = None
    N: int = 0         # turbulence grid N x N
    nu: float = 1e-4
    dt: float = 2e-3
    seed: int = 0


def serving_requests(n: int = 60, seed: int = 11, rate: float = 20.0, rbc_frac: float = 0.7):
    """Seeded Poisson arrivals (mean `rate` per second): 70 % RBC channel runs
    with the ensemble's sizes and parameter ranges, 30 % FP32 decaying
    turbulence N x N, N in TURB_SIZES (nu = 1e-4, dt = 2e-3, k^-3 spectrum with
    a per-request seed); each request runs a uniform 50-500 steps."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for k in range(n):
        t += float(rng.exponential(1.0 / rate))
        steps = int(rng.integers(50, 501))
        if rng.uniform() < rbc_frac:
            Nx, Nz = ENSEMBLE_SIZES[int(rng.integers(len(ENSEMBLE_SIZES)))]
            Ra = float(10.0 ** rng.uniform(5.0, 8.0))
            Pr = float(rng.uniform(0.7, 7.0))
            cfg = RBCConfig(Nx=Nx, Nz=Nz, Ra=Ra, Pr=Pr, dt=0.02, scheme="RK222", seed=5000 + k)
            out.append(ServeRequest("rbc", t, steps, rbc=cfg, dt=cfg.dt, seed=cfg.seed))
        else:
            N = TURB_SIZES[int(rng.integers(len(TURB_SIZES)))]
            out.append(ServeRequest("turb", t, steps, N=N, seed=7000 + k))
    return out


def turb_initial_spec(N: int, seed: int, amp: float = 10.0) -> np.ndarray:
    """Vorticity coefficients (N, N/2+1) with a k^-3 energy spectrum: |q^| ~ 1/k
    per mode for 1 <= |k| <= N/3, random phases from PCG64(seed), scaled to
    max |q| = amp on the grid (rfft along x, fft along y, unnormalised)."""
    rng = np.random.default_rng(seed)
    kx = np.arange(N // 2 + 1)[None, :]
    ky = np.concatenate([np.arange(N // 2), np.arange(-(N // 2), 0)])[:, None]
    k = np.sqrt(kx ** 2 + ky ** 2)
    mag = np.where((k >= 1.0) & (k <= N / 3.0), 1.0 / np.maximum(k, 1e-30), 0.0)
    phase = rng.uniform(0.0, 2 * np.pi, size=mag.shape)
    g = np.fft.irfft(np.fft.ifft(mag * np.exp(1j * phase), axis=0), n=N, axis=1)
    g *= amp / np.abs(g).max()
    return np.fft.fft(np.fft.rfft(g, axis=1), axis=0)


# ---------------------------------------------------------------------------
# Instance sharding across GPUs (independent solves, no data-path collective)
# ---------------------------------------------------------------------------
def instance_cost(item) -> float:
    """Relative device work of one independent instance: the byte model of one
    step times the steps it runs (RBCConfig members run `steps` given by the
    caller; ServeRequest carries its own)."""
    if isinstance(item, ServeRequest):
        if item.kind == "rbc":
            return step_model_bytes(item.rbc, "RK222") * item.nsteps
        M = 3 * item.N // 2
        return 12.0 * 8.0 * M * M * item.nsteps  # padded FP32 planes moved per step
    return step_model_bytes(item, item.scheme)


def shard_instances(costs, world: int):
    """Longest-processing-time assignment of independent instances to `world`
    ranks: instances in decreasing cost (index breaks ties) each go to the rank
    with the least assigned cost (lowest rank breaks ties).  Deterministic, so
    every rank computes the same partition without communicating; returns one
    ascending index list per rank."""
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = [0.0] * world
    out = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += float(costs[i])
    return [sorted(x) for x in out]


def combine_ensemble(parts):
    """Whole-job ensemble figures from per-rank parts (dicts with steps,
    total_ms, ms (per-member completion), plain_s, plain_done_ms): instance
    steps over the slowest rank's time, percentiles over all members."""
    steps = sum(p["steps"] for p in parts)
    total_ms = max(p["total_ms"] for p in parts)
    plain_s = max(p["plain_s"] for p in parts)
    ms = np.concatenate([np.asarray(p["ms"], dtype=np.float64) for p in parts])
    done = np.concatenate([np.asarray(p["plain_done_ms"], dtype=np.float64) for p in parts])
    return {
        "value": steps / (total_ms / 1e3),
        "plain_value": steps / plain_s,
        "total_ms": total_ms,
        "p50_ms": float(np.percentile(ms, 50)),
        "p99_ms": float(np.percentile(ms, 99)),
        "plain_p50_ms": float(np.percentile(done, 50)),
        "plain_p99_ms": float(np.percentile(done, 99)),
        "members": int(ms.size),
    }


def combine_serving(parts):
    """Whole-job serving figures from per-rank replays (dicts with completed,
    steps, wall_s, tts_ms list): requests and request-steps per second over the
    slowest rank's wall time, time-to-solution percentiles over all requests."""
    wall = max(p["wall_s"] for p in parts)
    tts = np.concatenate([np.asarray(p["tts_ms"], dtype=np.float64) for p in parts])
    completed = sum(p["completed"] for p in parts)
    return {
        "solves_per_s": completed / wall,
        "steps_per_s": sum(p["steps"] for p in parts) / wall,
        "p50_ms": float(np.percentile(tts, 50)) if tts.size else None,
        "p99_ms": float(np.percentile(tts, 99)) if tts.size else None,
        "completed": completed,
        "wall_s": wall,
    }
