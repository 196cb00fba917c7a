"""CPU oracle for the Tarang.jl IMEX timestep hot path (TEST INFRASTRUCTURE ONLY).

This module restates, in NumPy/SciPy Float64, the algorithm Tarang.jl v1.0.73 runs
on its CPU path for a RealFourier(x) x ChebyshevT(z) tau problem, specialised to
the 2D Boussinesq Rayleigh-Benard system of ``test/test_subproblem_rk.jl:50-57``.
It is the checker for the CUDA library and is imported only by ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` / reference leg of
``bench.py``.  Nothing in the shipped library imports or calls it.

Parity status: the reference is Julia (FFTW + SuiteSparse) and cannot run in
this environment, so the oracle is pinned against the reference's own analytic
known-answer tests (transform round trips, spectral derivatives, 3/2-dealiased
products, tau-method boundary enforcement, the tau_method.md Poisson quick
start) which ``tests/test_oracle_known_answers.py`` re-runs.  Bitwise FFTW
rounding is not reproduced; every comparison is a relative tolerance.

Array layout follows the reference's column-major storage exactly: a grid
field of logical size (Nx, Nz) is a NumPy array of shape (Nz, Nx) in C order,
a coefficient field (Nx/2+1, Nz) is shape (Nz, Nk).  Axis 1 is x, axis 0 is z.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np
import scipy.fft as sfft
import scipy.linalg as sla
import scipy.sparse as sps
import scipy.sparse.linalg as spsl

# ---------------------------------------------------------------------------
# Host threads.  The reference runs FFTW with TARANG_FFTW_THREADS threads and
# Julia tasks (src/core/runtime/runtime_init.jl:24-57); here pocketfft takes
# ``workers`` threads and the per-mode loops (independent sparse solves and
# mat-vecs, which release the GIL inside SuperLU) run on a thread pool.  The
# arithmetic of every mode is the same whatever the thread count.
# ---------------------------------------------------------------------------
_WORKERS = 1
_POOL = None


def set_threads(n: int) -> int:
    """Use n host threads for FFTs and per-mode loops (1 = serial); returns n."""
    global _WORKERS, _POOL
    n = max(1, int(n))
    if _POOL is not None:
        _POOL.shutdown(wait=True)
        _POOL = None
    _WORKERS = n
    if n > 1:
        from concurrent.futures import ThreadPoolExecutor

        _POOL = ThreadPoolExecutor(max_workers=n)
    return n


def get_threads() -> int:
    return _WORKERS


def _pmap(fn, items) -> list:
    """[fn(x) for x in items], on the thread pool when one is set."""
    items = list(items)
    if _POOL is None or len(items) < 2:
        return [fn(x) for x in items]
    nchunk = min(len(items), 4 * _WORKERS)
    bounds = [len(items) * i // nchunk for i in range(nchunk + 1)]
    parts = _POOL.map(lambda i: [fn(x) for x in items[bounds[i] : bounds[i + 1]]], range(nchunk))
    return [y for part in parts for y in part]


class _FFTThreads:
    """scipy.fft with the current worker count (same pocketfft arithmetic)."""

    def __getattr__(self, name):
        f = getattr(sfft, name)

        def call(*args, **kw):
            kw.setdefault("workers", _WORKERS)
            return f(*args, **kw)

        return call


_fx = _FFTThreads()

# ---------------------------------------------------------------------------
# Grids and wavenumbers
# ---------------------------------------------------------------------------


def fourier_grid(N: int, L: float, x0: float = 0.0) -> np.ndarray:
    """x_j = x0 + j L/N  (src/core/basis/basis_interface.jl:81-98, _native_grid(::RealFourier))."""
    return x0 + np.arange(N) * (L / N)


def cheb_grid(N: int, a: float, b: float) -> np.ndarray:
    """Gauss-Lobatto z_j = a + (b-a)/2 (1 - cos(pi j/(N-1)))  (basis_interface.jl:107-121).

    The native grid is -cos(pi k/(N-1)), so z_0 = a (bottom wall) and z_{N-1} = b.
    """
    native = -np.cos(np.pi * np.arange(N) / (N - 1))
    return (b - a) / 2.0 * native + (b + a) / 2.0


def wavenumbers_rfft(N: int, L: float) -> np.ndarray:
    """k = 2pi/L [0..N/2]  (src/core/basis/basis_wavenumbers.jl:68-79)."""
    return (2.0 * np.pi / L) * np.arange(N // 2 + 1)


# ---------------------------------------------------------------------------
# Transforms (reference conventions)
# ---------------------------------------------------------------------------


def cheb_forward(g: np.ndarray, axis: int = 0) -> np.ndarray:
    """ChebyshevT forward: REDFT00, x1/(N-1), halve both endpoints, flip odd degrees.

    src/core/transforms/transform_chebyshev.jl:135-183.  Complex input is
    transformed as separate real and imaginary parts (the same thing, since the
    map is real-linear).
    """
    N = g.shape[axis]
    out = sfft.dct(np.real(g), type=1, axis=axis, workers=_WORKERS) + (
        1j * sfft.dct(np.imag(g), type=1, axis=axis, workers=_WORKERS) if np.iscomplexobj(g) else 0.0
    )
    out = np.asarray(out) / (N - 1)
    sl = [slice(None)] * out.ndim
    sl[axis] = 0
    out[tuple(sl)] *= 0.5
    sl[axis] = N - 1
    out[tuple(sl)] *= 0.5
    sl[axis] = slice(1, None, 2)
    out[tuple(sl)] *= -1.0
    return out


def cheb_backward(c: np.ndarray, axis: int = 0) -> np.ndarray:
    """ChebyshevT backward: flip odd, double endpoints, REDFT00, /2 (transform_chebyshev.jl:187-244)."""
    N = c.shape[axis]
    s = np.array(c, dtype=c.dtype, copy=True)
    sl = [slice(None)] * s.ndim
    sl[axis] = slice(1, None, 2)
    s[tuple(sl)] *= -1.0
    sl[axis] = 0
    s[tuple(sl)] *= 2.0
    sl[axis] = N - 1
    s[tuple(sl)] *= 2.0
    out = sfft.dct(np.real(s), type=1, axis=axis, workers=_WORKERS) + (
        1j * sfft.dct(np.imag(s), type=1, axis=axis, workers=_WORKERS) if np.iscomplexobj(s) else 0.0
    )
    return np.asarray(out) / 2.0


def forward_2d(g: np.ndarray) -> np.ndarray:
    """Grid (Nz, Nx) real -> coefficients (Nz, Nx/2+1) complex.

    RealFourier first (unnormalised rfft, transform_fourier.jl:7-31), then
    ChebyshevT along z (the reference's forward order, mixed_transforms.jl:229-330).
    """
    return cheb_forward(_fx.rfft(g, axis=1), axis=0)


def backward_2d(c: np.ndarray, Nx: int) -> np.ndarray:
    """Coefficients (Nz, Nk) -> grid (Nz, Nx).  irfft divides by N and, like
    FFTW's c2r, ignores the imaginary parts of the DC and Nyquist bins
    (transform_fourier.jl:287-313)."""
    return _fx.irfft(cheb_backward(c, axis=0), n=Nx, axis=1)


# ---------------------------------------------------------------------------
# Chebyshev operators in the T basis
# ---------------------------------------------------------------------------


def cheb_diff_matrix(N: int, L: float) -> np.ndarray:
    """Dense T->T first-derivative matrix, scaled by 2/L.

    Row 0 weight j, rows k>=1 weight 2j, nonzero only for j>k with j-k odd
    (basis_operators.jl:826-853; scaling :754-770).
    """
    D = np.zeros((N, N))
    for k in range(N - 1):
        for j in range(k + 1, N):
            if (j - k) % 2 == 1:
                D[k, j] = float(j) if k == 0 else 2.0 * j
    return D * (2.0 / L)


def cheb_eval_row(N: int, zeta: float) -> np.ndarray:
    """Row T_n(zeta), zeta in [-1,1] (the stored-basis Interpolate row,
    matrices_subproblem_operators.jl:263-308)."""
    return np.cos(np.arange(N) * np.arccos(np.clip(zeta, -1.0, 1.0)))


def cheb_integ_row(N: int, L: float) -> np.ndarray:
    """w_n = int_0^L T_n dz = L/2 * 2/(1-n^2) for even n, 0 for odd n.

    The reference builds it by quadrature (matrices_subproblem_operators.jl:353-364);
    the odd entries come out at round-off level and are removed by the 1e-12 entry
    cutoff (subproblem_matrix_build.jl:88-100), so the exact row is used here.
    """
    w = np.zeros(N)
    for n in range(0, N, 2):
        w[n] = L / 2.0 * 2.0 / (1.0 - n * n)
    return w


# ---------------------------------------------------------------------------
# 3/2-dealiased product (nonlinear_padding.jl:58-443)
# ---------------------------------------------------------------------------


def padded_length(N: int, factor: float = 1.5) -> int:
    """M = ceil(factor N), bumped to even (nonlinear_padding.jl:103-108)."""
    M = int(math.ceil(factor * N))
    if M % 2 == 1:
        M += 1
    return M


def padded_multiply(a: np.ndarray, b: np.ndarray, factor: float = 1.5) -> np.ndarray:
    """Grid (Nz, Nx) x grid (Nz, Nx) -> dealiased product on the same grid.

    Full complex FFT along x, zero-pad N->M with the even-N Nyquist bin split
    X/2 at +-N/2, inverse FFT, multiply, forward FFT, fold -N/2 back into the
    Nyquist bin, truncate, inverse FFT on N points, real part times M/N
    (nonlinear_padding.jl:182-226, 294-346, 359-443).  The Chebyshev axis is not
    padded (:86-103).
    """
    N = a.shape[1]
    if N <= 4:
        raise ValueError("padded product is skipped by the reference for N <= 4")
    M = padded_length(N, factor)
    Nh = N // 2
    n_neg = N - Nh - 1

    def pad(x):
        s = _fx.fft(x.astype(complex), axis=1)
        p = np.zeros((x.shape[0], M), dtype=complex)
        p[:, : Nh + 1] = s[:, : Nh + 1]
        if n_neg > 0:
            p[:, M - n_neg :] = s[:, N - n_neg :]
        if N % 2 == 0 and M > N:
            p[:, Nh] *= 0.5
            p[:, M - Nh] = p[:, Nh]
        return _fx.ifft(p, axis=1)

    prod = pad(a) * pad(b)
    P = _fx.fft(prod, axis=1)
    if N % 2 == 0 and M > N:
        P[:, Nh] += P[:, M - Nh]
    R = np.zeros((a.shape[0], N), dtype=complex)
    R[:, : Nh + 1] = P[:, : Nh + 1]
    if n_neg > 0:
        R[:, N - n_neg :] = P[:, M - n_neg :]
    r = _fx.ifft(R, axis=1)
    return np.real(r) * (M / N)


# ---------------------------------------------------------------------------
# 2D Rayleigh-Benard tau problem
# ---------------------------------------------------------------------------

# Tableaus (src/core/timesteppers/types.jl:49-167)
_G2 = 1.0 - 1.0 / math.sqrt(2.0)
RK222 = dict(
    name="RK222",
    AE=np.array([[0.0, 0.0, 0.0], [_G2, 0.0, 0.0], [_G2, 1.0 - _G2, 0.0]]),
    AI=np.array([[0.0, 0.0, 0.0], [0.0, _G2, 0.0], [0.0, 1.0 - _G2, _G2]]),
    bE=np.array([0.0, 1.0 - _G2, _G2]),
    bI=np.array([0.0, 1.0 - _G2, _G2]),
    c=np.array([0.0, _G2, 1.0]),
)
_G3 = 0.4358665215084590
RK443 = dict(
    name="RK443",
    AE=np.array(
        [
            [0.0, 0.0, 0.0, 0.0],
            [0.4358665215084590, 0.0, 0.0, 0.0],
            [0.3212788860285571, 0.3966543747256624, 0.0, 0.0],
            [-0.105858296071263, 0.5529291479590279, 0.5529291481122351, 0.0],
        ]
    ),
    AI=np.array(
        [
            [0.0, 0.0, 0.0, 0.0],
            [0.0, _G3, 0.0, 0.0],
            [0.0, 0.2820667392457805, _G3, 0.0],
            [0.0, 1.208496649176010, -0.6443631706844688, _G3],
        ]
    ),
    bE=np.array([0.0, 1.208496649176010, -0.6443631706844688, 0.4358665215084590]),
    bI=np.array([0.0, 1.208496649176010, -0.6443631706844688, _G3]),
    c=np.array([0.0, _G3, 0.7179332607542195, 1.0]),
)
TABLEAUS = {"RK222": RK222, "RK443": RK443}


def sbdf_coefs(order: int, dt: float, dt_prev: Optional[float] = None):
    """SBDF1/SBDF2 (a, b, c) tuples (step_subproblem_multistep.jl:536-553)."""
    if order == 1:
        return (1.0 / dt, -1.0 / dt), (1.0,), (0.0, 1.0)
    w1 = dt / (dt if dt_prev is None else dt_prev)
    a = ((1.0 + 2.0 * w1) / ((1.0 + w1) * dt), -(1.0 + w1) / dt, w1 * w1 / ((1.0 + w1) * dt))
    return a, (1.0,), (0.0, 1.0 + w1, -w1)


@dataclass
class RBCParams:
    Nx: int
    Nz: int
    Lx: float = 4.0
    Lz: float = 1.0
    Ra: float = 2e6
    Pr: float = 1.0
    dealias: float = 1.5
    b_bottom: float = None  # value of b at z=0 (defaults to Lz)
    b_top: float = 0.0

    @property
    def kappa(self) -> float:
        return (self.Ra * self.Pr) ** -0.5

    @property
    def nu(self) -> float:
        return (self.Ra / self.Pr) ** -0.5

    def bottom(self) -> float:
        return self.Lz if self.b_bottom is None else self.b_bottom


def rbc_initial_b(p: RBCParams, seed: int = 42, amp: float = 1e-3) -> np.ndarray:
    """b0 = Lz - z + amp z (Lz - z) xi on the (x,z) grid, xi ~ N(0,1) from PCG64(seed).

    The reference draws xi with Julia's RNG (field_layout_operations.jl:34-60),
    which cannot be reproduced here; this seeded NumPy draw is fed identically to
    the oracle and to the CUDA library.  Returned in grid layout (Nz, Nx).
    """
    rng = np.random.default_rng(seed)
    xi = rng.standard_normal((p.Nx, p.Nz)).T  # (Nz, Nx), drawn in Julia (x,z) order
    z = cheb_grid(p.Nz, 0.0, p.Lz)[:, None]
    return (p.Lz - z) + amp * z * (p.Lz - z) * xi


class RBC2D:
    """Per-Fourier-mode tau system and IMEX steppers for 2D Boussinesq RBC.

    Unknown order inside one mode vector (the oracle's own; the reference's
    pre_right permutation only reorders):
        [p(Nz), b(Nz), ux(Nz), uz(Nz), tau_p, tau_b1, tau_b2, tau_u1x, tau_u1z, tau_u2x, tau_u2z]
    with tau_p present only at kx = 0 (valid-mode filtering,
    subproblem_matrix_build.jl:102-168).  Equation order:
        [continuity(Nz), b(Nz), u_x(Nz), u_z(Nz),
         b(z=0), u_x(z=0), u_z(z=0), b(z=Lz), u_x(z=Lz), u_z(z=Lz), integ(p)]
    with integ(p) present only at kx = 0.
    """

    TAU_NAMES = ("tau_p", "tau_b1", "tau_b2", "tau_u1x", "tau_u1z", "tau_u2x", "tau_u2z")

    def __init__(self, p: RBCParams):
        self.p = p
        Nx, Nz = p.Nx, p.Nz
        self.Nk = Nx // 2 + 1
        self.kx = wavenumbers_rfft(Nx, p.Lx)
        self.D = cheb_diff_matrix(Nz, p.Lz)
        self.D2 = self.D @ self.D
        self.z = cheb_grid(Nz, 0.0, p.Lz)
        self._mats: Dict[int, Tuple[np.ndarray, np.ndarray, np.ndarray, np.ndarray]] = {}
        self._lu: Dict[Tuple[int, float, float], tuple] = {}
        # state: coefficient fields (Nz, Nk) complex, taus (7, Nk) complex
        self.b = np.zeros((Nz, self.Nk), complex)
        self.ux = np.zeros_like(self.b)
        self.uz = np.zeros_like(self.b)
        self.pr = np.zeros_like(self.b)
        self.tau = np.zeros((7, self.Nk), complex)
        self.sim_time = 0.0
        self.iteration = 0
        self._ms_hist: List[Tuple[np.ndarray, np.ndarray]] = []  # SBDF (MX, F) history, newest first
        self._ms_dt_prev: Optional[float] = None
        # dynamic wall values of b: t -> (bottom, top) coefficient arrays (Nk,),
        # re-gathered into the BC rows at every stage time (None: constant BCs)
        self.wall_b = None

    def _stage_algf(self, m: int, algf: np.ndarray, t: float) -> np.ndarray:
        """ALG_F at time t: the b wall rows take the wall profile's coefficients
        (per-stage refresh of step_subproblem_rk.jl:547-560, gather_alg_F!
        subproblem_rhs.jl:523-607)."""
        if self.wall_b is None:
            return algf
        bot, top = self.wall_b(t)
        out = algf.copy()
        r_bc = 4 * self.p.Nz
        out[r_bc + 0] = bot[m]
        out[r_bc + 3] = top[m]
        return out

    # -- per-mode matrices (subproblem_matrix_build.jl:11-309) --------------
    def n_unknowns(self, m: int) -> int:
        return 4 * self.p.Nz + (7 if m == 0 else 6)

    def mode_matrices(self, m: int):
        """Sparse (CSR) M, L (complex), BC-row index list and ALG_F for Fourier mode m.

        Same entries the reference's build_matrices! assembles for this system
        (matrices_subproblem_operators.jl:19-330), including the 1e-12 entry
        cutoff applied to every block entry (subproblem_matrix_build.jl:88-100).
        """
        if m in self._mats:
            return self._mats[m]
        p = self.p
        N = p.Nz
        kx = self.kx[m]
        ikx = 1j * kx
        has_tp = m == 0
        ntau = 7 if has_tp else 6
        n = 4 * N + ntau
        cp, cb, cux, cuz = 0, N, 2 * N, 3 * N
        names = self.TAU_NAMES if has_tp else self.TAU_NAMES[1:]
        tcol = {nm: 4 * N + i for i, nm in enumerate(names)}
        rc, rb, rx, rz, r_bc = 0, N, 2 * N, 3 * N, 4 * N
        kap, nu = p.kappa, p.nu
        Lr, Lc, Lv = [], [], []
        idx = np.arange(N)
        dr, dc = np.nonzero(self.D)
        d2r, d2c = np.nonzero(self.D2)
        De = self.D[:, N - 1]
        der = np.nonzero(De)[0]

        def add(r0, c0, rr, cc, vv):
            vv = np.broadcast_to(np.asarray(vv, dtype=complex), np.shape(rr))
            keep = np.abs(vv) >= 1e-12  # entry cutoff
            Lr.append(r0 + np.asarray(rr)[keep])
            Lc.append(c0 + np.asarray(cc)[keep])
            Lv.append(vv[keep])

        def lap_block(r0, c0, coef):
            # coef * (-kx^2 I + D2): diagonal and strictly-upper parts are disjoint
            add(r0, c0, idx, idx, -coef * kx * kx * np.ones(N))
            add(r0, c0, d2r, d2c, coef * self.D2[d2r, d2c])

        # trace(grad_u) + tau_p = 0
        add(rc, cux, idx, idx, ikx * np.ones(N))
        add(rc, cuz, dr, dc, self.D[dr, dc])
        add(rc, tcol["tau_u1z"], [N - 1], [0], [1.0])
        if has_tp:
            add(rc, tcol["tau_p"], [0], [0], [1.0])  # 0-D field -> T_0 row (subproblem_expr_helpers.jl:189-193)
        # dt(b) - kappa div(grad_b) + lift(tau_b2) = -u.grad(b)
        lap_block(rb, cb, -kap)
        add(rb, tcol["tau_b1"], der, np.zeros_like(der), -kap * De[der])
        add(rb, tcol["tau_b2"], [N - 1], [0], [1.0])
        # dt(u) - nu div(grad_u) + grad(p) - b ez + lift(tau_u2) = -u.grad(u)
        lap_block(rx, cux, -nu)
        add(rx, tcol["tau_u1x"], der, np.zeros_like(der), -nu * De[der])
        add(rx, cp, idx, idx, ikx * np.ones(N))
        add(rx, tcol["tau_u2x"], [N - 1], [0], [1.0])
        lap_block(rz, cuz, -nu)
        add(rz, tcol["tau_u1z"], der, np.zeros_like(der), -nu * De[der])
        add(rz, cp, dr, dc, self.D[dr, dc])
        add(rz, cb, idx, idx, -np.ones(N))
        add(rz, tcol["tau_u2z"], [N - 1], [0], [1.0])
        # boundary conditions: T_n(-1) at z=0, T_n(1) at z=Lz (Interpolate rows)
        bot = cheb_eval_row(N, -1.0)
        top = cheb_eval_row(N, 1.0)
        zero = np.zeros(N, int)
        for i, (col, row) in enumerate(((cb, bot), (cux, bot), (cuz, bot), (cb, top), (cux, top), (cuz, top))):
            add(r_bc + i, col, zero, idx, row)
        bc_rows = list(range(r_bc, r_bc + 6))
        alg_f = np.zeros(n, complex)
        if m == 0:
            # constant BC value v projects to v*Nx at kx=0 (subproblem_rhs.jl:99-115)
            alg_f[r_bc + 0] = p.bottom() * p.Nx
            alg_f[r_bc + 3] = p.b_top * p.Nx
            # integ(p) = 0 : Lx * int T_n dz
            add(r_bc + 6, cp, zero, idx, p.Lx * cheb_integ_row(N, p.Lz))
            bc_rows.append(r_bc + 6)
        L = sps.coo_matrix((np.concatenate(Lv), (np.concatenate(Lr), np.concatenate(Lc))), shape=(n, n)).tocsr()
        L.sum_duplicates()
        Mi = np.concatenate([cb + idx, cux + idx, cuz + idx])
        Mr = np.concatenate([rb + idx, rx + idx, rz + idx])
        M = sps.coo_matrix((np.ones(3 * N, complex), (Mr, Mi)), shape=(n, n)).tocsr()
        out = (M, L, np.array(bc_rows), alg_f)
        self._mats[m] = out
        return out

    def dense_mode_matrices(self, m: int):
        """Dense copies of mode_matrices (small sizes / tests)."""
        M, L, bc, af = self.mode_matrices(m)
        return M.toarray(), L.toarray(), bc, af

    # -- gather/scatter between fields and mode vectors ---------------------
    def gather(self, m: int, b, ux, uz, pr, tau) -> np.ndarray:
        taus = tau[:, m] if m == 0 else tau[1:, m]
        return np.concatenate([pr[:, m], b[:, m], ux[:, m], uz[:, m], taus])

    def scatter(self, m: int, x: np.ndarray, b, ux, uz, pr, tau) -> None:
        N = self.p.Nz
        pr[:, m] = x[0:N]
        b[:, m] = x[N : 2 * N]
        ux[:, m] = x[2 * N : 3 * N]
        uz[:, m] = x[3 * N : 4 * N]
        if m == 0:
            tau[:, m] = x[4 * N :]
        else:
            tau[0, m] = 0.0
            tau[1:, m] = x[4 * N :]

    def equation_F(self, m: int, Fb, Fux, Fuz) -> np.ndarray:
        """gather_eqn_F!: PDE rows get the F coefficients, algebraic rows stay zero
        (subproblem_rhs.jl:411-482)."""
        N = self.p.Nz
        n = self.n_unknowns(m)
        f = np.zeros(n, complex)
        f[N : 2 * N] = Fb[:, m]
        f[2 * N : 3 * N] = Fux[:, m]
        f[3 * N : 4 * N] = Fuz[:, m]
        return f

    def mass_solve(self, m: int, rhs: np.ndarray) -> np.ndarray:
        """Min-norm least squares of the 0/1 selection M_min (SPQR on CPU,
        step_subproblem_rk.jl:873-905): copy the b/u rows, zero p and taus."""
        N = self.p.Nz
        x = np.zeros_like(rhs)
        x[N : 4 * N] = rhs[N : 4 * N]
        return x

    def _lhs_lu(self, m: int, alpha: float, beta: float):
        """Sparse LU of alpha M + beta L, cached per (mode, alpha, beta).

        The reference factors the same matrix with UMFPACK (SparseLUSolver,
        src/tools/matsolvers.jl:65-147); SuperLU (splu) is the SciPy equivalent.
        """
        key = (m, alpha, beta)
        lu = self._lu.get(key)
        if lu is None:
            M, L, _, _ = self.mode_matrices(m)
            A = (alpha * M + beta * L).tocsc()
            try:
                lu = spsl.splu(A)
            except RuntimeError as e:
                raise np.linalg.LinAlgError(f"singular tau matrix at mode {m}: {e}")
            self._lu[key] = lu
        return lu

    # -- state helpers -------------------------------------------------------
    def set_b_grid(self, bg: np.ndarray) -> None:
        self.b = forward_2d(bg)

    def fields(self):
        return self.b, self.ux, self.uz, self.pr, self.tau

    def projected(self, c: np.ndarray) -> np.ndarray:
        """A c->g->c round trip through rfft/irfft drops Im of the DC and Nyquist
        x-modes (the re-gather hazard of step_subproblem_rk_batched.jl:33-37)."""
        out = np.array(c, copy=True)
        out[:, 0] = out[:, 0].real
        if self.p.Nx % 2 == 0:
            out[:, self.p.Nx // 2] = out[:, self.p.Nx // 2].real
        return out

    # -- RHS: lazy evaluator semantics (lazy_rhs.jl:712-1157) -----------------
    def rhs(self, b, ux, uz):
        """F = -(u.grad f) for f in (b, ux, uz); returns coefficient fields."""
        p = self.p
        Nx = p.Nx
        bg, uxg, uzg = (backward_2d(c, Nx) for c in (b, ux, uz))
        kmul = (1j * self.kx)[None, :]

        def dx(g):
            return backward_2d(kmul * forward_2d(g), Nx)

        def dz(g):
            return backward_2d(self.D @ forward_2d(g), Nx)

        out = []
        for fg in (bg, uxg, uzg):
            t1 = padded_multiply(uxg, dx(fg), p.dealias)
            t2 = padded_multiply(uzg, dz(fg), p.dealias)
            out.append(forward_2d(-(t1 + t2)))
        return out

    # -- IMEX Runge-Kutta (step_subproblem_rk.jl:393-739) ---------------------
    def step_rk(self, dt: float, ts: dict) -> None:
        Nk = self.Nk
        s = ts["AE"].shape[0]
        AE, AI, bE, bI = ts["AE"], ts["AI"], ts["bE"], ts["bI"]
        x0 = [self.gather(m, *self.fields()) for m in range(Nk)]
        MX0 = _pmap(lambda m: self.mode_matrices(m)[0] @ x0[m], range(Nk))
        F: List[List[np.ndarray]] = []
        LX: List[List[np.ndarray]] = []
        for i in range(s):
            a_ii = AI[i, i]

            def stage_solve(m):
                M, L, bc, algf = self.mode_matrices(m)
                rhs = MX0[m].copy()
                for j in range(i):
                    if abs(dt * AE[i, j]) > 1e-14:
                        rhs += dt * AE[i, j] * F[j][m]
                    if abs(dt * AI[i, j]) > 1e-14:
                        rhs -= dt * AI[i, j] * LX[j][m]
                if abs(a_ii) < 1e-14:
                    return self.mass_solve(m, rhs)
                algf = self._stage_algf(m, algf, self.sim_time + dt * ts["c"][i])
                rhs[bc] = dt * a_ii * algf[bc]
                return self._lhs_lu(m, 1.0, dt * a_ii).solve(rhs)

            xs = _pmap(stage_solve, range(Nk))
            for m in range(Nk):
                self.scatter(m, xs[m], *self.fields())
            Fb, Fux, Fuz = self.rhs(self.b, self.ux, self.uz)
            pb, pux, puz = (self.projected(c) for c in (self.b, self.ux, self.uz))
            F.append(_pmap(lambda m: self.equation_F(m, Fb, Fux, Fuz), range(Nk)))
            LX.append(_pmap(lambda m: self.mode_matrices(m)[1] @ self.gather(m, pb, pux, puz, self.pr, self.tau),
                            range(Nk)))

        def final(m):
            rhs = MX0[m].copy()
            for j in range(s):
                if abs(dt * bE[j]) > 1e-14:
                    rhs += dt * bE[j] * F[j][m]
                if abs(dt * bI[j]) > 1e-14:
                    rhs -= dt * bI[j] * LX[j][m]
            return self.mass_solve(m, rhs)

        xs = _pmap(final, range(Nk))
        for m in range(Nk):
            self.scatter(m, xs[m], *self.fields())
        self.sim_time += dt
        self.iteration += 1

    # -- SBDF1/SBDF2 (step_subproblem_multistep.jl:197-405) -------------------
    def step_sbdf(self, dt: float, order: int = 2) -> None:
        Nk = self.Nk
        use_order = 1 if (order == 1 or len(self._ms_hist) < 1) else 2
        a, bcoef, c = sbdf_coefs(use_order, dt, self._ms_dt_prev)
        Fb, Fux, Fuz = self.rhs(self.b, self.ux, self.uz)
        pb, pux, puz = (self.projected(cf) for cf in (self.b, self.ux, self.uz))
        MXc = _pmap(lambda m: self.mode_matrices(m)[0] @ self.gather(m, pb, pux, puz, self.pr, self.tau), range(Nk))
        Fc = _pmap(lambda m: self.equation_F(m, Fb, Fux, Fuz), range(Nk))
        hist = [(MXc, Fc)] + self._ms_hist

        def solve(m):
            M, L, bc, algf = self.mode_matrices(m)
            rhs = np.zeros(self.n_unknowns(m), complex)
            for k in range(1, len(c)):
                if abs(c[k]) >= 1e-14 and k - 1 < len(hist):
                    rhs += c[k] * hist[k - 1][1][m]
            for k in range(1, len(a)):
                if abs(a[k]) >= 1e-14 and k - 1 < len(hist):
                    rhs -= a[k] * hist[k - 1][0][m]
            algf = self._stage_algf(m, algf, self.sim_time + dt)
            rhs[bc] = bcoef[0] * algf[bc]
            return self._lhs_lu(m, a[0], bcoef[0]).solve(rhs)

        xs = _pmap(solve, range(Nk))
        for m in range(Nk):
            self.scatter(m, xs[m], *self.fields())
        self._ms_hist = hist[:1] if order == 1 else hist[:2]
        self._ms_dt_prev = dt
        self.sim_time += dt
        self.iteration += 1

    def step(self, dt: float, scheme: str) -> None:
        if scheme in TABLEAUS:
            self.step_rk(dt, TABLEAUS[scheme])
        elif scheme == "SBDF1":
            self.step_sbdf(dt, 1)
        elif scheme == "SBDF2":
            self.step_sbdf(dt, 2)
        else:
            raise ValueError(scheme)

    def state_dict(self) -> Dict[str, np.ndarray]:
        return dict(b=self.b.copy(), ux=self.ux.copy(), uz=self.uz.copy(), p=self.pr.copy(), tau=self.tau.copy())


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    """Relative L2 error ||a-b|| / ||b|| (0 when both vanish)."""
    nb = np.linalg.norm(b)
    na = np.linalg.norm(a - b)
    if nb == 0.0:
        return float(na)
    return float(na / nb)


def run_rbc(p: RBCParams, scheme: str, dt: float, nsteps: int, seed: int = 42) -> RBC2D:
    """Build the RBC problem with the seeded initial b and advance nsteps."""
    sim = RBC2D(p)
    sim.set_b_grid(rbc_initial_b(p, seed))
    for _ in range(nsteps):
        sim.step(dt, scheme)
    return sim


# ---------------------------------------------------------------------------
# 2D doubly periodic decaying turbulence (vorticity form), DiagonalIMEX_SBDF2
# (examples/2d_decaying_turbulence_gpu.jl).  Layout: a grid field of logical
# size (Nx, Ny) is an array of shape (Ny, Nx); coefficients (Nx/2+1, Ny) are
# shape (Ny, Nx/2+1): rfft along x, fft along y, unnormalised.
# ---------------------------------------------------------------------------
def turb_wavenumbers(Nx: int, Ny: int, Lx: float, Ly: float):
    """kx: rfft layout 0..Nx/2 (basis_wavenumbers.jl:68-79); ky: fft order with
    -Ny/2 at the Nyquist index (basis_wavenumbers.jl:95-108)."""
    kx = 2 * np.pi / Lx * np.arange(Nx // 2 + 1)
    ky = 2 * np.pi / Ly * np.concatenate([np.arange(Ny // 2), np.arange(-(Ny // 2), 0)])
    return kx[None, :], ky[:, None]


def turb_forward(g: np.ndarray) -> np.ndarray:
    """Grid (Ny, Nx) real -> coefficients: rfft along x then fft along y."""
    return _fx.fft(_fx.rfft(g, axis=1), axis=0)


def turb_backward(c: np.ndarray, Nx: int) -> np.ndarray:
    """Coefficients -> grid: ifft along y, irfft along x (Im of DC and Nyquist dropped)."""
    return _fx.irfft(_fx.ifft(c, axis=0), n=Nx, axis=1)


def _pad_full(A: np.ndarray, M: Tuple[int, int]) -> np.ndarray:
    """Zero-pad a full complex spectrum with the even-N Nyquist split X/2 at
    +-N/2, axis x first then y (nonlinear_padding.jl:164-262)."""
    Ny, Nx = A.shape
    My, Mx = M
    P = np.zeros((My, Mx), dtype=complex)

    def ranges(N, Mn):
        h = N // 2
        pos = (slice(0, h + 1), slice(0, h + 1))
        nneg = N - h - 1
        neg = (slice(N - nneg, N), slice(Mn - nneg, Mn)) if nneg > 0 else None
        return pos, neg

    (py, pyp), ny_ = ranges(Ny, My)
    (px, pxp), nx_ = ranges(Nx, Mx)
    P[pyp, pxp] = A[py, px]
    if ny_:
        P[ny_[1], pxp] = A[ny_[0], px]
    if nx_:
        P[pyp, nx_[1]] = A[py, nx_[0]]
    if ny_ and nx_:
        P[ny_[1], nx_[1]] = A[ny_[0], nx_[0]]
    for axis, N, Mn in ((1, Nx, Mx), (0, Ny, My)):
        if N % 2 == 0 and Mn > N:
            nyq, mir = N // 2, Mn - N // 2
            if axis == 1:
                P[:, nyq] *= 0.5
                P[:, mir] = P[:, nyq]
            else:
                P[nyq, :] *= 0.5
                P[mir, :] = P[nyq, :]
    return P


def _truncate_full(P: np.ndarray, N: Tuple[int, int]) -> np.ndarray:
    """Fold the -N/2 images into +N/2 (x then y) and truncate
    (nonlinear_padding.jl:208-346)."""
    P = P.copy()
    My, Mx = P.shape
    Ny, Nx = N
    for axis, n, Mn in ((1, Nx, Mx), (0, Ny, My)):
        if n % 2 == 0 and Mn > n:
            nyq, mir = n // 2, Mn - n // 2
            if axis == 1:
                P[:, nyq] += P[:, mir]
            else:
                P[nyq, :] += P[mir, :]
    out = np.zeros((Ny, Nx), dtype=complex)
    hy, hx = Ny // 2, Nx // 2
    ny_, nx_ = Ny - hy - 1, Nx - hx - 1
    out[: hy + 1, : hx + 1] = P[: hy + 1, : hx + 1]
    if ny_:
        out[Ny - ny_:, : hx + 1] = P[My - ny_:, : hx + 1]
    if nx_:
        out[: hy + 1, Nx - nx_:] = P[: hy + 1, Mx - nx_:]
    if ny_ and nx_:
        out[Ny - ny_:, Nx - nx_:] = P[My - ny_:, Mx - nx_:]
    return out


def padded_multiply_2d(a: np.ndarray, b: np.ndarray, factor: float = 1.5) -> np.ndarray:
    """evaluate_padded_multiply for two real grid fields on a doubly periodic
    grid (nonlinear_padding.jl:359-443): fftn, pad with Nyquist split, ifftn
    (1/M), product, fftn, fold + truncate, ifftn (1/N), real part, times M/N
    per axis."""
    Ny, Nx = a.shape
    My, Mx = padded_length(Ny, factor), padded_length(Nx, factor)
    Pa = _fx.ifftn(_pad_full(_fx.fftn(a), (My, Mx)))
    Pb = _fx.ifftn(_pad_full(_fx.fftn(b), (My, Mx)))
    R = _truncate_full(_fx.fftn(Pa * Pb), (Ny, Nx))
    return np.real(_fx.ifftn(R)) * (Mx / Nx) * (My / Ny)


def turb_rhs(q: np.ndarray, Nx: int, Lx: float, Ly: float) -> np.ndarray:
    """F = -u.grad(q) in coefficients: psi = -q/k^2 (k=0 gauge 0,
    state_utils.jl:1059-1075), u = (-d_y psi, d_x psi) (:1077-1104), derivative
    multipliers i k (lazy_rhs.jl:1190-1238), dealiased products."""
    Ny = q.shape[0]
    kx, ky = turb_wavenumbers(Nx, Ny, Lx, Ly)
    k2 = kx ** 2 + ky ** 2
    psi = np.where(k2 > 1e-12, -q / np.where(k2 > 1e-12, k2, 1.0), 0.0)
    u = turb_backward(-1j * ky * psi, Nx)
    v = turb_backward(1j * kx * psi, Nx)
    qx = turb_backward(1j * kx * q, Nx)
    qy = turb_backward(1j * ky * q, Nx)
    F = -(padded_multiply_2d(u, qx) + padded_multiply_2d(v, qy))
    return turb_forward(F)


def run_turb(q0: np.ndarray, Nx: int, Lx: float, Ly: float, nu: float, dt: float, nsteps: int) -> np.ndarray:
    """DiagonalIMEX_SBDF2 with constant dt (step_diagonal_imex.jl:329-388,
    674-689), L^ = nu k^2: SBDF1 startup, then
    q_{n+1} = (2 q_n - q_{n-1}/2 + dt (2 F_n - F_{n-1})) / (3/2 + dt L^)."""
    Ny = q0.shape[0]
    kx, ky = turb_wavenumbers(Nx, Ny, Lx, Ly)
    L = nu * (kx ** 2 + ky ** 2)
    q, qm, Fm = q0.copy(), None, None
    for n in range(nsteps):
        Fn = turb_rhs(q, Nx, Lx, Ly)
        if n == 0:
            qn = (q + dt * Fn) / (1.0 + dt * L)
        else:
            qn = (2.0 * q - 0.5 * qm + dt * (2.0 * Fn - Fm)) / (1.5 + dt * L)
        qm, q, Fm = q, qn, Fn
    return q


def turb_step_rk(q: np.ndarray, Nx: int, Lx: float, Ly: float, nu: float, dt: float, ts: dict) -> np.ndarray:
    """One DiagonalIMEX_RK222 / RK443 step (_step_diagonal_imex_rk_impl!,
    step_diagonal_imex.jl:183-296; tableaus types.jl:511-620, the same numbers
    as the subproblem RK222 / RK443) with L^ = nu k^2:
      Y_s = q_n + dt sum_{j<s} (AE_sj F_j - AI_sj L^ Y_j),  Y_s /= 1 + dt AI_ss L^
      F_s = RHS(Y_s)
      q_{n+1} = q_n + dt sum_s (bE_s F_s - bI_s L^ Y_s).
    Stage states stay in coefficients (no grid round trip between stages); the
    RHS does its own, as in the reference's evaluate_rhs."""
    Ny = q.shape[0]
    kx, ky = turb_wavenumbers(Nx, Ny, Lx, Ly)
    L = nu * (kx ** 2 + ky ** 2)
    AE, AI, bE, bI = ts["AE"], ts["AI"], ts["bE"], ts["bI"]
    s = AE.shape[0]
    Y: List[np.ndarray] = []
    F: List[Optional[np.ndarray]] = []
    for i in range(s):
        y = q.copy()
        for j in range(i):
            if abs(AE[i, j]) > 1e-14:
                y += dt * AE[i, j] * F[j]
            if abs(AI[i, j]) > 1e-14:
                y -= dt * AI[i, j] * L * Y[j]
        if abs(AI[i, i]) > 1e-14:
            y = y / (1.0 + dt * AI[i, i] * L)
        Y.append(y)
        # F_s enters a later stage or the update only where its weight is
        # nonzero (the first stage's never is in these tableaus)
        used = abs(bE[i]) > 1e-14 or any(abs(AE[k, i]) > 1e-14 for k in range(i + 1, s))
        F.append(turb_rhs(y, Nx, Lx, Ly) if used else None)
    out = q.copy()
    for i in range(s):
        if abs(bE[i]) > 1e-14:
            out += dt * bE[i] * F[i]
        if abs(bI[i]) > 1e-14:
            out -= dt * bI[i] * L * Y[i]
    return out


def run_turb_rk(q0: np.ndarray, Nx: int, Lx: float, Ly: float, nu: float, dt: float, nsteps: int,
                scheme: str = "RK222") -> np.ndarray:
    """nsteps DiagonalIMEX_RK222 / RK443 steps of constant dt."""
    q = q0.copy()
    for _ in range(nsteps):
        q = turb_step_rk(q, Nx, Lx, Ly, nu, dt, TABLEAUS[scheme])
    return q


def turb_initial_spec(Nx: int, Ny: int, seed: int, kmin: float = 1.0, kmax: Optional[float] = None,
                      amp: float = 10.0) -> np.ndarray:
    """Seeded initial vorticity with a k^-3 energy spectrum (|q^| ~ 1/k per mode
    for kmin <= |k| <= kmax, random phases), scaled to max |q| = amp on the grid."""
    kmax = kmax if kmax is not None else min(Nx, Ny) / 3.0
    rng = np.random.default_rng(seed)
    kx, ky = turb_wavenumbers(Nx, Ny, 2 * np.pi, 2 * np.pi)
    k = np.sqrt(kx ** 2 + ky ** 2)
    mag = np.where((k >= kmin) & (k <= kmax), 1.0 / np.maximum(k, 1e-30), 0.0)
    phase = rng.uniform(0.0, 2 * np.pi, size=mag.shape)
    g = turb_backward(mag * np.exp(1j * phase), Nx)
    g *= amp / np.abs(g).max()
    return turb_forward(g)


# ---------------------------------------------------------------------------
# 3D Rayleigh-Benard: RealFourier x, RealFourier y, ChebyshevT z
# (ChannelDomain3D, src/extras/quick_domains.jl:124-143; equations of
# examples/ivp/rotating_rayleigh_benard_3d.jl:80-104 without rotation, in the
# free-fall scaling of test/test_subproblem_rk.jl:23-24).
#
# Layout: a grid field of logical size (Nx, Ny, Nz) is an array of shape
# (Nz, Ny, Nx); coefficients (Nx/2+1, Ny, Nz) are shape (Nz, Ny, Nx/2+1): rfft
# along x, fft along y (ky in FFT order, -Ny/2 at the Nyquist index), then the
# ChebyshevT transform along z, all unnormalised in x and y like the 2D case.
# ---------------------------------------------------------------------------


def forward_3d(g: np.ndarray) -> np.ndarray:
    """Grid (Nz, Ny, Nx) -> coefficients (Nz, Ny, Nx/2+1)."""
    return cheb_forward(_fx.fft(_fx.rfft(g, axis=2), axis=1), axis=0)


def backward_3d(c: np.ndarray, Nx: int) -> np.ndarray:
    """Coefficients -> grid: ChebyshevT backward, ifft along y, irfft along x
    (Im of the kx = 0 and Nyquist bins dropped at every y, as FFTW's c2r)."""
    return _fx.irfft(_fx.ifft(cheb_backward(c, axis=0), axis=1), n=Nx, axis=2)


def _pad_xy(A: np.ndarray, My: int, Mx: int) -> np.ndarray:
    """_pad_full over the last two axes (y, x) of a stack of full spectra."""
    Ny, Nx = A.shape[-2:]
    P = np.zeros(A.shape[:-2] + (My, Mx), dtype=complex)
    hy, hx = Ny // 2, Nx // 2
    ny_, nx_ = Ny - hy - 1, Nx - hx - 1
    P[..., : hy + 1, : hx + 1] = A[..., : hy + 1, : hx + 1]
    if ny_:
        P[..., My - ny_:, : hx + 1] = A[..., Ny - ny_:, : hx + 1]
    if nx_:
        P[..., : hy + 1, Mx - nx_:] = A[..., : hy + 1, Nx - nx_:]
    if ny_ and nx_:
        P[..., My - ny_:, Mx - nx_:] = A[..., Ny - ny_:, Nx - nx_:]
    if Nx % 2 == 0 and Mx > Nx:
        P[..., :, hx] *= 0.5
        P[..., :, Mx - hx] = P[..., :, hx]
    if Ny % 2 == 0 and My > Ny:
        P[..., hy, :] *= 0.5
        P[..., My - hy, :] = P[..., hy, :]
    return P


def _truncate_xy(P: np.ndarray, Ny: int, Nx: int) -> np.ndarray:
    """_truncate_full over the last two axes: fold the -N/2 images, truncate."""
    P = P.copy()
    My, Mx = P.shape[-2:]
    hy, hx = Ny // 2, Nx // 2
    if Nx % 2 == 0 and Mx > Nx:
        P[..., :, hx] += P[..., :, Mx - hx]
    if Ny % 2 == 0 and My > Ny:
        P[..., hy, :] += P[..., My - hy, :]
    out = np.zeros(P.shape[:-2] + (Ny, Nx), dtype=complex)
    ny_, nx_ = Ny - hy - 1, Nx - hx - 1
    out[..., : hy + 1, : hx + 1] = P[..., : hy + 1, : hx + 1]
    if ny_:
        out[..., Ny - ny_:, : hx + 1] = P[..., My - ny_:, : hx + 1]
    if nx_:
        out[..., : hy + 1, Nx - nx_:] = P[..., : hy + 1, Mx - nx_:]
    if ny_ and nx_:
        out[..., Ny - ny_:, Nx - nx_:] = P[..., My - ny_:, Mx - nx_:]
    return out


def padded_multiply_3d(a: np.ndarray, b: np.ndarray, factor: float = 1.5) -> np.ndarray:
    """evaluate_padded_multiply for two real grid fields (Nz, Ny, Nx): 3/2
    padding along both Fourier axes only (nonlinear_padding.jl:86-103,
    359-443), per z level exactly padded_multiply_2d."""
    Ny, Nx = a.shape[-2:]
    My, Mx = padded_length(Ny, factor), padded_length(Nx, factor)
    ax = (-2, -1)
    Pa = _fx.ifftn(_pad_xy(_fx.fftn(a, axes=ax), My, Mx), axes=ax)
    Pb = _fx.ifftn(_pad_xy(_fx.fftn(b, axes=ax), My, Mx), axes=ax)
    R = _truncate_xy(_fx.fftn(Pa * Pb, axes=ax), Ny, Nx)
    return np.real(_fx.ifftn(R, axes=ax)) * (Mx / Nx) * (My / Ny)


@dataclass
class RBC3Params:
    Nx: int
    Ny: int
    Nz: int
    Lx: float = 4.0
    Ly: float = 4.0
    Lz: float = 1.0
    Ra: float = 1e7
    Pr: float = 1.0
    dealias: float = 1.5
    b_bottom: float = None
    b_top: float = 0.0

    @property
    def kappa(self) -> float:
        return (self.Ra * self.Pr) ** -0.5

    @property
    def nu(self) -> float:
        return (self.Ra / self.Pr) ** -0.5

    def bottom(self) -> float:
        return self.Lz if self.b_bottom is None else self.b_bottom


def rbc3_initial_b(p: RBC3Params, seed: int = 42, amp: float = 1e-3) -> np.ndarray:
    """b0 = Lz - z + amp z (Lz - z) xi on the (x, y, z) grid, xi ~ N(0,1) from
    PCG64(seed) drawn in Julia (x, y, z) order; returned as (Nz, Ny, Nx)."""
    rng = np.random.default_rng(seed)
    xi = rng.standard_normal((p.Nx, p.Ny, p.Nz)).transpose(2, 1, 0)
    z = cheb_grid(p.Nz, 0.0, p.Lz)[:, None, None]
    return (p.Lz - z) + amp * z * (p.Lz - z) * xi


class RBC3D:
    """Per-(kx, ky) tau system of 3D Boussinesq RBC in the reference's own
    Cartesian form (one complex system per Fourier mode pair, as
    build_matrices! assembles it, subproblem_matrix_build.jl:11-309) and the
    IMEX Runge-Kutta stepper of step_subproblem_rk.jl:393-739.

    Unknowns per mode: [p, b, ux, uy, uz](Nz each), then tau_p (only at
    kx = ky = 0), tau_b1, tau_b2, tau_u1 (x, y, z), tau_u2 (x, y, z).
    Equations: continuity, b, u_x, u_y, u_z (Nz rows each), then the wall rows
    b, ux, uy, uz at z = 0 and at z = Lz, and integ(p) at kx = ky = 0.
    """

    TAU_NAMES = ("tau_p", "tau_b1", "tau_b2", "tau_u1x", "tau_u1y", "tau_u1z", "tau_u2x", "tau_u2y", "tau_u2z")

    def __init__(self, p: RBC3Params):
        self.p = p
        Nx, Ny, Nz = p.Nx, p.Ny, p.Nz
        self.Kx = Nx // 2 + 1
        self.kx = 2 * np.pi / p.Lx * np.arange(self.Kx)
        self.ky = 2 * np.pi / p.Ly * np.concatenate([np.arange(Ny // 2), np.arange(-(Ny // 2), 0)])
        self.D = cheb_diff_matrix(Nz, p.Lz)
        self.D2 = self.D @ self.D
        self._mats: Dict[Tuple[int, int], tuple] = {}
        self._lu: Dict[Tuple[int, int, float, float], object] = {}
        shape = (Nz, Ny, self.Kx)
        self.b = np.zeros(shape, complex)
        self.ux = np.zeros(shape, complex)
        self.uy = np.zeros(shape, complex)
        self.uz = np.zeros(shape, complex)
        self.pr = np.zeros(shape, complex)
        self.tau = np.zeros((9, Ny, self.Kx), complex)
        self.sim_time = 0.0
        self.iteration = 0
        # dynamic wall values of b: t -> (bottom, top) coefficient arrays (Ny, Kx)
        self.wall_b = None

    def modes(self):
        return [(iy, ix) for iy in range(self.p.Ny) for ix in range(self.Kx)]

    def mode_matrices(self, iy: int, ix: int):
        """Sparse M, L, BC-row list and ALG_F of Fourier mode (kx[ix], ky[iy])."""
        key = (iy, ix)
        if key in self._mats:
            return self._mats[key]
        p = self.p
        N = p.Nz
        kx, ky = self.kx[ix], self.ky[iy]
        k2 = kx * kx + ky * ky
        dc = ix == 0 and iy == 0
        names = self.TAU_NAMES if dc else self.TAU_NAMES[1:]
        n = 5 * N + len(names)
        cp, cb, cux, cuy, cuz = 0, N, 2 * N, 3 * N, 4 * N
        tcol = {nm: 5 * N + i for i, nm in enumerate(names)}
        rc, rb, rx, ry, rz, r_bc = 0, N, 2 * N, 3 * N, 4 * N, 5 * N
        kap, nu = p.kappa, p.nu
        Lr, Lc, Lv = [], [], []
        idx = np.arange(N)
        dr, dcol = np.nonzero(self.D)
        d2r, d2c = np.nonzero(self.D2)
        De = self.D[:, N - 1]
        der = np.nonzero(De)[0]

        def add(r0, c0, rr, cc, vv):
            vv = np.broadcast_to(np.asarray(vv, dtype=complex), np.shape(rr))
            keep = np.abs(vv) >= 1e-12  # entry cutoff (subproblem_matrix_build.jl:88-100)
            Lr.append(r0 + np.asarray(rr)[keep])
            Lc.append(c0 + np.asarray(cc)[keep])
            Lv.append(vv[keep])

        def lap_block(r0, c0, coef):
            add(r0, c0, idx, idx, -coef * k2 * np.ones(N))
            add(r0, c0, d2r, d2c, coef * self.D2[d2r, d2c])

        # trace(grad_u) + tau_p = 0
        add(rc, cux, idx, idx, 1j * kx * np.ones(N))
        add(rc, cuy, idx, idx, 1j * ky * np.ones(N))
        add(rc, cuz, dr, dcol, self.D[dr, dcol])
        add(rc, tcol["tau_u1z"], [N - 1], [0], [1.0])
        if dc:
            add(rc, tcol["tau_p"], [0], [0], [1.0])
        # dt(b) - kappa div(grad_b) + lift(tau_b2) = -u.grad(b)
        lap_block(rb, cb, -kap)
        add(rb, tcol["tau_b1"], der, np.zeros_like(der), -kap * De[der])
        add(rb, tcol["tau_b2"], [N - 1], [0], [1.0])
        # dt(u) - nu div(grad_u) + grad(p) - b ez + lift(tau_u2) = -u.grad(u)
        for r0, c0, t1, t2, grad in ((rx, cux, "tau_u1x", "tau_u2x", 1j * kx), (ry, cuy, "tau_u1y", "tau_u2y", 1j * ky)):
            lap_block(r0, c0, -nu)
            add(r0, tcol[t1], der, np.zeros_like(der), -nu * De[der])
            add(r0, cp, idx, idx, grad * np.ones(N))
            add(r0, tcol[t2], [N - 1], [0], [1.0])
        lap_block(rz, cuz, -nu)
        add(rz, tcol["tau_u1z"], der, np.zeros_like(der), -nu * De[der])
        add(rz, cp, dr, dcol, self.D[dr, dcol])
        add(rz, cb, idx, idx, -np.ones(N))
        add(rz, tcol["tau_u2z"], [N - 1], [0], [1.0])
        bot = cheb_eval_row(N, -1.0)
        top = cheb_eval_row(N, 1.0)
        zero = np.zeros(N, int)
        walls = ((cb, bot), (cux, bot), (cuy, bot), (cuz, bot), (cb, top), (cux, top), (cuy, top), (cuz, top))
        for i, (col, row) in enumerate(walls):
            add(r_bc + i, col, zero, idx, row)
        bc_rows = list(range(r_bc, r_bc + 8))
        alg_f = np.zeros(n, complex)
        if dc:
            # a constant BC value v projects to v Nx Ny at kx = ky = 0 (subproblem_rhs.jl:99-115)
            alg_f[r_bc + 0] = p.bottom() * p.Nx * p.Ny
            alg_f[r_bc + 4] = p.b_top * p.Nx * p.Ny
            add(r_bc + 8, cp, zero, idx, p.Lx * p.Ly * cheb_integ_row(N, p.Lz))
            bc_rows.append(r_bc + 8)
        L = sps.coo_matrix((np.concatenate(Lv), (np.concatenate(Lr), np.concatenate(Lc))), shape=(n, n)).tocsr()
        L.sum_duplicates()
        Mi = np.concatenate([cb + idx, cux + idx, cuy + idx, cuz + idx])
        Mr = np.concatenate([rb + idx, rx + idx, ry + idx, rz + idx])
        M = sps.coo_matrix((np.ones(4 * N, complex), (Mr, Mi)), shape=(n, n)).tocsr()
        out = (M, L, np.array(bc_rows), alg_f)
        self._mats[key] = out
        return out

    def _fields(self):
        return (self.pr, self.b, self.ux, self.uy, self.uz)

    def gather(self, iy, ix, fields, tau) -> np.ndarray:
        taus = tau[:, iy, ix] if (ix == 0 and iy == 0) else tau[1:, iy, ix]
        return np.concatenate([f[:, iy, ix] for f in fields] + [taus])

    def scatter(self, iy, ix, x) -> None:
        N = self.p.Nz
        for i, f in enumerate(self._fields()):
            f[:, iy, ix] = x[i * N : (i + 1) * N]
        if ix == 0 and iy == 0:
            self.tau[:, iy, ix] = x[5 * N :]
        else:
            self.tau[0, iy, ix] = 0.0
            self.tau[1:, iy, ix] = x[5 * N :]

    def equation_F(self, iy, ix, F) -> np.ndarray:
        N = self.p.Nz
        n = 5 * N + (9 if (ix == 0 and iy == 0) else 8)
        f = np.zeros(n, complex)
        for i, Ff in enumerate(F):
            f[(i + 1) * N : (i + 2) * N] = Ff[:, iy, ix]
        return f

    def mass_solve(self, rhs: np.ndarray) -> np.ndarray:
        """Min-norm solve of the 0/1 selection M: copy the b/u rows, zero p and taus."""
        N = self.p.Nz
        x = np.zeros_like(rhs)
        x[N : 5 * N] = rhs[N : 5 * N]
        return x

    def _lhs_lu(self, iy, ix, alpha, beta):
        key = (iy, ix, alpha, beta)
        lu = self._lu.get(key)
        if lu is None:
            M, L, _, _ = self.mode_matrices(iy, ix)
            try:
                lu = spsl.splu((alpha * M + beta * L).tocsc())
            except RuntimeError as e:
                raise np.linalg.LinAlgError(f"singular tau matrix at mode ({ix}, {iy}): {e}")
            self._lu[key] = lu
        return lu

    def set_b_grid(self, bg: np.ndarray) -> None:
        self.b = forward_3d(bg)

    def projected(self, c: np.ndarray) -> np.ndarray:
        """The grid round trip of a coefficient field (Hermitian projection of
        the kx = 0 and kx = Nx/2 planes in ky)."""
        return forward_3d(backward_3d(c, self.p.Nx))

    def rhs(self, b, ux, uy, uz):
        """F = -(u.grad f) for f in (b, ux, uy, uz) with lazy-evaluator semantics:
        every factor is a grid field from a coefficient round trip, each product
        3/2-dealiased (lazy_rhs.jl:712-1336)."""
        p = self.p
        Nx = p.Nx
        g = [backward_3d(c, Nx) for c in (b, ux, uy, uz)]
        KX = (1j * self.kx)[None, None, :]
        KY = (1j * self.ky)[None, :, None]

        def dx(f):
            return backward_3d(KX * forward_3d(f), Nx)

        def dy(f):
            return backward_3d(KY * forward_3d(f), Nx)

        def dz(f):
            return backward_3d(np.tensordot(self.D, forward_3d(f), axes=(1, 0)), Nx)

        out = []
        for fg in g:
            t = padded_multiply_3d(g[1], dx(fg), p.dealias)
            t = t + padded_multiply_3d(g[2], dy(fg), p.dealias)
            t = t + padded_multiply_3d(g[3], dz(fg), p.dealias)
            out.append(forward_3d(-t))
        return out

    def step_rk(self, dt: float, ts: dict, modes=None, rhs_fn=None, proj_fn=None) -> None:
        """One IMEX RK step.  `modes` restricts the per-mode work to a subset
        (a rank of a mode-sharded step), `rhs_fn()` then supplies F for those
        modes and `proj_fn(c)` the grid round trip of a field on them; by
        default every mode, RBC3D.rhs and RBC3D.projected."""
        AE, AI, bE, bI = ts["AE"], ts["AI"], ts["bE"], ts["bI"]
        s = AE.shape[0]
        modes = self.modes() if modes is None else modes
        rhs_fn = rhs_fn or (lambda: self.rhs(self.b, self.ux, self.uy, self.uz))
        proj_fn = proj_fn or self.projected

        def mapped(fn):
            return dict(zip(modes, _pmap(fn, modes)))

        x0 = {m: self.gather(*m, self._fields(), self.tau) for m in modes}
        MX0 = mapped(lambda m: self.mode_matrices(*m)[0] @ x0[m])
        F, LX = [], []
        for i in range(s):
            a_ii = AI[i, i]
            walls = None
            if abs(a_ii) >= 1e-14 and self.wall_b is not None:
                walls = self.wall_b(self.sim_time + dt * ts["c"][i])

            def stage_solve(m):
                M, L, bc, algf = self.mode_matrices(*m)
                rhs = MX0[m].copy()
                for j in range(i):
                    if abs(dt * AE[i, j]) > 1e-14:
                        rhs += dt * AE[i, j] * F[j][m]
                    if abs(dt * AI[i, j]) > 1e-14:
                        rhs -= dt * AI[i, j] * LX[j][m]
                if abs(a_ii) < 1e-14:
                    return self.mass_solve(rhs)
                if walls is not None:
                    bot, top = walls
                    algf = algf.copy()
                    algf[5 * self.p.Nz + 0] = bot[m]
                    algf[5 * self.p.Nz + 4] = top[m]
                rhs[bc] = dt * a_ii * algf[bc]
                return self._lhs_lu(*m, 1.0, dt * a_ii).solve(rhs)

            xs = mapped(stage_solve)
            for m in modes:
                self.scatter(*m, xs[m])
            Fc = rhs_fn()
            proj = [self.pr] + [proj_fn(c) for c in (self.b, self.ux, self.uy, self.uz)]
            F.append(mapped(lambda m: self.equation_F(*m, Fc)))
            LX.append(mapped(lambda m: self.mode_matrices(*m)[1] @ self.gather(*m, proj, self.tau)))

        def final(m):
            rhs = MX0[m].copy()
            for j in range(s):
                if abs(dt * bE[j]) > 1e-14:
                    rhs += dt * bE[j] * F[j][m]
                if abs(dt * bI[j]) > 1e-14:
                    rhs -= dt * bI[j] * LX[j][m]
            return self.mass_solve(rhs)

        xs = mapped(final)
        for m in modes:
            self.scatter(*m, xs[m])
        self.sim_time += dt
        self.iteration += 1

    def step_sbdf(self, dt: float, order: int = 2) -> None:
        """SBDF1/SBDF2 (step_subproblem_multistep.jl:197-405; SBDF1 start,
        step_multistep.jl:341-356) on the 3D system; M X from the projected
        fields as the 2D restatement."""
        hist_prev = getattr(self, "_ms_hist", [])
        use_order = 1 if (order == 1 or len(hist_prev) < 1) else 2
        a, bcoef, c = sbdf_coefs(use_order, dt, getattr(self, "_ms_dt_prev", None))
        Fc3 = self.rhs(self.b, self.ux, self.uy, self.uz)
        proj = [self.pr] + [self.projected(cf) for cf in (self.b, self.ux, self.uy, self.uz)]
        modes = self.modes()
        def mapped(fn):
            return dict(zip(modes, _pmap(fn, modes)))

        MXc = mapped(lambda m: self.mode_matrices(*m)[0] @ self.gather(*m, proj, self.tau))
        Fc = mapped(lambda m: self.equation_F(*m, Fc3))
        hist = [(MXc, Fc)] + hist_prev
        walls = self.wall_b(self.sim_time + dt) if self.wall_b is not None else None

        def solve(m):
            M, L, bc, algf = self.mode_matrices(*m)
            rhs = np.zeros(M.shape[0], complex)
            for k in range(1, len(c)):
                if abs(c[k]) >= 1e-14 and k - 1 < len(hist):
                    rhs += c[k] * hist[k - 1][1][m]
            for k in range(1, len(a)):
                if abs(a[k]) >= 1e-14 and k - 1 < len(hist):
                    rhs -= a[k] * hist[k - 1][0][m]
            if walls is not None:
                bot, top = walls
                algf = algf.copy()
                algf[5 * self.p.Nz + 0] = bot[m]
                algf[5 * self.p.Nz + 4] = top[m]
            rhs[bc] = bcoef[0] * algf[bc]
            return self._lhs_lu(*m, a[0], bcoef[0]).solve(rhs)

        xs = mapped(solve)
        for m in modes:
            self.scatter(*m, xs[m])
        self._ms_hist = hist[:1] if order == 1 else hist[:2]
        self._ms_dt_prev = dt
        self.sim_time += dt
        self.iteration += 1

    def step(self, dt: float, scheme: str) -> None:
        if scheme in TABLEAUS:
            self.step_rk(dt, TABLEAUS[scheme])
        elif scheme == "SBDF1":
            self.step_sbdf(dt, 1)
        elif scheme == "SBDF2":
            self.step_sbdf(dt, 2)
        else:
            raise ValueError(scheme)

    def state_dict(self) -> Dict[str, np.ndarray]:
        return dict(b=self.b.copy(), ux=self.ux.copy(), uy=self.uy.copy(), uz=self.uz.copy(), p=self.pr.copy(),
                    tau=self.tau.copy())


# ---------------------------------------------------------------------------
# The 3D RHS in pencil form: the CPU stand-in for the per-rank kernels of a
# mode-sharded step (a rank owns a kx range, all ky and z).  The same
# arithmetic as RBC3D.rhs (lazy_rhs.jl:712-1336 with padded_multiply_3d,
# nonlinear_padding.jl:86-103, 182-443) reordered by axis, as the reference's
# pencil transposes reorder it (subproblem_io.jl:100-330): the z and y work
# per kx column, the x work per padded y row.
# ---------------------------------------------------------------------------
def _y_pad(S: np.ndarray, My: int) -> np.ndarray:
    """Zero-pad a full y spectrum (axis -2, FFT order) to My rows with the
    even-Ny Nyquist split X/2 at +-Ny/2 (_pad_full's y part)."""
    Ny = S.shape[-2]
    hy, nneg = Ny // 2, Ny - Ny // 2 - 1
    P = np.zeros(S.shape[:-2] + (My, S.shape[-1]), dtype=complex)
    P[..., : hy + 1, :] = S[..., : hy + 1, :]
    if nneg:
        P[..., My - nneg:, :] = S[..., Ny - nneg:, :]
    if Ny % 2 == 0 and My > Ny:
        P[..., hy, :] *= 0.5
        P[..., My - hy, :] = P[..., hy, :]
    return P


def _y_truncate(P: np.ndarray, Ny: int) -> np.ndarray:
    """Fold the -Ny/2 image into +Ny/2 and truncate (_truncate_full's y part)."""
    My = P.shape[-2]
    P = P.copy()
    hy, nneg = Ny // 2, Ny - Ny // 2 - 1
    if Ny % 2 == 0 and My > Ny:
        P[..., hy, :] += P[..., My - hy, :]
    out = np.zeros(P.shape[:-2] + (Ny, P.shape[-1]), dtype=complex)
    out[..., : hy + 1, :] = P[..., : hy + 1, :]
    if nneg:
        out[..., Ny - nneg:, :] = P[..., My - nneg:, :]
    return out


def rhs3_stage_modes(sim: "RBC3D", coeffs: Sequence[np.ndarray], kx_lo: int) -> np.ndarray:
    """Coefficients (b, ux, uy, uz), each (Nz, Ny, Kx_r) for kx indices kx_lo..,
    -> 12 arrays [field][value, d/dy, d/dz] on (z grid, padded y grid, kx):
    the grid round trip's projection of the kx = 0 and kx = Nx/2 planes (Im
    dropped after the inverse y transform, as FFTW's c2r drops it), z
    derivative in coefficient space, Chebyshev backward, y padding, inverse y
    transform (1/My)."""
    p = sim.p
    Ny = p.Ny
    My = padded_length(Ny, p.dealias)
    Kr = coeffs[0].shape[-1]
    ix = kx_lo + np.arange(Kr)
    edge = (ix == 0) | (ix == p.Nx // 2)
    KY = (1j * sim.ky)[None, :, None]
    out = []
    for c in coeffs:
        # projection: the kx = 0 / Nyquist planes of c through the y round trip with Im dropped
        t = _fx.ifft(cheb_backward(c, axis=0), axis=1)
        t[..., edge] = np.real(t[..., edge])
        pc = cheb_forward(_fx.fft(t, axis=1), axis=0)
        for S in (pc, KY * pc, np.tensordot(sim.D, pc, axes=(1, 0))):
            g = _fx.ifft(cheb_backward(S, axis=0), axis=1)  # (z, y, kx): Ny-point inverse (1/Ny)
            g[..., edge] = np.real(g[..., edge])
            out.append(_fx.ifft(_y_pad(_fx.fft(g, axis=1), My), axis=1))  # My-point inverse (1/My)
    return np.stack(out)


def rhs3_stage_rows(sim: "RBC3D", rows: np.ndarray) -> np.ndarray:
    """12 arrays (z, y rows, Kx) -> the 4 products -(u.grad f) for f = b, ux,
    uy, uz on these rows, forward x transform, x Nyquist fold and truncation:
    (4, z, y rows, Kx).  d/dx from the kx bins (Im dropped at kx = 0 and Nx/2,
    as the grid round trip does), x padding with the Nyquist split, inverse
    real x transform on Mx points (1/Mx)."""
    p = sim.p
    Nx = p.Nx
    Mx = padded_length(Nx, p.dealias)
    hx = Nx // 2
    KX = 1j * sim.kx

    def x_grid(X):
        H = np.zeros(X.shape[:-1] + (Mx // 2 + 1,), dtype=complex)
        H[..., :hx] = X[..., :hx]
        if Nx % 2 == 0 and Mx > Nx:
            H[..., hx] = 0.5 * X[..., hx]
        else:
            H[..., hx] = X[..., hx]
        return _fx.irfft(H, n=Mx, axis=-1)

    f = rows.reshape((4, 3) + rows.shape[1:])
    grids = {}
    for i in range(4):
        val, dy, dz = f[i]
        dxs = KX * val
        dxs[..., 0] = np.real(dxs[..., 0])
        dxs[..., hx] = np.real(dxs[..., hx])
        grids[i] = (x_grid(val), x_grid(dxs), x_grid(dy), x_grid(dz))
    u, v, w = grids[1][0], grids[2][0], grids[3][0]
    out = []
    for i in range(4):
        _, gx, gy, gz = grids[i]
        X = _fx.rfft(-(u * gx + v * gy + w * gz), axis=-1)[..., : hx + 1]
        if Nx % 2 == 0 and Mx > Nx:
            X[..., hx] = 2.0 * np.real(X[..., hx])
        out.append(X)
    return np.stack(out)


def rhs3_stage_back(sim: "RBC3D", back: np.ndarray) -> List[np.ndarray]:
    """4 arrays (z, padded y, Kx_r) -> the F coefficients (Nz, Ny, Kx_r): forward
    y transform, y Nyquist fold and truncation, the 3/2 rule's (Mx/Nx)(My/Ny)
    scaling, Chebyshev forward."""
    p = sim.p
    My, Mx = padded_length(p.Ny, p.dealias), padded_length(p.Nx, p.dealias)
    scale = (Mx / p.Nx) * (My / p.Ny)
    return [cheb_forward(_y_truncate(_fx.fft(b, axis=1), p.Ny) * scale, axis=0) for b in back]


def run_rbc3(p: RBC3Params, scheme: str, dt: float, nsteps: int, seed: int = 42) -> RBC3D:
    """Build the 3D RBC problem with the seeded initial b and advance nsteps (RK)."""
    sim = RBC3D(p)
    sim.set_b_grid(rbc3_initial_b(p, seed))
    for _ in range(nsteps):
        sim.step_rk(dt, TABLEAUS[scheme])
    return sim
