"""Host-side mirror of Tarang.jl's user API for the arch=GPU() timestep path.

Names and argument meanings follow the reference so that a script written
against Tarang.jl reads the same here (Julia's ``!`` suffix dropped):

    domain = ChannelDomain(256, 64; Lx=4.0, Lz=1.0)      src/extras/quick_domains.jl:109-121
    b = ScalarField(domain, "b"); u = VectorField(domain, "u")
    problem = IVP([p, b, u, tau_p, ...])                 src/core/problems/
    add_equation(problem, "...") / add_bc(problem, "...")
    solver = InitialValueSolver(problem, RK222(), dt=0.125)   src/core/solvers/solver_types.jl:993
    step(solver, dt) / run(solver, stop_time=...)        src/core/solvers/solver_stepping.jl:24-205

Everything numerical runs in libtarang_b200.so.  The equation strings are
matched against the Boussinesq template of test/test_subproblem_rk.jl:50-57
(the program the library implements); any other system raises
NotImplementedError instead of falling back to a CPU path.
"""
from __future__ import annotations

import ctypes
import math
import re
from ctypes import byref, c_double, c_float, c_int, c_longlong, c_size_t, c_void_p
from typing import Dict, List, Optional, Sequence

import numpy as np

from . import _lib as L
from ._lib import TarangError, check, lib

# ---------------------------------------------------------------------------
# Architectures and contexts (src/core/architectures.jl:107)
# ---------------------------------------------------------------------------


class CPU:
    """The reference's CPU architecture; not served by this library."""


class GPU:
    def __init__(self, device: int = 0):
        self.device = device


_CONTEXTS: Dict[int, c_void_p] = {}


def _context(device: int = 0) -> c_void_p:
    ctx = _CONTEXTS.get(device)
    if ctx is None:
        ctx = c_void_p()
        check(lib.tb_context_create(device, byref(ctx)))
        _CONTEXTS[device] = ctx
    return ctx


# ---------------------------------------------------------------------------
# Bases and domains
# ---------------------------------------------------------------------------


class RealFourier:
    def __init__(self, name: str = "x", size: int = 64, bounds=(0.0, 2 * math.pi), dealias: float = 1.0):
        self.name, self.size, self.bounds, self.dealias = name, int(size), tuple(map(float, bounds)), float(dealias)

    @property
    def length(self) -> float:
        return self.bounds[1] - self.bounds[0]


class ChebyshevT(RealFourier):
    pass


class Domain:
    """RealFourier x (, RealFourier y) x ChebyshevT z, or the doubly periodic
    RealFourier x RealFourier y of a PeriodicDomain."""

    def __init__(self, bases: Sequence, arch=None):
        self.bases = tuple(bases)
        self.arch = arch if arch is not None else GPU()
        if isinstance(self.arch, CPU):
            raise NotImplementedError("the B200 library serves arch=GPU() only")
        # doubly periodic: two RealFourier bases, no ChebyshevT direction
        self.periodic = len(self.bases) == 2 and not any(isinstance(b, ChebyshevT) for b in self.bases)
        if self.periodic:
            self.xbasis, self.ybasis = self.bases
            self.zbasis = None
        elif len(self.bases) == 3:
            self.xbasis, self.ybasis, self.zbasis = self.bases
        else:
            self.xbasis, self.zbasis = self.bases
            self.ybasis = None
        self._tplan = None

    @property
    def ndim(self) -> int:
        if self.periodic:
            return 2
        return 3 if self.ybasis is not None else 2

    @property
    def Nx(self) -> int:
        return self.xbasis.size

    @property
    def Ny(self) -> int:
        return self.ybasis.size if self.ybasis is not None else 1

    @property
    def Nz(self) -> int:
        return self.zbasis.size if self.zbasis is not None else 1

    @property
    def Nk(self) -> int:
        return self.Nx // 2 + 1

    def coeff_shape(self):
        """Coefficient layout of a field: (Nz, Nx/2+1), (Nz, Ny, Nx/2+1), or
        (Ny, Nx/2+1) on a periodic domain (rfft along x, fft along y)."""
        if self.periodic:
            return (self.Ny, self.Nk)
        return (self.Nz, self.Ny, self.Nk) if self.ndim == 3 else (self.Nz, self.Nk)

    def grid_shape(self):
        if self.periodic:
            return (self.Ny, self.Nx)
        return (self.Nz, self.Ny, self.Nx) if self.ndim == 3 else (self.Nz, self.Nx)

    def grids(self):
        """(x, [y,] z) grids: x_j = j Lx/Nx, z_j = a + (b-a)/2 (1 - cos(pi j/(Nz-1))) (basis_interface.jl:81-121)."""
        x = self.xbasis.bounds[0] + np.arange(self.Nx) * self.xbasis.length / self.Nx
        if self.periodic:
            return x, self.ybasis.bounds[0] + np.arange(self.Ny) * self.ybasis.length / self.Ny
        a, b = self.zbasis.bounds
        z = (b - a) / 2 * (-np.cos(np.pi * np.arange(self.Nz) / (self.Nz - 1))) + (b + a) / 2
        if self.ndim == 3:
            y = self.ybasis.bounds[0] + np.arange(self.Ny) * self.ybasis.length / self.Ny
            return x, y, z
        return x, z

    def transform_plan(self) -> "Plan":
        """A plan used only for field transforms (physics parameters unused)."""
        if self._tplan is None:
            if self.periodic:
                self._tplan = PeriodicTransform(self.Nx, self.Ny, device=self.arch.device)
            elif self.ndim == 3:
                self._tplan = Plan3D(self.Nx, self.Ny, self.Nz, 1.0, 1.0, L.TB_RK222, self.xbasis.length,
                                     self.ybasis.length, self.zbasis.length, device=self.arch.device)
            else:
                self._tplan = Plan(self, kappa=1.0, nu=1.0, b_bottom=0.0, b_top=0.0, timestepper=L.TB_RK222)
        return self._tplan


class PeriodicTransform:
    """FP64 grid <-> coefficient transforms of a doubly periodic domain on the
    device (tb_periodic_*): coefficients (Ny, Nx/2+1) = fft_y(rfft_x(grid)),
    unnormalised; backward with 1/(Nx Ny)."""

    def __init__(self, Nx: int, Ny: int, device: int = 0):
        self.Nx, self.Ny = int(Nx), int(Ny)
        self.ctx = _context(device)
        self.ptr = c_void_p()
        check(lib.tb_periodic_create(self.ctx, self.Nx, self.Ny, byref(self.ptr)), self.ctx)

    def __del__(self):
        ptr = getattr(self, "ptr", None)
        if ptr:
            lib.tb_periodic_destroy(ptr)
            self.ptr = None

    def forward(self, grid: np.ndarray) -> np.ndarray:
        g = np.ascontiguousarray(grid, dtype=np.float64)
        if g.shape != (self.Ny, self.Nx):
            raise ValueError(f"grid shape {g.shape}, expected {(self.Ny, self.Nx)}")
        out = np.empty((self.Ny, self.Nx // 2 + 1), np.complex128)
        check(lib.tb_periodic_forward(self.ptr, g.ctypes.data_as(c_void_p), out.ctypes.data_as(c_void_p),
                                      L.TB_HOST), self.ctx)
        return out

    def backward(self, coeff: np.ndarray) -> np.ndarray:
        c = np.ascontiguousarray(coeff, dtype=np.complex128)
        if c.shape != (self.Ny, self.Nx // 2 + 1):
            raise ValueError(f"coefficient shape {c.shape}, expected {(self.Ny, self.Nx // 2 + 1)}")
        out = np.empty((self.Ny, self.Nx), np.float64)
        check(lib.tb_periodic_backward(self.ptr, c.ctypes.data_as(c_void_p), out.ctypes.data_as(c_void_p),
                                       L.TB_HOST), self.ctx)
        return out


def PeriodicDomain(*N: int, L: Optional[Sequence[float]] = None, dtype=np.float64, device=None, arch=None,
                   dealias: float = 1.5) -> Domain:
    """RealFourier x RealFourier on [0, Lx) x [0, Ly), default 2 pi each
    (quick_domains.jl:33-58); the 2D form the library steps (decaying
    turbulence)."""
    if len(N) != 2:
        raise NotImplementedError("the B200 library steps 2D periodic domains")
    Ls = (2 * math.pi, 2 * math.pi) if L is None else tuple(L)
    arch = device if device is not None else arch
    xb = RealFourier("x", size=N[0], bounds=(0.0, Ls[0]), dealias=dealias)
    yb = RealFourier("y", size=N[1], bounds=(0.0, Ls[1]), dealias=dealias)
    return Domain((xb, yb), arch=arch)


def ChannelDomain(Nx: int, Nz: int, Lx: float = 2 * math.pi, Lz: float = 2.0, dtype=np.float64, arch=None,
                  dealias: float = 1.5) -> Domain:
    """RealFourier(x in [0,Lx)) x ChebyshevT(z in [0,Lz]) with the given dealias (quick_domains.jl:109-121)."""
    if dtype not in (np.float64, float):
        raise NotImplementedError("the FP64 path stores Float64 fields")
    return Domain((RealFourier("x", Nx, (0.0, Lx), dealias), ChebyshevT("z", Nz, (0.0, Lz), dealias)), arch)


def ChannelDomain3D(Nx: int, Ny: int, Nz: int, Lx: float = 4 * math.pi, Ly: float = 2 * math.pi, Lz: float = 2.0,
                    dtype=np.float64, arch=None, dealias: float = 1.5, zbounds=None) -> Domain:
    """RealFourier x, y x ChebyshevT z (quick_domains.jl:124-143: z in (-1, 1)
    by default there; zbounds overrides, e.g. (0, Lz))."""
    if dtype not in (np.float64, float):
        raise NotImplementedError("the FP64 path stores Float64 fields")
    zb = (-1.0, 1.0) if zbounds is None else tuple(map(float, zbounds))
    return Domain((RealFourier("x", Nx, (0.0, Lx), dealias), RealFourier("y", Ny, (0.0, Ly), dealias),
                   ChebyshevT("z", Nz, zb, dealias)), arch)


# ---------------------------------------------------------------------------
# Plans (the C ABI object behind a solver)
# ---------------------------------------------------------------------------

_TS_IDS = {"RK222": L.TB_RK222, "RK443": L.TB_RK443, "SBDF1": L.TB_SBDF1, "SBDF2": L.TB_SBDF2}


class Plan:
    def __init__(self, domain: Domain, kappa: float, nu: float, b_bottom: float, b_top: float, timestepper: int,
                 precision: int = L.TB_PREC_F64):
        self.domain = domain
        self.ctx = _context(domain.arch.device)
        d = L.tb_problem_desc()
        d.ndim = 2
        d.Nx, d.Ny, d.Nz = domain.Nx, 1, domain.Nz
        d.Lx, d.Ly, d.Lz = domain.xbasis.length, 1.0, domain.zbasis.length
        d.dealias = domain.xbasis.dealias if domain.xbasis.dealias > 1 else 1.5
        d.precision = precision
        d.timestepper = timestepper
        d.program = L.TB_PROGRAM_RBC
        d.kappa, d.nu, d.b_bottom, d.b_top = kappa, nu, b_bottom, b_top
        self.desc = d
        self.ptr = c_void_p()
        check(lib.tb_plan_create(self.ctx, byref(d), byref(self.ptr)), self.ctx)

    def __del__(self):
        ptr = getattr(self, "ptr", None)
        if ptr:
            lib.tb_plan_destroy(ptr)
            self.ptr = None

    # state I/O (host numpy, coefficient layout (Nz, Nk) complex128)
    def set_state(self, field: int, arr: np.ndarray) -> None:
        # the C call reads the field's whole extent from the pointer, so the
        # host array must have exactly the field's shape
        a = np.ascontiguousarray(arr, dtype=np.complex128)
        if a.shape != self._field_shape(field):
            raise ValueError(f"field {field}: shape {a.shape}, expected {self._field_shape(field)}")
        check(lib.tb_set_state(self.ptr, field, a.ctypes.data_as(c_void_p), L.TB_HOST), self.ctx)

    def get_state(self, field: int) -> np.ndarray:
        out = np.empty(self._field_shape(field), np.complex128)
        check(lib.tb_get_state(self.ptr, field, out.ctypes.data_as(c_void_p), L.TB_HOST), self.ctx)
        return out

    def _field_shape(self, field: int):
        return (7, self.domain.Nk) if field == L.TB_FIELD_TAU else (self.domain.Nz, self.domain.Nk)

    def _field_arrays(self, arrays: Dict[int, np.ndarray], writable: bool):
        fields = list(arrays)
        arrs = []
        for f in fields:
            a = arrays[f]
            if writable:
                if a.dtype != np.complex128 or not a.flags.c_contiguous or not a.flags.writeable:
                    raise ValueError("output buffers must be writable C-contiguous complex128 arrays")
            else:
                a = np.ascontiguousarray(a, dtype=np.complex128)
            if a.shape != self._field_shape(f):
                raise ValueError(f"field {f}: shape {a.shape}, expected {self._field_shape(f)}")
            arrs.append(a)
        fa = (c_int * len(fields))(*fields)
        pa = (c_void_p * len(fields))(*[a.ctypes.data for a in arrs])
        return fields, arrs, fa, pa

    def set_states(self, arrays: Dict[int, np.ndarray], keep_history: bool = False, wait: bool = True) -> None:
        """Several fields from host arrays in one call (one wait for all copies).
        A set restarts the multistep (SBDF) history unless keep_history.  With
        wait=False the call returns once the copies are queued (TB_NO_WAIT): a
        pinned source must stay unchanged until the plan's next wait (step,
        get_states, wait); the next step queues behind the copies."""
        fields, arrs, fa, pa = self._field_arrays(arrays, False)
        where = L.TB_HOST | (L.TB_KEEP_HISTORY if keep_history else 0) | (0 if wait else L.TB_NO_WAIT)
        check(lib.tb_set_states(self.ptr, len(fields), fa, pa, where), self.ctx)

    def get_states(self, out: Dict[int, np.ndarray]) -> Dict[int, np.ndarray]:
        """Fill out[field] (C-contiguous complex128 of the field's shape, e.g.
        pinned host memory) for every field in one call; returns out."""
        fields, arrs, fa, pa = self._field_arrays(out, True)
        check(lib.tb_get_states(self.ptr, len(fields), fa, pa, L.TB_HOST), self.ctx)
        return out

    def step(self, dt: float, nsteps: int = 1) -> None:
        check(lib.tb_step(self.ptr, float(dt), int(nsteps)), self.ctx)

    def sim_time(self) -> float:
        t, it = c_double(), c_longlong()
        check(lib.tb_sim_time(self.ptr, byref(t), byref(it)), self.ctx)
        return t.value

    # asynchronous stepping (several plans in flight)
    def step_async(self, dt: float, nsteps: int = 1, graph_steps: int = 1) -> None:
        check(lib.tb_step_async(self.ptr, float(dt), int(nsteps), int(graph_steps)), self.ctx)

    def idle(self) -> bool:
        v = c_int()
        check(lib.tb_plan_query(self.ptr, byref(v)), self.ctx)
        return bool(v.value)

    def wait(self) -> None:
        check(lib.tb_plan_wait(self.ptr), self.ctx)

    def device_bytes(self) -> int:
        v = c_size_t()
        check(lib.tb_plan_device_bytes(self.ptr, byref(v)), self.ctx)
        return int(v.value)

    def last_step_ms(self) -> float:
        ms = c_float()
        check(lib.tb_last_step_ms(self.ptr, byref(ms)), self.ctx)
        return ms.value

    def set_profiling(self, on: bool) -> None:
        check(lib.tb_set_profiling(self.ptr, 1 if on else 0), self.ctx)
        if on:
            check(lib.tb_profile_reset(self.ptr), self.ctx)

    def profile(self) -> Dict[str, tuple]:
        """{kernel name: (total ms, launches)} accumulated while profiling was on."""
        n = c_int()
        check(lib.tb_profile_count(self.ptr, byref(n)), self.ctx)
        out = {}
        buf = ctypes.create_string_buffer(64)
        for i in range(n.value):
            ms, cnt = c_double(), c_longlong()
            check(lib.tb_profile_entry(self.ptr, i, buf, 64, byref(ms), byref(cnt)), self.ctx)
            out[buf.value.decode()] = (ms.value, cnt.value)
        return out

    def set_wall_values(self, wall: int, value: np.ndarray, rate: Optional[np.ndarray] = None) -> None:
        """b at wall 0 (z = 0) or 1 (z = Lz): coefficients of the wall profile at
        the current time (complex Nx/2+1; (Ny, Nx/2+1) in 3D) and their rate."""
        v = np.ascontiguousarray(value, dtype=np.complex128)
        r = None if rate is None else np.ascontiguousarray(rate, dtype=np.complex128)
        check(lib.tb_set_wall_values(self.ptr, int(wall), v.ctypes.data_as(c_void_p),
                                     None if r is None else r.ctypes.data_as(c_void_p), L.TB_HOST), self.ctx)

    def save_state(self, path: str) -> None:
        """Grid-space NetCDF checkpoint of the state and clock (solver_checkpoint.jl:88-125)."""
        from .checkpoint import save_state

        save_state(self, path)

    def load_state(self, path: str) -> None:
        """Restore the state and clock from a checkpoint (solver_checkpoint.jl:146-194)."""
        from .checkpoint import load_state

        load_state(self, path)

    def variant(self):
        """(tau-solve partitions, 3D x-pass rows per CTA or 0): the plan's kernel shapes."""
        a, b = c_int(), c_int()
        check(lib.tb_plan_get_variant(self.ptr, byref(a), byref(b)), self.ctx)
        return a.value, b.value

    def set_variant(self, tau_parts: int = 0, xrows: int = 0) -> None:
        check(lib.tb_plan_set_variant(self.ptr, int(tau_parts), int(xrows)), self.ctx)

    def set_gemm_path(self, tensor_cores: bool) -> None:
        """Mixed precision: FP32 transform GEMMs on the tcgen05 tensor cores
        (True) or on the SIMT FP32 kernel (False).  The default is the SIMT
        kernel in 2D and the tensor cores in 3D (Nz <= 128)."""
        check(lib.tb_plan_set_gemm_path(self.ptr, 1 if tensor_cores else 0), self.ctx)

    def gemm_path(self) -> bool:
        v = c_int()
        check(lib.tb_plan_get_gemm_path(self.ptr, byref(v)), self.ctx)
        return bool(v.value)

    def tune(self, dt: float, trial_steps: int = 4):
        """Time every feasible kernel-shape combination on trial steps from the
        current state (restored afterwards) and keep the fastest."""
        a, b = c_int(), c_int()
        check(lib.tb_plan_tune(self.ptr, float(dt), int(trial_steps), byref(a), byref(b)), self.ctx)
        return a.value, b.value

    def kernels_per_step(self) -> int:
        n = c_int()
        check(lib.tb_kernels_per_step(self.ptr, byref(n)), self.ctx)
        return n.value

    # device transforms (torch tensors provide device memory)
    def forward(self, grid: np.ndarray) -> np.ndarray:
        import torch

        g = torch.as_tensor(np.ascontiguousarray(grid, dtype=np.float64), device="cuda")
        nf = g.numel() // (self.domain.Nz * self.domain.Nx)
        c = torch.empty(nf * self.domain.Nz * self.domain.Nk * 2, dtype=torch.float64, device="cuda")
        check(lib.tb_transform_forward(self.ptr, c_void_p(g.data_ptr()), c_void_p(c.data_ptr()), nf), self.ctx)
        out = c.cpu().numpy().view(np.complex128)
        return out.reshape(grid.shape[:-2] + (self.domain.Nz, self.domain.Nk))

    def backward(self, coeff: np.ndarray) -> np.ndarray:
        import torch

        c = torch.as_tensor(np.ascontiguousarray(coeff, dtype=np.complex128).view(np.float64), device="cuda")
        nf = c.numel() // (2 * self.domain.Nz * self.domain.Nk)
        g = torch.empty(nf * self.domain.Nz * self.domain.Nx, dtype=torch.float64, device="cuda")
        check(lib.tb_transform_backward(self.ptr, c_void_p(c.data_ptr()), c_void_p(g.data_ptr()), nf), self.ctx)
        return g.cpu().numpy().reshape(coeff.shape[:-2] + (self.domain.Nz, self.domain.Nx))

    def dealiased_multiply(self, a: np.ndarray, b: np.ndarray) -> np.ndarray:
        import torch

        ta = torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device="cuda")
        tb_ = torch.as_tensor(np.ascontiguousarray(b, dtype=np.float64), device="cuda")
        out = torch.empty_like(ta)
        check(lib.tb_dealiased_multiply(self.ptr, c_void_p(ta.data_ptr()), c_void_p(tb_.data_ptr()),
                                        c_void_p(out.data_ptr())), self.ctx)
        return out.cpu().numpy()

    def rhs_advection(self, b: np.ndarray, ux: np.ndarray, uz: np.ndarray):
        import torch

        inp = np.ascontiguousarray(np.stack([b, ux, uz]), dtype=np.complex128)
        ti = torch.as_tensor(inp.view(np.float64), device="cuda")
        to = torch.empty_like(ti)
        check(lib.tb_rhs_advection(self.ptr, c_void_p(ti.data_ptr()), c_void_p(to.data_ptr())), self.ctx)
        o = to.cpu().numpy().view(np.complex128)
        return o[0], o[1], o[2]


class Plan3D(Plan):
    """3D Rayleigh-Benard plan: RealFourier x, RealFourier y, ChebyshevT z
    (ChannelDomain3D, src/extras/quick_domains.jl:124-143; bounds (0, Lz) in z).

    Coefficient fields are complex (Nz, Ny, Nx/2+1) arrays (the reference's
    column-major (Nx/2+1, Ny, Nz): rfft along x, fft along y in FFT order, then
    ChebyshevT along z); taus are (9, Ny, Nx/2+1) in the order tau_p, tau_b1,
    tau_b2, tau_u1x, tau_u1y, tau_u1z, tau_u2x, tau_u2y, tau_u2z.  Fields: TB_FIELD_B,
    TB_FIELD_UX, TB_FIELD_UY, TB_FIELD_UZ, TB_FIELD_P, TB_FIELD_TAU.
    """

    def __init__(self, Nx: int, Ny: int, Nz: int, kappa: float, nu: float, timestepper: int = L.TB_RK222,
                 Lx: float = 4.0, Ly: float = 4.0, Lz: float = 1.0, b_bottom: Optional[float] = None,
                 b_top: float = 0.0, precision: int = L.TB_PREC_F64, device: int = 0):
        self.Nx, self.Ny, self.Nz = int(Nx), int(Ny), int(Nz)
        self.Kx = self.Nx // 2 + 1
        self.domain = None
        self.ctx = _context(device)
        d = rbc3_desc(Nx, Ny, Nz, kappa, nu, timestepper, Lx, Ly, Lz, b_bottom, b_top, precision)
        self.desc = d
        self.ptr = c_void_p()
        check(lib.tb_plan_create(self.ctx, byref(d), byref(self.ptr)), self.ctx)

    def _shape(self, field: int):
        return (9, self.Ny, self.Kx) if field == L.TB_FIELD_TAU else (self.Nz, self.Ny, self.Kx)

    def set_state(self, field: int, arr: np.ndarray) -> None:
        a = np.ascontiguousarray(arr, dtype=np.complex128)
        if a.shape != self._shape(field):
            raise ValueError(f"field {field}: shape {a.shape}, expected {self._shape(field)}")
        check(lib.tb_set_state(self.ptr, field, a.ctypes.data_as(c_void_p), L.TB_HOST), self.ctx)

    def get_state(self, field: int) -> np.ndarray:
        out = np.empty(self._shape(field), np.complex128)
        check(lib.tb_get_state(self.ptr, field, out.ctypes.data_as(c_void_p), L.TB_HOST), self.ctx)
        return out

    def forward(self, grid: np.ndarray) -> np.ndarray:
        """Grid (Nz, Ny, Nx) real -> coefficients (Nz, Ny, Nx/2+1) on the device."""
        import torch

        g = torch.as_tensor(np.ascontiguousarray(grid, dtype=np.float64), device="cuda")
        c = torch.empty(self.Nz * self.Ny * self.Kx * 2, dtype=torch.float64, device="cuda")
        check(lib.tb_transform_forward(self.ptr, c_void_p(g.data_ptr()), c_void_p(c.data_ptr()), 1), self.ctx)
        return c.cpu().numpy().view(np.complex128).reshape(self.Nz, self.Ny, self.Kx)

    def backward(self, coeff: np.ndarray) -> np.ndarray:
        """Coefficients (Nz, Ny, Nx/2+1) -> grid (Nz, Ny, Nx) on the device."""
        import torch

        c = torch.as_tensor(np.ascontiguousarray(coeff, dtype=np.complex128).view(np.float64), device="cuda")
        g = torch.empty(self.Nz * self.Ny * self.Nx, dtype=torch.float64, device="cuda")
        check(lib.tb_transform_backward(self.ptr, c_void_p(c.data_ptr()), c_void_p(g.data_ptr()), 1), self.ctx)
        return g.cpu().numpy().reshape(self.Nz, self.Ny, self.Nx)


def rbc3_desc(Nx: int, Ny: int, Nz: int, kappa: float, nu: float, timestepper: int = 0, Lx: float = 4.0,
              Ly: float = 4.0, Lz: float = 1.0, b_bottom: Optional[float] = None, b_top: float = 0.0,
              precision: int = 0):
    d = L.tb_problem_desc()
    d.ndim, d.Nx, d.Ny, d.Nz = 3, int(Nx), int(Ny), int(Nz)
    d.Lx, d.Ly, d.Lz, d.dealias = float(Lx), float(Ly), float(Lz), 1.5
    d.precision, d.timestepper, d.program = int(precision), int(timestepper), L.TB_PROGRAM_RBC
    d.kappa, d.nu = float(kappa), float(nu)
    d.b_bottom, d.b_top = float(Lz if b_bottom is None else b_bottom), float(b_top)
    return d


# ---------------------------------------------------------------------------
# Fields
# ---------------------------------------------------------------------------


class Ensemble:
    """Independent plans (uneven sizes, own parameters and dt) stepped together.

    Counterpart of the reference's batched ensemble path
    (src/core/timesteppers/mode_batch.jl:23-668): ``run`` steps every member
    ``nsteps`` at its own dt and returns the per-member completion times (ms
    from the run's start, device clock) and the run's total; ``tune`` picks the
    worker-stream count and steps per graph by timing them on the members
    (their state is restored afterwards).
    """

    def __init__(self, plans: Sequence[Plan]):
        if not plans:
            raise ValueError("empty ensemble")
        self.plans = list(plans)
        self.ctx = self.plans[0].ctx
        arr = (c_void_p * len(self.plans))(*[p.ptr.value for p in self.plans])
        self.ptr = c_void_p()
        check(lib.tb_ensemble_create(self.ctx, len(self.plans), arr, byref(self.ptr)), self.ctx)

    def __del__(self):
        ptr = getattr(self, "ptr", None)
        if ptr:
            lib.tb_ensemble_destroy(ptr)
            self.ptr = None

    def _dts(self, dt) -> np.ndarray:
        d = np.broadcast_to(np.asarray(dt, dtype=np.float64), (len(self.plans),))
        return np.ascontiguousarray(d)

    def tune(self, dt, trial_steps: int = 8):
        d = self._dts(dt)
        s, g = c_int(), c_int()
        check(lib.tb_ensemble_tune(self.ptr, d.ctypes.data_as(c_void_p), int(trial_steps), byref(s), byref(g)),
              self.ctx)
        return s.value, g.value

    def set_config(self, streams: int, graph_steps: int) -> None:
        check(lib.tb_ensemble_set_config(self.ptr, int(streams), int(graph_steps)), self.ctx)

    def config(self):
        s, g = c_int(), c_int()
        check(lib.tb_ensemble_config(self.ptr, byref(s), byref(g)), self.ctx)
        return s.value, g.value

    def set_form(self, fused: bool) -> None:
        """Fused: same-shape members stepped as one stacked plan per shape."""
        check(lib.tb_ensemble_set_form(self.ptr, 1 if fused else 0), self.ctx)

    def form(self):
        """(fused, number of stacked group plans)."""
        f, g = c_int(), c_int()
        check(lib.tb_ensemble_get_form(self.ptr, byref(f), byref(g)), self.ctx)
        return bool(f.value), g.value

    def run(self, dt, nsteps: int):
        d = self._dts(dt)
        ms = np.zeros(len(self.plans), dtype=np.float32)
        tot = c_float()
        check(lib.tb_ensemble_run(self.ptr, d.ctypes.data_as(c_void_p), int(nsteps), ms.ctypes.data_as(c_void_p),
                                  byref(tot)), self.ctx)
        return ms, tot.value


class Turb2D:
    """Doubly periodic 2D decaying turbulence in FP32 (DiagonalIMEX_SBDF2 by
    default, or DiagonalIMEX_RK222 / RK443 with timestepper=TB_RK222 /
    TB_RK443), the reference's examples/2d_decaying_turbulence_gpu.jl on the C
    ABI.  Coefficients are complex (Ny, Nx/2+1) arrays (rfft along x, fft
    along y)."""

    def __init__(self, Nx: int, Ny: int, nu: float, q0_spec: np.ndarray, Lx: float = 2 * math.pi,
                 Ly: float = 2 * math.pi, device: int = 0, timestepper: int = L.TB_SBDF2):
        self.Nx, self.Ny = int(Nx), int(Ny)
        self.ctx = _context(device)
        d = turb_desc(Nx, Ny, nu, Lx, Ly, timestepper)
        q = np.ascontiguousarray(q0_spec, dtype=np.complex128)
        if q.shape != (self.Ny, self.Nx // 2 + 1):
            raise ValueError(f"vorticity shape {q.shape}, expected {(self.Ny, self.Nx // 2 + 1)}")
        self.ptr = c_void_p()
        check(lib.tb_turb_create(self.ctx, byref(d), q.ctypes.data_as(c_void_p), byref(self.ptr)), self.ctx)

    def __del__(self):
        ptr = getattr(self, "ptr", None)
        if ptr:
            lib.tb_turb_destroy(ptr)
            self.ptr = None

    def step(self, dt: float, nsteps: int = 1) -> None:
        check(lib.tb_turb_step(self.ptr, float(dt), int(nsteps)), self.ctx)

    def set_vorticity(self, q_spec: np.ndarray) -> None:
        """Replace q (complex (Ny, Nx/2+1)); the step history restarts."""
        q = np.ascontiguousarray(q_spec, dtype=np.complex128)
        if q.shape != (self.Ny, self.Nx // 2 + 1):
            raise ValueError(f"vorticity shape {q.shape}, expected {(self.Ny, self.Nx // 2 + 1)}")
        check(lib.tb_turb_set_vorticity(self.ptr, q.ctypes.data_as(c_void_p)), self.ctx)

    def vorticity(self) -> np.ndarray:
        out = np.zeros((self.Ny, self.Nx // 2 + 1), dtype=np.complex128)
        check(lib.tb_turb_get_vorticity(self.ptr, out.ctypes.data_as(c_void_p)), self.ctx)
        return out


def turb_desc(Nx: int, Ny: int, nu: float, Lx: float = 2 * math.pi, Ly: float = 2 * math.pi,
              timestepper: int = L.TB_SBDF2):
    """Descriptor of the doubly periodic vorticity problem; timestepper
    TB_SBDF2 (DiagonalIMEX_SBDF2), TB_RK222 or TB_RK443 (DiagonalIMEX_RK222 /
    RK443)."""
    d = L.tb_problem_desc()
    d.ndim, d.Nx, d.Ny, d.Nz = 2, int(Nx), int(Ny), 1
    d.Lx, d.Ly, d.Lz, d.dealias = float(Lx), float(Ly), 1.0, 1.5
    d.precision, d.timestepper, d.program = 0, int(timestepper), L.TB_PROGRAM_TURB2D
    d.kappa, d.nu, d.b_bottom, d.b_top = 0.0, float(nu), 0.0, 0.0
    return d


def rbc_desc(Nx: int, Nz: int, kappa: float, nu: float, timestepper: int = 0, Lx: float = 4.0, Lz: float = 1.0,
             b_bottom: Optional[float] = None, b_top: float = 0.0):
    d = L.tb_problem_desc()
    d.ndim, d.Nx, d.Ny, d.Nz = 2, int(Nx), 1, int(Nz)
    d.Lx, d.Ly, d.Lz, d.dealias = float(Lx), 1.0, float(Lz), 1.5
    d.precision, d.timestepper, d.program = L.TB_PREC_F64, int(timestepper), L.TB_PROGRAM_RBC
    d.kappa, d.nu = float(kappa), float(nu)
    d.b_bottom, d.b_top = float(Lz if b_bottom is None else b_bottom), float(b_top)
    return d


class Server:
    """Request server with continuous batching (tb_server_* in the C ABI).

    ``submit`` takes a problem descriptor (``rbc_desc`` / ``turb_desc``), dt,
    the step count and the initial data (RBC: buoyancy grid (Nz, Nx); TURB2D:
    vorticity coefficients (Ny, Nx/2+1) complex) and returns an id; results
    come back as coefficient arrays once the request is done."""

    def __init__(self, budget_bytes: int, max_running: int = 16, chunk_steps: int = 10, device: int = 0):
        self.ctx = _context(device)
        self.ptr = c_void_p()
        self._keep = {}
        self._shape = {}
        check(lib.tb_server_create(self.ctx, int(budget_bytes), int(max_running), int(chunk_steps),
                                   byref(self.ptr)), self.ctx)

    def __del__(self):
        self.close()

    def close(self):
        ptr = getattr(self, "ptr", None)
        if ptr:
            lib.tb_server_destroy(ptr)
            self.ptr = None

    def set_cohort(self, max_members: int) -> None:
        """Same-shape RBC requests at one dt, with step counts within 25 % of
        each other, queued together run as one stacked plan of up to
        ``max_members`` (1, the default: every request alone)."""
        check(lib.tb_server_set_cohort(self.ptr, int(max_members)), self.ctx)

    def submit(self, desc, dt: float, nsteps: int, init: np.ndarray) -> int:
        if desc.program == L.TB_PROGRAM_TURB2D:
            data = np.ascontiguousarray(init, dtype=np.complex128)
            shape = (desc.Ny, desc.Nx // 2 + 1)
            if data.shape != shape:
                raise ValueError(f"initial vorticity shape {data.shape}, expected {shape}")
            nf = 1
        else:
            data = np.ascontiguousarray(init, dtype=np.float64)
            if data.shape != (desc.Nz, desc.Nx):
                raise ValueError(f"initial grid shape {data.shape}, expected {(desc.Nz, desc.Nx)}")
            shape = (desc.Nz, desc.Nx // 2 + 1)
            nf = 3
        r = L.tb_request()
        r.desc, r.dt, r.nsteps = desc, float(dt), int(nsteps)
        r.init_grid = data.ctypes.data_as(c_void_p)
        rid = c_longlong()
        check(lib.tb_server_submit(self.ptr, byref(r), byref(rid)), self.ctx)
        self._shape[rid.value] = (shape, nf)
        return rid.value

    def poll(self, rid: int):
        st, t = c_int(), c_double()
        check(lib.tb_server_poll(self.ptr, int(rid), byref(st), byref(t)), self.ctx)
        return st.value, t.value

    def result(self, rid: int):
        shape, nf = self._shape[rid]
        out = []
        for f in range(nf):
            a = np.zeros(shape, dtype=np.complex128)
            n = c_size_t()
            check(lib.tb_server_result(self.ptr, int(rid), f, a.ctypes.data_as(c_void_p), byref(n)), self.ctx)
            out.append(a)
        return out

    def wait_all(self) -> None:
        check(lib.tb_server_wait_all(self.ptr), self.ctx)

    def stats(self) -> Dict[str, float]:
        st = L.tb_server_stats()
        check(lib.tb_server_get_stats(self.ptr, byref(st)), self.ctx)
        return {name: getattr(st, name) for name, _ in st._fields_}


class ScalarField:
    """A scalar field on a domain (or a tau field with ``bases=(xbasis,)`` / ``()``).

    Data are held in coefficient layout (Nz, Nx/2+1) complex, the reference's
    ``:c`` storage; ``f["g"]`` / ``f["c"]`` read and write grid / coefficient data.
    """

    def __init__(self, domain: Domain, name: str, bases: Optional[tuple] = None):
        self.domain = domain
        self.name = name
        self.bases = domain.bases if bases is None else tuple(bases)
        full = len(self.bases) == len(domain.bases)
        if full:
            shape = domain.coeff_shape()
        elif not self.bases:  # a constant (gauge multiplier)
            shape = ()
        else:  # a tau field on the Fourier bases
            shape = (domain.Ny, domain.Nk) if domain.ndim == 3 else (domain.Nk,)
        self._coeff = np.zeros(shape, np.complex128)
        self._solver = None
        self._slot = None  # (field selector, row) inside the solver's plan

    def _pull(self) -> None:
        if self._solver is not None:
            self._coeff = self._solver._read(self._slot)

    def _push(self) -> None:
        if self._solver is not None:
            self._solver._write(self._slot, self._coeff)

    def __getitem__(self, layout: str) -> np.ndarray:
        self._pull()
        if layout == "c":
            return self._coeff.copy()
        if layout == "g":
            if len(self.bases) != len(self.domain.bases):
                raise NotImplementedError("grid view of tau fields")
            return self.domain.transform_plan().backward(self._coeff)
        raise KeyError(layout)

    def __setitem__(self, layout: str, value) -> None:
        if layout == "c":
            self._coeff = np.array(value, dtype=np.complex128).reshape(self._coeff.shape)
        elif layout == "g":
            g = np.broadcast_to(np.asarray(value, dtype=np.float64), self.domain.grid_shape())
            self._coeff = self.domain.transform_plan().forward(np.ascontiguousarray(g))
        else:
            raise KeyError(layout)
        self._push()


class VectorField:
    def __init__(self, domain: Domain, name: str, bases: Optional[tuple] = None):
        self.domain = domain
        self.name = name
        comps = ("x", "y") if domain.periodic else (("x", "y", "z") if domain.ndim == 3 else ("x", "z"))
        self.components = [ScalarField(domain, f"{name}_{c}", bases) for c in comps]


def unit_vector_fields(domain: Domain):
    """Constant unit vectors ((ex, [ey,] ez)); used only as tokens in equation strings."""
    return ("ex", "ey", "ez") if domain.ndim == 3 else ("ex", "ez")


# ---------------------------------------------------------------------------
# Problems, time steppers, solvers
# ---------------------------------------------------------------------------


class IVP:
    def __init__(self, variables: List):
        self.variables = list(variables)
        self.parameters: Dict[str, object] = {}
        self.equations: List[str] = []
        self.bcs: List[str] = []


def add_parameters(problem: IVP, **kw) -> None:
    problem.parameters.update(kw)


def add_equation(problem: IVP, eq: str) -> None:
    problem.equations.append(eq)


def add_bc(problem: IVP, bc: str) -> None:
    problem.bcs.append(bc)


class _TS:
    name = ""

    def __repr__(self):
        return self.name + "()"


class RK222(_TS):
    name = "RK222"


class RK443(_TS):
    name = "RK443"


class SBDF1(_TS):
    name = "SBDF1"


class SBDF2(_TS):
    name = "SBDF2"


class DiagonalIMEX_RK222(_TS):
    """Diagonal implicit treatment per Fourier mode (pure Fourier problems)."""
    name = "DiagonalIMEX_RK222"


class DiagonalIMEX_RK443(_TS):
    name = "DiagonalIMEX_RK443"


class DiagonalIMEX_SBDF2(_TS):
    name = "DiagonalIMEX_SBDF2"


_DIAG_TS = {"DiagonalIMEX_RK222": L.TB_RK222, "DiagonalIMEX_RK443": L.TB_RK443, "DiagonalIMEX_SBDF2": L.TB_SBDF2}


def _norm(s: str) -> str:
    s = s.replace(" ", "").replace("∂t", "dt").replace("τ_lift", "lift").replace("·", "⋅")
    return s


def _value(tok: str, params: Dict[str, object]) -> float:
    try:
        return float(tok)
    except ValueError:
        if tok in params:
            return float(params[tok])
        raise NotImplementedError(f"boundary value {tok!r} is not a number or scalar parameter")


def _match_boussinesq(problem: IVP):
    """Recognise the Boussinesq system of test/test_subproblem_rk.jl:50-57."""
    P = problem.parameters
    eqs = [_norm(e) for e in problem.equations]
    cont = scal = mom = None
    for e in eqs:
        m = re.fullmatch(r"trace\(grad_(\w+)\)\+(\w+)=0", e)
        if m:
            cont = m
            continue
        m = re.fullmatch(r"dt\((\w+)\)-(\w+)\*div\(grad_\1\)\+lift\((\w+)\)=-(\w+)⋅∇\(\1\)", e)
        if m:
            scal = m
            continue
        m = re.fullmatch(r"dt\((\w+)\)-(\w+)\*div\(grad_\1\)\+∇\((\w+)\)-(\w+)\*ez\+lift\((\w+)\)=-\1⋅∇\(\1\)", e)
        if m:
            mom = m
            continue
        raise NotImplementedError(f"equation not in the supported Boussinesq program: {e!r}")
    if not (cont and scal and mom):
        raise NotImplementedError("the B200 path implements the full Boussinesq system (continuity, b, u)")
    bname, kname = scal.group(1), scal.group(2)
    uname, nname, pname = mom.group(1), mom.group(2), mom.group(3)
    if mom.group(4) != bname or scal.group(4) != uname or cont.group(1) != uname:
        raise NotImplementedError("inconsistent field names in the Boussinesq system")
    Lz = None
    bvals = {}
    saw_integ = False
    for bc in (_norm(b) for b in problem.bcs):
        m = re.fullmatch(r"(\w+)\(z=([\w.+-]+)\)=([\w.+-]+)", bc)
        if m:
            fld, zpos, val = m.group(1), m.group(2), m.group(3)
            z = _value(zpos, P)
            v = _value(val, P)
            if fld == bname:
                bvals[z] = v
            elif fld == uname:
                if v != 0.0:
                    raise NotImplementedError("only no-slip velocity walls are implemented")
            else:
                raise NotImplementedError(f"boundary condition on unknown field {fld!r}")
            continue
        if re.fullmatch(rf"integ\({pname}\)=0", bc):
            saw_integ = True
            continue
        raise NotImplementedError(f"boundary condition not supported: {bc!r}")
    if len(bvals) != 2 or not saw_integ:
        raise NotImplementedError("expected b at both walls and integ(p) = 0")
    z0, z1 = sorted(bvals)
    return dict(kappa=_value(kname, P), nu=_value(nname, P), b_bottom=bvals[z0], b_top=bvals[z1],
                names=dict(b=bname, u=uname, p=pname))


def _match_vorticity(problem: IVP):
    """Recognise the 2D vorticity system of examples/2d_decaying_turbulence_gpu.jl:
    dt(q) - nu*Δ(q) = -u⋅∇(q),  Δ(psi) + tau_psi - q = 0,  u - skew(grad(psi)) = 0,
    integ(psi) = 0."""
    P = problem.parameters
    trans = poisson = vel = None
    for e in (_norm(e) for e in problem.equations):
        m = re.fullmatch(r"dt\((\w+)\)-(\w+)\*Δ\(\1\)=-(\w+)⋅∇\(\1\)", e)
        if m:
            trans = m
            continue
        m = re.fullmatch(r"Δ\((\w+)\)\+(\w+)-(\w+)=0", e)
        if m:
            poisson = m
            continue
        m = re.fullmatch(r"(\w+)-skew\(grad\((\w+)\)\)=0", e)
        if m:
            vel = m
            continue
        raise NotImplementedError(f"equation not in the supported vorticity program: {e!r}")
    if not (trans and poisson and vel):
        raise NotImplementedError("the B200 path implements the full vorticity system (q, psi, u)")
    qname, nuname, uname = trans.group(1), trans.group(2), trans.group(3)
    psiname, tauname = poisson.group(1), poisson.group(2)
    if poisson.group(3) != qname or vel.group(1) != uname or vel.group(2) != psiname:
        raise NotImplementedError("inconsistent field names in the vorticity system")
    bcs = [_norm(b) for b in problem.bcs]
    if bcs != [f"integ({psiname})=0"]:
        raise NotImplementedError("expected the single gauge condition integ(psi) = 0")
    return dict(nu=_value(nuname, P), names=dict(q=qname, psi=psiname, u=uname, tau=tauname))


class InitialValueSolver:
    """Builds the library plan for the problem and binds its fields to the plan's state."""

    def __init__(self, problem: IVP, timestepper: _TS, dt: Optional[float] = None):
        for v in problem.variables:
            dom = v.domain
            if getattr(dom, "periodic", False):
                self._init_periodic(problem, timestepper, dt, dom)
                return
        self.periodic = False
        if timestepper.name not in _TS_IDS:
            raise NotImplementedError(f"{timestepper!r} on a ChebyshevT problem (use RK222/RK443/SBDF1/SBDF2)")
        spec = _match_boussinesq(problem)
        fields = {}
        domain = None
        for v in problem.variables:
            if isinstance(v, VectorField):
                fields[v.name] = v
                domain = v.domain
            else:
                fields[v.name] = v
                if len(v.bases) == len(v.domain.bases):
                    domain = v.domain
        self.domain = domain
        self.problem = problem
        self.timestepper = timestepper
        self.dt = dt
        ts = _TS_IDS[timestepper.name]
        if domain.ndim == 3:
            self.plan = Plan3D(domain.Nx, domain.Ny, domain.Nz, spec["kappa"], spec["nu"], ts, domain.xbasis.length,
                               domain.ybasis.length, domain.zbasis.length, spec["b_bottom"], spec["b_top"],
                               device=domain.arch.device)
        else:
            self.plan = Plan(domain, spec["kappa"], spec["nu"], spec["b_bottom"], spec["b_top"], ts)
        names = spec["names"]
        b, u, p = fields[names["b"]], fields[names["u"]], fields[names["p"]]
        ucomp = ([L.TB_FIELD_UX, L.TB_FIELD_UY, L.TB_FIELD_UZ] if domain.ndim == 3 else [L.TB_FIELD_UX, L.TB_FIELD_UZ])
        binds = [(b, (L.TB_FIELD_B, None))] + [(c, (sel, None)) for c, sel in zip(u.components, ucomp)] + \
                [(p, (L.TB_FIELD_P, None))]
        for f, slot in binds:
            f._solver, f._slot = self, slot
            f._push()
        self.sim_time = 0.0
        self.iteration = 0

    def _init_periodic(self, problem: IVP, timestepper: _TS, dt: Optional[float], domain: Domain) -> None:
        """The doubly periodic vorticity problem on the FP32 turbulence program;
        psi and u are derived from q on every read (psi^ = -q^/k^2, 0 at k = 0;
        u = skew(grad psi) = (-d_y psi, d_x psi))."""
        if timestepper.name not in _DIAG_TS:
            raise NotImplementedError(f"{timestepper!r} on a periodic problem (use DiagonalIMEX_SBDF2/RK222/RK443)")
        spec = _match_vorticity(problem)
        fields = {v.name: v for v in problem.variables}
        self.periodic = True
        self.domain, self.problem, self.timestepper, self.dt = domain, problem, timestepper, dt
        names = spec["names"]
        q = fields[names["q"]]
        self.plan = Turb2D(domain.Nx, domain.Ny, spec["nu"], q._coeff, domain.xbasis.length, domain.ybasis.length,
                           device=domain.arch.device, timestepper=_DIAG_TS[timestepper.name])
        kx = 2 * np.pi / domain.xbasis.length * np.arange(domain.Nk)
        ky = 2 * np.pi / domain.ybasis.length * np.concatenate(
            [np.arange(domain.Ny // 2), np.arange(-(domain.Ny // 2), 0)])
        self._kx, self._ky = kx[None, :], ky[:, None]
        u = fields[names["u"]]
        binds = [(q, "q"), (fields[names["psi"]], "psi"), (u.components[0], "ux"), (u.components[1], "uy"),
                 (fields[names["tau"]], "tau")]
        for f, slot in binds:
            f._solver, f._slot = self, slot
        self.sim_time = 0.0
        self.iteration = 0

    def _psi(self) -> np.ndarray:
        q = self.plan.vorticity()
        k2 = self._kx ** 2 + self._ky ** 2
        return np.where(k2 > 1e-12, -q / np.where(k2 > 1e-12, k2, 1.0), 0.0)

    def _read(self, slot):
        if not self.periodic:
            sel, row = slot
            data = self.plan.get_state(sel)
            return data if row is None else data[row].copy()
        if slot == "q":
            return self.plan.vorticity()
        if slot == "psi":
            return self._psi()
        if slot == "ux":
            return -1j * self._ky * self._psi()
        if slot == "uy":
            return 1j * self._kx * self._psi()
        return np.zeros((), np.complex128)  # the gauge multiplier vanishes at the solution

    def _write(self, slot, coeff: np.ndarray) -> None:
        if not self.periodic:
            sel, row = slot
            if row is None:
                self.plan.set_state(sel, coeff)
            else:
                taus = self.plan.get_state(sel)
                taus[row] = coeff
                self.plan.set_state(sel, taus)
            return
        if slot != "q":
            raise NotImplementedError("psi and u follow from q on a periodic problem; set q")
        self.plan.set_vorticity(coeff)

    def step(self, dt: Optional[float] = None, nsteps: int = 1) -> None:
        dt = self.dt if dt is None else dt
        if dt is None:
            raise ValueError("dt not given")
        self.plan.step(dt, nsteps)
        if self.periodic:
            self.sim_time += nsteps * dt
            self.iteration += nsteps
            return
        t, it = c_double(), c_longlong()
        check(lib.tb_sim_time(self.plan.ptr, byref(t), byref(it)), self.plan.ctx)
        self.sim_time, self.iteration = t.value, it.value


def step(solver: InitialValueSolver, dt: Optional[float] = None) -> None:
    """step!(solver, dt) (solver_stepping.jl:24-38)."""
    solver.step(dt)


def run(solver: InitialValueSolver, stop_time: Optional[float] = None, stop_iteration: Optional[int] = None,
        log_interval: int = 0, dt: Optional[float] = None, callbacks: Sequence = ()) -> None:
    """run!(solver; stop_time, stop_iteration, callbacks) (solver_stepping.jl:115-205),
    fixed dt; callbacks are (interval, fn) pairs, fn(solver) called every
    interval iterations (the reference's ``interval => fn``)."""
    dt = solver.dt if dt is None else dt
    if dt is None:
        raise ValueError("dt not given")
    n = None
    if stop_iteration is not None:
        n = int(stop_iteration) - solver.iteration
    if stop_time is not None:
        nt = int(math.ceil((stop_time - solver.sim_time) / dt - 1e-9))
        n = nt if n is None else min(n, nt)
    if n is None:
        raise ValueError("give stop_time or stop_iteration")
    cbs = [(int(k), fn) for k, fn in callbacks]
    if any(k < 1 for k, _ in cbs):
        raise ValueError("callback intervals must be >= 1")
    end = solver.iteration + max(n, 0)
    while solver.iteration < end:
        nxt = end
        for k, _ in cbs:
            nxt = min(nxt, (solver.iteration // k + 1) * k)
        solver.step(dt, nxt - solver.iteration)
        for k, fn in cbs:
            if solver.iteration % k == 0:
                fn(solver)
