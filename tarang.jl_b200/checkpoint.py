"""Checkpoints of a plan as NetCDF files: the counterpart of the reference's
save_state / load_state! (src/tools/solver_checkpoint.jl:88-194).

The state is written in grid space (the reference transforms every field to
:g before writing): one float64 variable per field (b, ux, [uy,] uz, p) with
dimensions (z, [y,] x) - the reference's column-major (x, [y,] z) arrays -
and the global attributes sim_time, iteration and dt.  The file is written
under a temporary name and renamed, so a file with the clock attributes is
always complete (the reference writes them last for the same reason).
Loading requires all three clock attributes, as the reference does, and
restarts the multistep history.  NetCDF classic (64-bit offset) format via
scipy.io.netcdf_file.
"""
from __future__ import annotations

import ctypes
import os
from typing import Dict, Sequence, Tuple

import numpy as np

CLOCK_ATTRS = ("sim_time", "iteration", "dt")


def field_names(ndim: int) -> Tuple[str, ...]:
    return ("b", "ux", "uy", "uz", "p") if ndim == 3 else ("b", "ux", "uz", "p")


def write_checkpoint(path: str, fields: Dict[str, np.ndarray], clock: Sequence[float]) -> None:
    """Grid fields (each (Nz, Nx) or (Nz, Ny, Nx)) and the clock (sim_time,
    iteration, dt) to a NetCDF file at path."""
    from scipy.io import netcdf_file

    first = next(iter(fields.values()))
    dims = ("z", "y", "x") if first.ndim == 3 else ("z", "x")
    tmp = path + ".partial"
    with netcdf_file(tmp, "w", version=2) as f:
        for name, n in zip(dims, first.shape):
            f.createDimension(name, n)
        for name, arr in fields.items():
            v = f.createVariable(name, "d", dims)
            v[...] = np.asarray(arr, dtype=np.float64)
        f.sim_time = np.array([clock[0]], dtype=np.float64)  # double attributes, not float32
        # the reference writes the iteration as a Julia Int (64-bit); classic
        # NetCDF has no 64-bit integer, and a double holds every count up to
        # 2^53 exactly, where a 32-bit int would wrap at 2^31
        f.iteration = np.array([float(int(clock[1]))], dtype=np.float64)
        f.dt = np.array([clock[2]], dtype=np.float64)
    os.replace(tmp, path)


def read_checkpoint(path: str, names: Sequence[str]):
    """(fields stacked in `names` order, clock array) from a checkpoint file."""
    from scipy.io import netcdf_file

    with netcdf_file(path, "r", mmap=False) as f:
        attrs = f._attributes
        missing = [k for k in CLOCK_ATTRS if k not in attrs]
        if missing:
            raise ValueError(f"checkpoint '{path}' lacks the clock attribute(s) {', '.join(missing)}; the fields "
                             "would load with the wrong simulation time")
        absent = [n for n in names if n not in f.variables]
        if absent:
            raise KeyError(f"checkpoint '{path}' has no variable(s) {', '.join(absent)}")
        data = np.stack([np.array(f.variables[n][...], dtype=np.float64) for n in names])
        clock = np.array([np.asarray(attrs[k], dtype=np.float64).ravel()[0] for k in CLOCK_ATTRS])
    return data, clock


def save_state(plan, path: str) -> None:
    """Stage the plan's state to the grid on the device and write it (the
    device-to-host copy runs on a side stream; this waits for it)."""
    from ._lib import check, lib

    ndim = 3 if hasattr(plan, "Ny") else 2
    names = field_names(ndim)
    shape = (plan.Nz, plan.Ny, plan.Nx) if ndim == 3 else (plan.domain.Nz, plan.domain.Nx)
    host = np.empty((len(names),) + shape, np.float64)
    clock = np.zeros(3)
    check(lib.tb_checkpoint_stage(plan.ptr, host.ctypes.data_as(ctypes.c_void_p), host.size,
                                  clock.ctypes.data_as(ctypes.c_void_p)), plan.ctx)
    check(lib.tb_checkpoint_wait(plan.ptr), plan.ctx)
    write_checkpoint(path, dict(zip(names, host)), clock)


def load_state(plan, path: str) -> None:
    """Set the plan's state and clock from a checkpoint file."""
    from ._lib import TB_HOST, check, lib

    ndim = 3 if hasattr(plan, "Ny") else 2
    data, clock = read_checkpoint(path, field_names(ndim))
    data = np.ascontiguousarray(data)
    check(lib.tb_checkpoint_load(plan.ptr, data.ctypes.data_as(ctypes.c_void_p), TB_HOST,
                                 clock.ctypes.data_as(ctypes.c_void_p)), plan.ctx)
