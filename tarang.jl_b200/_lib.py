"""ctypes binding of libtarang_b200.so (the C ABI declared in include/tarang_b200.h).

The shared library is built in-tree by ``tarang.jl_b200/csrc/Makefile``.  There is
no CPU fallback: if the library is missing or cannot be loaded, importing this
module raises.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, Structure, c_char_p, c_double, c_float, c_int, c_longlong, c_size_t, c_void_p

HERE = os.path.dirname(os.path.abspath(__file__))
# TARANG_B200_LIB selects another build of the same ABI (the phase-clock build
# of solve_clocks.py); the default is the product library beside this file
LIB_PATH = os.environ.get("TARANG_B200_LIB") or os.path.join(HERE, "libtarang_b200.so")

TB_OK, TB_EINVAL, TB_ENOMEM, TB_ESINGULAR, TB_ETIMEOUT, TB_ECUDA, TB_ENOTSUPPORTED, TB_EBUDGET, TB_ESTATE = range(9)
TB_HOST, TB_DEVICE = 0, 1
TB_KEEP_HISTORY = 0x10
TB_NO_WAIT = 0x20
TB_RK222, TB_RK443, TB_SBDF1, TB_SBDF2 = 0, 1, 2, 3
TB_PROGRAM_RBC = 0
TB_PROGRAM_TURB2D = 1
TB_REQ_QUEUED, TB_REQ_RUNNING, TB_REQ_DONE, TB_REQ_FAILED = 0, 1, 2, 3
TB_PREC_F64, TB_PREC_MIXED = 0, 1
TB_FIELD_B, TB_FIELD_UX, TB_FIELD_UZ, TB_FIELD_P, TB_FIELD_TAU, TB_FIELD_UY = range(6)


class tb_problem_desc(Structure):
    _fields_ = [
        ("ndim", c_int),
        ("Nx", c_int),
        ("Ny", c_int),
        ("Nz", c_int),
        ("Lx", c_double),
        ("Ly", c_double),
        ("Lz", c_double),
        ("dealias", c_double),
        ("precision", c_int),
        ("timestepper", c_int),
        ("program", c_int),
        ("kappa", c_double),
        ("nu", c_double),
        ("b_bottom", c_double),
        ("b_top", c_double),
    ]


class tb_request(Structure):
    _fields_ = [("desc", tb_problem_desc), ("dt", c_double), ("nsteps", c_int), ("init_grid", c_void_p)]


class tb_server_stats(Structure):
    _fields_ = [
        ("submitted", c_longlong), ("completed", c_longlong), ("failed", c_longlong), ("running", c_longlong),
        ("queued", c_longlong), ("elapsed_ms", c_double), ("solves_per_s", c_double), ("steps_per_s", c_double),
        ("p50_ms", c_double), ("p99_ms", c_double), ("mean_wait_ms", c_double), ("peak_bytes", c_size_t),
        ("budget_bytes", c_size_t), ("peak_running", c_int), ("mean_setup_ms", c_double),
        ("peak_cohort", c_int), ("cohort_requests", c_longlong),
    ]


class TarangError(RuntimeError):
    """Raised when a library call returns a non-OK tb_status."""

    def __init__(self, status: int, message: str):
        super().__init__(f"[tb_status {status}] {message}")
        self.status = status


# name -> (restype, argtypes); every symbol include/tarang_b200.h declares.
SIGNATURES = {
    "tb_context_create": (c_int, [c_int, POINTER(c_void_p)]),
    "tb_context_destroy": (c_int, [c_void_p]),
    "tb_last_error": (c_char_p, [c_void_p]),
    "tb_status_string": (c_char_p, [c_int]),
    "tb_version": (c_int, []),
    "tb_plan_create": (c_int, [c_void_p, POINTER(tb_problem_desc), POINTER(c_void_p)]),
    "tb_plan_destroy": (c_int, [c_void_p]),
    "tb_set_state": (c_int, [c_void_p, c_int, c_void_p, c_int]),
    "tb_get_state": (c_int, [c_void_p, c_int, c_void_p, c_int]),
    "tb_set_states": (c_int, [c_void_p, c_int, c_void_p, c_void_p, c_int]),
    "tb_periodic_create": (c_int, [c_void_p, c_int, c_int, POINTER(c_void_p)]),
    "tb_periodic_destroy": (c_int, [c_void_p]),
    "tb_periodic_forward": (c_int, [c_void_p, c_void_p, c_void_p, c_int]),
    "tb_periodic_backward": (c_int, [c_void_p, c_void_p, c_void_p, c_int]),
    "tb_turb_set_vorticity": (c_int, [c_void_p, c_void_p]),
    "tb_get_states": (c_int, [c_void_p, c_int, c_void_p, c_void_p, c_int]),
    "tb_step": (c_int, [c_void_p, c_double, c_int]),
    "tb_sim_time": (c_int, [c_void_p, POINTER(c_double), POINTER(c_longlong)]),
    "tb_synchronize": (c_int, [c_void_p]),
    "tb_last_step_ms": (c_int, [c_void_p, POINTER(c_float)]),
    "tb_set_profiling": (c_int, [c_void_p, c_int]),
    "tb_profile_count": (c_int, [c_void_p, POINTER(c_int)]),
    "tb_profile_entry": (c_int, [c_void_p, c_int, c_char_p, c_int, POINTER(c_double), POINTER(c_longlong)]),
    "tb_profile_reset": (c_int, [c_void_p]),
    "tb_kernels_per_step": (c_int, [c_void_p, POINTER(c_int)]),
    "tb_plan_set_variant": (c_int, [c_void_p, c_int, c_int]),
    "tb_set_wall_values": (c_int, [c_void_p, c_int, c_void_p, c_void_p, c_int]),
    "tb_checkpoint_stage": (c_int, [c_void_p, c_void_p, c_size_t, c_void_p]),
    "tb_checkpoint_wait": (c_int, [c_void_p]),
    "tb_checkpoint_load": (c_int, [c_void_p, c_void_p, c_int, c_void_p]),
    "tb_plan_get_variant": (c_int, [c_void_p, POINTER(c_int), POINTER(c_int)]),
    "tb_plan_set_gemm_path": (c_int, [c_void_p, c_int]),
    "tb_plan_get_gemm_path": (c_int, [c_void_p, POINTER(c_int)]),
    "tb_plan_tune": (c_int, [c_void_p, c_double, c_int, POINTER(c_int), POINTER(c_int)]),
    "tb_tau_layout_query": (c_int, [c_int, c_double, c_double, c_int, POINTER(c_int)]),
    "tb_transform_forward": (c_int, [c_void_p, c_void_p, c_void_p, c_int]),
    "tb_transform_backward": (c_int, [c_void_p, c_void_p, c_void_p, c_int]),
    "tb_dealiased_multiply": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "tb_dealiased_multiply_noalloc": (c_int, [c_int, c_int, c_int, c_void_p, c_void_p, c_void_p]),
    "tb_rhs_advection": (c_int, [c_void_p, c_void_p, c_void_p]),
    "tb_batched_lu_factor": (c_int, [c_void_p, c_int, c_int, c_void_p, c_void_p, POINTER(c_int)]),
    "tb_batched_lu_solve": (c_int, [c_void_p, c_int, c_int, c_void_p, c_void_p, c_void_p]),
    "tb_step_async": (c_int, [c_void_p, c_double, c_int, c_int]),
    "tb_plan_query": (c_int, [c_void_p, POINTER(c_int)]),
    "tb_plan_wait": (c_int, [c_void_p]),
    "tb_plan_device_bytes": (c_int, [c_void_p, POINTER(c_size_t)]),
    "tb_ensemble_create": (c_int, [c_void_p, c_int, c_void_p, POINTER(c_void_p)]),
    "tb_ensemble_destroy": (c_int, [c_void_p]),
    "tb_ensemble_tune": (c_int, [c_void_p, c_void_p, c_int, POINTER(c_int), POINTER(c_int)]),
    "tb_ensemble_set_config": (c_int, [c_void_p, c_int, c_int]),
    "tb_ensemble_config": (c_int, [c_void_p, POINTER(c_int), POINTER(c_int)]),
    "tb_ensemble_set_form": (c_int, [c_void_p, c_int]),
    "tb_ensemble_get_form": (c_int, [c_void_p, POINTER(c_int), POINTER(c_int)]),
    "tb_ensemble_run": (c_int, [c_void_p, c_void_p, c_int, c_void_p, POINTER(c_float)]),
    "tb_turb_create": (c_int, [c_void_p, POINTER(tb_problem_desc), c_void_p, POINTER(c_void_p)]),
    "tb_turb_destroy": (c_int, [c_void_p]),
    "tb_turb_step": (c_int, [c_void_p, c_double, c_int]),
    "tb_turb_get_vorticity": (c_int, [c_void_p, c_void_p]),
    "tb_server_create": (c_int, [c_void_p, c_size_t, c_int, c_int, POINTER(c_void_p)]),
    "tb_server_submit": (c_int, [c_void_p, POINTER(tb_request), POINTER(c_longlong)]),
    "tb_server_set_cohort": (c_int, [c_void_p, c_int]),
    "tb_server_poll": (c_int, [c_void_p, c_longlong, POINTER(c_int), POINTER(c_double)]),
    "tb_server_result": (c_int, [c_void_p, c_longlong, c_int, c_void_p, POINTER(c_size_t)]),
    "tb_server_wait_all": (c_int, [c_void_p]),
    "tb_server_get_stats": (c_int, [c_void_p, POINTER(tb_server_stats)]),
    "tb_server_destroy": (c_int, [c_void_p]),
}


def load(path: str = LIB_PATH) -> ctypes.CDLL:
    if not os.path.exists(path):
        raise ImportError(
            f"{path} is missing: build it with `make -C tarang.jl_b200/csrc` "
            "(there is no CPU fallback for the B200 path)"
        )
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = load()


def check(status: int, ctx=None) -> None:
    if status != TB_OK:
        msg = lib.tb_last_error(ctx)
        text = msg.decode() if msg else lib.tb_status_string(status).decode()
        raise TarangError(status, text)
