"""tarang_b200: sm_100a implementation of Tarang.jl's IMEX timestep hot path.

The numerical work runs in libtarang_b200.so (CUDA, C ABI in
include/tarang_b200.h); this package is the thin host layer that mirrors the
reference's user API.  Import it with ``load_package()`` from the repository
root helper or by path: the directory name contains a dot, so it is loaded
under the module name ``tarang_b200``.
"""
from ._lib import TarangError, lib  # noqa: F401  (fails loudly if the .so is missing)
from .api import (  # noqa: F401
    CPU,
    GPU,
    IVP,
    RK222,
    RK443,
    SBDF1,
    SBDF2,
    DiagonalIMEX_RK222,
    DiagonalIMEX_RK443,
    DiagonalIMEX_SBDF2,
    PeriodicDomain,
    PeriodicTransform,
    ChannelDomain,
    ChannelDomain3D,
    ChebyshevT,
    Domain,
    Ensemble,
    InitialValueSolver,
    Plan,
    Plan3D,
    Server,
    Turb2D,
    rbc_desc,
    rbc3_desc,
    turb_desc,
    RealFourier,
    ScalarField,
    VectorField,
    add_bc,
    add_equation,
    add_parameters,
    run,
    step,
    unit_vector_fields,
)

__version__ = "0.1.0"
