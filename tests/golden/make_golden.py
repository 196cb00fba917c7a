"""Generate the golden fixtures used by the parity tests.

Run from the repository root:  python tests/golden/make_golden.py [--large]

The fixtures are outputs of the CPU oracle (oracle/tarang_oracle.py) on seeded
inputs at sizes the oracle finishes in seconds.  ``--large`` (about ten
minutes on 8 host threads) adds the full-size 2D benchmark runs -- 1024x256,
Ra 1e8, dt 0.01, seed 42, 100 steps of RK443 and of SBDF2 -- and a 3D run of
the 3D benchmark's parameters (Ra 1e7, dt 5e-3, RK222) on a 64x64x32 grid for
20 steps.  The oracle's state is bitwise the same at any thread count.  The oracle itself is pinned to
the reference's analytic known-answer tests (tests/test_oracle_known_answers.py);
these files freeze its outputs so that both the oracle and the CUDA library are
checked against the same numbers on every run.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.tarang_oracle import (  # noqa: E402
    RBC2D,
    RBC3Params,
    RBCParams,
    backward_2d,
    forward_2d,
    padded_multiply,
    rbc_initial_b,
    run_rbc,
    run_rbc3,
    run_turb,
    run_turb_rk,
    set_threads,
    turb_initial_spec,
)

CASES = [
    # name, Nx, Nz, Ra, scheme, dt, nsteps
    ("rbc_rk222_32x16", 32, 16, 2e6, "RK222", 0.125, 6),
    ("rbc_rk443_48x24", 48, 24, 1e8, "RK443", 0.01, 6),
    ("rbc_sbdf2_32x16", 32, 16, 1e8, "SBDF2", 0.01, 6),
    ("rbc_rk222_64x17", 64, 17, 1e6, "RK222", 0.05, 5),
]

LARGE_CASES = [
    # the 2D benchmark grid: ChannelDomain(1024, 256), Lx 4, Lz 1, Ra 1e8, Pr 1
    ("rbc_c2_rk443_1024x256", 1024, 256, 1e8, "RK443", 0.01, 100),
    ("rbc_c2_sbdf2_1024x256", 1024, 256, 1e8, "SBDF2", 0.01, 100),
]

LARGE_3D_CASES = [
    # name, Nx, Ny, Nz, Ra, scheme, dt, nsteps (Lx = Ly = 4, Lz = 1, Pr 1, seed 42)
    ("rbc3_rk222_64x64x32", 64, 64, 32, 1e7, "RK222", 5e-3, 20),
]

TURB_CASES = [
    # name, N, scheme, nu, dt, nsteps, seed (doubly periodic vorticity, 2 pi box)
    ("turb_sbdf2_32", 32, "SBDF2", 1e-3, 2e-3, 6, 21),
    ("turb_rk443_32", 32, "RK443", 1e-3, 2e-3, 6, 21),
]


def make_turb_fixture(path: str, N, scheme, nu, dt, nsteps, seed) -> None:
    q0 = turb_initial_spec(N, N, seed=seed)
    if scheme == "SBDF2":
        q = run_turb(q0, N, 2 * np.pi, 2 * np.pi, nu, dt, nsteps)
    else:
        q = run_turb_rk(q0, N, 2 * np.pi, 2 * np.pi, nu, dt, nsteps, scheme)
    np.savez_compressed(path, N=N, scheme=scheme, nu=nu, dt=dt, nsteps=nsteps, seed=seed, q0=q0, q=q)


def make_transform_fixture(path: str) -> None:
    rng = np.random.default_rng(2024)
    out = {}
    for Nx, Nz in ((16, 11), (24, 16), (96, 24)):
        g = rng.standard_normal((Nz, Nx))
        a = rng.standard_normal((Nz, Nx))
        b = rng.standard_normal((Nz, Nx))
        c = forward_2d(rng.standard_normal((Nz, Nx)))
        key = f"{Nx}x{Nz}"
        out[f"grid_{key}"] = g
        out[f"coeff_{key}"] = forward_2d(g)
        out[f"bcoeff_{key}"] = c
        out[f"bgrid_{key}"] = backward_2d(c, Nx)
        out[f"a_{key}"] = a
        out[f"b_{key}"] = b
        out[f"prod_{key}"] = padded_multiply(a, b)
        p = RBCParams(Nx=Nx, Nz=Nz)
        sim = RBC2D(p)
        ins = [forward_2d(rng.standard_normal((Nz, Nx))) for _ in range(3)]
        outs = sim.rhs(*ins)
        for i in range(3):
            out[f"rhs_in{i}_{key}"] = ins[i]
            out[f"rhs_out{i}_{key}"] = outs[i]
    np.savez_compressed(path, **out)


def make_step_fixture(path: str, Nx, Nz, Ra, scheme, dt, nsteps, with_b0: bool = True) -> None:
    """with_b0=False leaves out the initial field (the seeded noise of seed 42,
    which the tests rebuild with the oracle's rbc_initial_b) to keep the
    full-size files small."""
    p = RBCParams(Nx=Nx, Nz=Nz, Lx=4.0, Lz=1.0, Ra=Ra, Pr=1.0)
    sim = run_rbc(p, scheme, dt, nsteps, seed=42)
    extra = {"b0": forward_2d(rbc_initial_b(p, 42))} if with_b0 else {}
    np.savez_compressed(
        path,
        Nx=Nx, Nz=Nz, Ra=Ra, dt=dt, nsteps=nsteps, scheme=scheme,
        b=sim.b, ux=sim.ux, uz=sim.uz, p=sim.pr, tau=sim.tau, **extra,
    )


def make_step3_fixture(path: str, Nx, Ny, Nz, Ra, scheme, dt, nsteps) -> None:
    p = RBC3Params(Nx=Nx, Ny=Ny, Nz=Nz, Ra=Ra)
    sim = run_rbc3(p, scheme, dt, nsteps, seed=42)
    np.savez_compressed(
        path,
        Nx=Nx, Ny=Ny, Nz=Nz, Ra=Ra, dt=dt, nsteps=nsteps, scheme=scheme,
        b=sim.b, ux=sim.ux, uy=sim.uy, uz=sim.uz,
    )


def main() -> None:
    if "--large" in sys.argv:
        set_threads(os.cpu_count() or 1)
        for name, Nx, Nz, Ra, scheme, dt, ns in LARGE_CASES:
            make_step_fixture(os.path.join(HERE, f"{name}.npz"), Nx, Nz, Ra, scheme, dt, ns, with_b0=False)
            print("wrote", name, flush=True)
        for name, *case in LARGE_3D_CASES:
            make_step3_fixture(os.path.join(HERE, f"{name}.npz"), *case)
            print("wrote", name, flush=True)
        return
    make_transform_fixture(os.path.join(HERE, "transforms.npz"))
    for name, Nx, Nz, Ra, scheme, dt, ns in CASES:
        make_step_fixture(os.path.join(HERE, f"{name}.npz"), Nx, Nz, Ra, scheme, dt, ns)
    for name, *case in TURB_CASES:
        make_turb_fixture(os.path.join(HERE, f"{name}.npz"), *case)
    print("wrote fixtures to", HERE)


if __name__ == "__main__":
    main()
