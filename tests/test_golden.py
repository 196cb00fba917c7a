"""The oracle reproduces the committed golden fixtures (regression pin)."""
import os

import numpy as np
import pytest

from oracle.tarang_oracle import (
    RBC2D,
    RBCParams,
    backward_2d,
    forward_2d,
    padded_multiply,
    rel_l2,
    run_rbc,
)

CASES = ["rbc_rk222_32x16", "rbc_rk443_48x24", "rbc_sbdf2_32x16", "rbc_rk222_64x17"]


def test_transform_fixture(golden_dir):
    d = np.load(os.path.join(golden_dir, "transforms.npz"))
    for key in ("16x11", "24x16", "96x24"):
        Nx = int(key.split("x")[0])
        assert rel_l2(forward_2d(d[f"grid_{key}"]), d[f"coeff_{key}"]) < 1e-14
        assert rel_l2(backward_2d(d[f"bcoeff_{key}"], Nx), d[f"bgrid_{key}"]) < 1e-14
        assert rel_l2(padded_multiply(d[f"a_{key}"], d[f"b_{key}"]), d[f"prod_{key}"]) < 1e-14
        Nz = int(key.split("x")[1])
        sim = RBC2D(RBCParams(Nx=Nx, Nz=Nz))
        outs = sim.rhs(*(d[f"rhs_in{i}_{key}"] for i in range(3)))
        for i in range(3):
            assert rel_l2(outs[i], d[f"rhs_out{i}_{key}"]) < 1e-13


@pytest.mark.parametrize("name", CASES)
def test_step_fixture(golden_dir, name):
    d = np.load(os.path.join(golden_dir, f"{name}.npz"))
    p = RBCParams(Nx=int(d["Nx"]), Nz=int(d["Nz"]), Lx=4.0, Lz=1.0, Ra=float(d["Ra"]))
    sim = run_rbc(p, str(d["scheme"]), float(d["dt"]), int(d["nsteps"]), seed=42)
    for f, arr in (("b", sim.b), ("ux", sim.ux), ("uz", sim.uz)):
        assert rel_l2(arr, d[f]) < 1e-12, f


@pytest.mark.parametrize("name", ["turb_sbdf2_32", "turb_rk443_32"])
def test_turbulence_fixture(golden_dir, name):
    from oracle.tarang_oracle import run_turb, run_turb_rk, turb_initial_spec

    d = np.load(os.path.join(golden_dir, f"{name}.npz"))
    N, scheme, seed = int(d["N"]), str(d["scheme"]), int(d["seed"])
    q0 = turb_initial_spec(N, N, seed=seed)
    assert rel_l2(q0, d["q0"]) < 1e-15
    args = (q0, N, 2 * np.pi, 2 * np.pi, float(d["nu"]), float(d["dt"]), int(d["nsteps"]))
    q = run_turb(*args) if scheme == "SBDF2" else run_turb_rk(*args, scheme)
    assert rel_l2(q, d["q"]) < 1e-12
