"""The oracle gives the same state whatever its host thread count (the CPU
baseline runs it on all host cores)."""
import numpy as np
import pytest

import oracle.tarang_oracle as O


@pytest.fixture
def restore_threads():
    yield
    O.set_threads(1)


@pytest.mark.parametrize("scheme", ["RK443", "SBDF2"])
def test_threads_2d_bitwise(restore_threads, scheme):
    p = O.RBCParams(Nx=32, Nz=16, Lx=4.0, Lz=1.0, Ra=1e5)
    out = {}
    for th in (1, 4):
        O.set_threads(th)
        sim = O.run_rbc(p, scheme, 0.01, 3, seed=42)
        out[th] = sim.state_dict()
    for k in out[1]:
        assert np.array_equal(out[1][k], out[4][k]), k


def test_threads_3d_bitwise(restore_threads):
    p = O.RBC3Params(Nx=8, Ny=8, Nz=8, Ra=1e5)
    out = {}
    for th in (1, 3):
        O.set_threads(th)
        sim = O.run_rbc3(p, "RK222", 0.005, 2, seed=42)
        out[th] = (sim.b.copy(), sim.ux.copy(), sim.uy.copy(), sim.uz.copy())
    for a, b in zip(out[1], out[3]):
        assert np.array_equal(a, b)
