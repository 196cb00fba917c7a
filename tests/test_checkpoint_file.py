"""The checkpoint file format on CPU: grid fields and the clock survive a
write/read round trip, and a file without the clock attributes is refused."""
import numpy as np
import pytest

from __graft_entry__ import load_package

load_package()
from tarang_b200 import checkpoint as ck  # noqa: E402


def test_round_trip_2d_and_3d(tmp_path):
    rng = np.random.default_rng(0)
    for ndim, shape in ((2, (8, 16)), (3, (6, 4, 8))):
        names = ck.field_names(ndim)
        fields = {n: rng.standard_normal(shape) for n in names}
        path = str(tmp_path / f"c{ndim}.nc")
        ck.write_checkpoint(path, fields, (1.25, 40, 0.01))
        data, clock = ck.read_checkpoint(path, names)
        assert np.array_equal(data, np.stack([fields[n] for n in names]))
        assert list(clock) == [1.25, 40.0, 0.01]


def test_iteration_beyond_int32_survives(tmp_path):
    # the reference stores the iteration as a 64-bit Int
    names = ck.field_names(2)
    fields = {n: np.zeros((2, 4)) for n in names}
    path = str(tmp_path / "big.nc")
    ck.write_checkpoint(path, fields, (3.0, 2**31 + 7, 0.5))
    _, clock = ck.read_checkpoint(path, names)
    assert int(clock[1]) == 2**31 + 7


def test_missing_clock_is_refused(tmp_path):
    from scipy.io import netcdf_file

    path = str(tmp_path / "noclock.nc")
    with netcdf_file(path, "w", version=2) as f:
        f.createDimension("z", 2)
        f.createDimension("x", 2)
        for n in ck.field_names(2):
            f.createVariable(n, "d", ("z", "x"))[...] = 0.0
    with pytest.raises(ValueError, match="clock"):
        ck.read_checkpoint(path, ck.field_names(2))
