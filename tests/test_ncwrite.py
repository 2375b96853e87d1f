"""The core's netCDF-3 (CDF-2) writer, read back with scipy's independent
netCDF reader: dimensions, attributes, fixed and record variables, fill values
of unwritten slabs and the record count."""
import os
import shutil
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "native", "ncwrite_check.cpp")
INC = os.path.join(os.path.dirname(HERE), "sfincs_b200", "csrc", "host")


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_writer_round_trips_through_an_independent_reader(tmp_path):
    from scipy.io import netcdf_file

    exe = str(tmp_path / "ncwrite_check")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", INC, SRC, "-o", exe], check=True)
    path = str(tmp_path / "check.nc")
    subprocess.run([exe, path], check=True)
    with open(path, "rb") as f:
        assert f.read(4) == b"CDF\x02"
    f = netcdf_file(path, "r", mmap=False)
    assert f.title == b"writer check"
    assert f.dimensions["n"] == 3 and f.dimensions["m"] == 5 and f.dimensions["time"] is None
    x = f.variables["x"]
    assert x.units == b"m" and x._FillValue == np.float32(-99999.0)
    assert np.array_equal(x[:], (0.5 * np.arange(15, dtype=np.float32)).reshape(3, 5))
    assert np.array_equal(f.variables["msk"][:], (np.arange(15) % 3).reshape(3, 5))
    assert list(f.variables["msk"].flag_values) == [0, 1, 2]
    xd = f.variables["xd"][:]
    assert xd.dtype.kind == "f" and xd.dtype.itemsize == 8 and np.array_equal(xd, [1.0, 2.5, -3.25, 1e300, -0.0])
    assert b"".join(f.variables["name"][0]) == b"abc    "
    zmax = f.variables["zsmax"][:]
    assert np.all(zmax[0] == np.float32(-99999.0))  # prefilled
    assert np.array_equal(zmax[1].ravel(), 100.0 + np.arange(15))
    assert int(f.variables["scalar"].getValue()) == 42
    assert np.array_equal(f.variables["time"][:], [0.0, 600.0, 1200.0])
    zs = f.variables["zs"][:]
    assert zs.shape == (3, 3, 5) and zs[2, 2, 4] == 214.0
    assert np.array_equal(f.variables["qd"][:][:, 0], [0.125, 1.125, 2.125])
    f.close()
