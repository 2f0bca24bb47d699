"""CPU: the reference's NetCDF grid files (NetCDFGrid3DWriter / NetCDFGrid3DReader,
ocustorage/gridnetcdf.h:67-183), written and read here without libnetcdf.

Files written by the library are read with scipy's own NetCDF-3 implementation
(scipy.io.netcdf_file), which checks the classic format independently, and must carry the
reference writer's structure: an unlimited Time dimension and Time variable, global attributes
nx..hz, one coordinate dimension + variable per axis offset named as the reference names them
(values i * h + offset), grid variables on (Time, X, Y, Z).  Files written by scipy in that
structure are read back by the library's reader.
"""
import os

import numpy as np
import pytest
from scipy.io import netcdf_file

import opencurrent_b200 as ocu


def write_sample(path):
    nx, ny, nz = 6, 5, 4
    rng = np.random.default_rng(3)
    w = ocu.NetCDFGrid3DWriter()
    w.open(path, nx, ny, nz, 0.5, 0.25, 0.125)
    w.define_variable("temperature", ocu.NC_FLOAT, ocu.GS_CENTER_POINT)
    w.define_variable("u", ocu.NC_DOUBLE, ocu.GS_U_FACE)
    w.define_variable("w", ocu.NC_FLOAT, ocu.GS_W_FACE)
    w.define_variable("flag", ocu.NC_INT, ocu.GS_CUSTOM, 0.25, 0.5, 0.75)
    data = {
        ("temperature", 0): rng.standard_normal((nx, ny, nz)).astype(np.float32),
        ("u", 0): rng.standard_normal((nx + 1, ny, nz)),
        ("w", 0): rng.standard_normal((nx, ny, nz + 1)).astype(np.float32),
        ("flag", 0): rng.integers(-5, 5, (nx, ny, nz)).astype(np.int32),
        ("temperature", 1): rng.standard_normal((nx, ny, nz)).astype(np.float32),
        ("u", 1): rng.standard_normal((nx + 1, ny, nz)),
    }
    for (name, lvl), a in data.items():
        if lvl == 1 and name == "temperature":
            assert w.add_time_level(0.75) == 1
        w.add_data(name, a, lvl)
    w.close()
    return data


def test_written_file_is_classic_netcdf_with_the_reference_structure(tmp_path):
    path = str(tmp_path / "grids.nc")
    data = write_sample(path)
    f = netcdf_file(path, "r", mmap=False)
    try:
        assert f.dimensions["Time"] is None and f.variables["Time"].shape[0] == 2
        assert list(f.variables["Time"][:]) == [0.0, 0.75]
        assert (f.nx, f.ny, f.nz) == (6, 5, 4)
        assert np.float32(f.hx) == np.float32(0.5) and np.float32(f.hz) == np.float32(0.125)
        for name, n in [("XAxisCentered", 6), ("XAxisUFace", 7), ("YAxisCentered", 5), ("ZAxisCentered", 4),
                        ("ZAxisWFace", 5), ("XAxisOffset0.2500", 6), ("ZAxisOffset0.7500", 4)]:
            assert f.dimensions[name] == n, name
        h = {"X": 0.5, "Y": 0.25, "Z": 0.125}
        for name, off in [("XAxisCentered", 0.5), ("XAxisUFace", 0.0), ("ZAxisOffset0.7500", 0.75)]:
            n = f.dimensions[name]
            np.testing.assert_array_equal(f.variables[name][:], (np.arange(n) * np.float32(h[name[0]]) +
                                                                np.float32(off)).astype(np.float32))
        assert f.variables["u"].dimensions == ("Time", "XAxisUFace", "YAxisCentered", "ZAxisCentered")
        assert f.variables["flag"].dimensions == ("Time", "XAxisOffset0.2500", "YAxisCentered", "ZAxisOffset0.7500")
        for (name, lvl), a in data.items():
            np.testing.assert_array_equal(f.variables[name][lvl], a)
        # variables without data at a level hold the format's fill value
        assert np.all(f.variables["w"][1] == np.float32(9.96921e36))
        assert np.all(f.variables["flag"][1] == -2147483647)
    finally:
        f.close()


def test_round_trip_through_the_library_reader(tmp_path):
    path = str(tmp_path / "grids.nc")
    data = write_sample(path)
    r = ocu.NetCDFGrid3DReader()
    r.open(path)
    assert (r.nx, r.ny, r.nz, r.hx, r.hy, r.hz) == (6, 5, 4, 0.5, 0.25, 0.125)
    assert r.num_time_levels() == 2 and r.get_time(1) == 0.75
    assert r.list_variables() == ["temperature", "u", "w", "flag"]
    assert r.variable_type("u") == ocu.NC_DOUBLE and r.variable_size("u") == (7, 5, 4)
    for (name, lvl), a in data.items():
        b = r.read_variable(name, lvl)
        assert b.dtype == a.dtype
        np.testing.assert_array_equal(b, a)
    r.close()


def test_reads_a_file_written_by_another_implementation(tmp_path):
    path = str(tmp_path / "scipy.nc")
    nx, ny, nz = 4, 3, 5
    rng = np.random.default_rng(9)
    p = rng.standard_normal((3, nx, ny, nz))
    f = netcdf_file(path, "w", version=2)
    f.nx, f.ny, f.nz = np.int32(nx), np.int32(ny), np.int32(nz)
    f.hx, f.hy, f.hz = np.float32(0.1), np.float32(0.2), np.float32(0.3)
    f.createDimension("Time", None)
    t = f.createVariable("Time", "f", ("Time",))
    for name, n in [("XAxisCentered", nx), ("YAxisCentered", ny), ("ZAxisCentered", nz)]:
        f.createDimension(name, n)
        f.createVariable(name, "f", (name,))[:] = np.arange(n) + 0.5
    v = f.createVariable("pressure", "d", ("Time", "XAxisCentered", "YAxisCentered", "ZAxisCentered"))
    v[:] = p
    t[:] = [0.0, 1.0, 2.5]
    f.close()
    r = ocu.NetCDFGrid3DReader()
    r.open(path)
    assert (r.nx, r.ny, r.nz) == (nx, ny, nz) and r.num_time_levels() == 3 and r.get_time(2) == 2.5
    assert r.list_variables() == ["pressure"]
    for lvl in range(3):
        np.testing.assert_array_equal(r.read_variable("pressure", lvl), p[lvl])


def test_errors(tmp_path):
    path = str(tmp_path / "e.nc")
    w = ocu.NetCDFGrid3DWriter()
    w.open(path, 4, 4, 4)
    w.define_variable("a", ocu.NC_FLOAT)
    with pytest.raises(ocu.OcuError):
        w.define_variable("a", ocu.NC_FLOAT)                        # previously defined
    with pytest.raises(ocu.OcuError):
        w.define_variable("b", 2)                                   # NC_CHAR: not a grid type
    with pytest.raises(ocu.OcuError):
        w.add_data("a", np.zeros((4, 4, 5), np.float32))            # dimension mismatch
    with pytest.raises(ocu.OcuError):
        w.add_data("a", np.zeros((4, 4, 4), np.float64))            # type mismatch
    with pytest.raises(ocu.OcuError):
        w.add_data("c", np.zeros((4, 4, 4), np.float32))            # not defined
    with pytest.raises(ocu.OcuError):
        w.add_data("a", np.zeros((4, 4, 4), np.float32), 3)         # level not added
    w.close()
    with open(str(tmp_path / "junk.nc"), "wb") as f:
        f.write(b"not a netcdf file")
    with pytest.raises(ocu.OcuError):
        ocu.NetCDFGrid3DReader().open(str(tmp_path / "junk.nc"))
