"""Snapshot files in the reference's netCDF layout: the writer's files are
read back bit-exactly by this module's reader and by an independent netCDF
reader (scipy.io.netcdf_file), with the reference's names, dimensions and
attributes (nf90_operators_module.f:979-1353)."""
import numpy as np
import pytest

from dim2d_finite_volume_b200 import snapshot as S


def _state(nx=13, ny=9, seed=1):
    rng = np.random.default_rng(seed)
    return (rng.standard_normal((4, ny, nx)), np.linspace(-0.6, 0.6, nx),
            np.linspace(-0.5, 0.5, ny), 0.125)


def test_round_trip_bit_exact(tmp_path):
    q, x, y, t = _state()
    p = tmp_path / "snap.nc"
    S.write_netcdf(p, q, x, y, t, {"title": "t", "dt": 1e-3, "nsteps": 7})
    q2, x2, y2, t2, att = S.read_snapshot(p)
    assert np.array_equal(q2, q) and np.array_equal(x2, x) and np.array_equal(y2, y)
    assert t2 == t
    assert att["title"] == "t" and att["dt"] == 1e-3 and att["nsteps"] == 7


def test_independent_reader_sees_the_reference_layout(tmp_path):
    scipy_io = pytest.importorskip("scipy.io")
    q, x, y, t = _state(nx=10, ny=7)
    p = tmp_path / "snap.nc"
    S.write_netcdf(p, q, x, y, t, {"title": "run", "x_min": -0.6})
    f = scipy_io.netcdf_file(str(p), "r", mmap=False)
    try:
        assert f.dimensions["time"] == 1 and f.dimensions["x"] == 10 and f.dimensions["y"] == 7
        for k, (name, long_name, units) in enumerate(S.VARIABLES):
            v = f.variables[name]
            assert v.dimensions == ("y", "x", "time")
            assert np.array_equal(v.data[:, :, 0], q[k])
            assert v.long_name.decode() == long_name and v.units.decode() == units
        assert np.array_equal(f.variables["x"].data, x)
        assert f.variables["x"].axis.decode() == "X"
        assert f.variables["time"].data[0] == t
        assert f.title.decode() == "run" and f.x_min == -0.6
    finally:
        f.close()


def test_reader_reads_independent_writer(tmp_path):
    scipy_io = pytest.importorskip("scipy.io")
    q, x, y, t = _state(nx=6, ny=5, seed=3)
    p = tmp_path / "other.nc"
    f = scipy_io.netcdf_file(str(p), "w", version=2)
    f.createDimension("time", 1)
    f.createDimension("x", 6)
    f.createDimension("y", 5)
    for name, data, dims in (("time", np.array([t]), ("time",)), ("x", x, ("x",)),
                             ("y", y, ("y",))):
        f.createVariable(name, "d", dims)[:] = data
    for k, (name, _, _) in enumerate(S.VARIABLES):
        f.createVariable(name, "d", ("y", "x", "time"))[:] = q[k][:, :, None]
    f.title = "written elsewhere"
    f.close()
    q2, x2, y2, t2, att = S.read_snapshot(p)
    assert np.array_equal(q2, q) and np.array_equal(x2, x) and t2 == t
    assert att["title"] == "written elsewhere"
