"""The result file of the reference's driver (Common/IO.h:136-276, :340-377) through
adi_nc_write_header / adi_nc_write_layer, read back with an independent NetCDF
reader (scipy.io.netcdf_file): dimensions, variables and their dimensions, every
attribute, the axes (the reference's float arithmetic), the time axis, the sampled
depths, written layers and fill values elsewhere.  Host code only (runs without a GPU).
"""
import numpy as np
import pytest

FILL = 9.9692099683868690e+36


def _axes(pmin, pmax, n):
    out = []
    for a in range(3):
        dd = np.float32(np.float32(pmax[a]) - np.float32(pmin[a])) / np.float32(n[a])
        out.append(np.array([np.float32(pmin[a]) + np.float32(dd * np.float32(i)) for i in range(n[a])], np.float32))
    return out


@pytest.mark.parametrize("degree_units", [False, True])
def test_result_file_matches_the_reference_layout(adi_lib, tmp_path, degree_units):
    from scipy.io import netcdf_file
    from adi_b200 import ncout
    path = str(tmp_path / "case_res.nc")
    pmin, pmax = (0.0, -1.5, 0.25), (2.0, 1.5, 1.0)
    dims = (7, 5, 4)
    rng = np.random.default_rng(3)
    depth = rng.uniform(0.0, 10.0, size=(13, 9)).astype(np.float32)
    out_vars = ["u", "v", "w", "T", "d"]
    ncout.write_header(path, pmin, pmax, 0.25, 1.0, dims, out_vars, depth=depth, xy_degree_units=degree_units)
    vel = [rng.standard_normal(dims + (3,)).astype(np.float32) for _ in range(2)]
    T = [rng.standard_normal(dims) for _ in range(2)]
    ncout.write_layer(path, vel[0], T[0], 0, out_vars)
    ncout.write_layer(path, vel[1], T[1], 2, out_vars)
    with netcdf_file(path, "r", mmap=False) as f:
        assert f.version_byte == 2
        assert f.dimensions == {"x": 7, "y": 5, "z": 4, "t": None}
        assert list(f.variables) == ["x", "y", "z", "time", "u", "v", "w", "T", "d"]
        for name, axis in zip("xyz", _axes(pmin, pmax, dims)):
            np.testing.assert_array_equal(f.variables[name][:], axis)
        x, y, z, t = (f.variables[k] for k in ("x", "y", "z", "time"))
        np.testing.assert_array_equal(x.actual_range, np.float32([0.0, 2.0]))
        assert x.long_name == b"x coord" and y.long_name == b"y coord" and z.long_name == b"z coord"
        assert x.units == (b"degree_north" if degree_units else b"metres")
        assert y.units == (b"degree_east" if degree_units else b"metres")
        assert z.units == b"metres" and t.units == b"s" and t.long_name == b"time"
        np.testing.assert_array_equal(t.actual_range, [0.0, 1.0])
        np.testing.assert_array_equal(t[:], [0.0, 0.25, 0.5, 0.75])   # time / timestep records
        for k, long_name, units in (("u", b"x-velocity", b"m/s"), ("v", b"y-velocity", b"m/s"),
                                    ("w", b"z-velocity", b"m/s"), ("T", b"temperature", b"tmp")):
            v = f.variables[k]
            assert v.dimensions == ("t", "x", "y", "z") and v.typecode() == "d"
            assert v.units == units and v.long_name == long_name and v.var_desc == k.encode()
            np.testing.assert_array_equal(v.actual_range, [-1.0, 1.0])
            np.testing.assert_array_equal(v.valid_range, [-1.0, 1.0])
            assert v.missing_value == np.float32(99999.0)
            comp = "uvw".find(k)
            for rec, src in ((0, 0), (2, 1)):
                want = T[src] if k == "T" else vel[src][..., comp].astype(np.float64)
                np.testing.assert_array_equal(v[rec], want)
            assert np.all(v[1] == FILL) and np.all(v[3] == FILL)
        d = f.variables["d"]
        assert d.dimensions == ("x", "y") and d.typecode() == "f" and d.units == b"m"
        want = np.array([[depth[i * 13 // 7, j * 9 // 5] for j in range(5)] for i in range(7)], np.float32)
        np.testing.assert_array_equal(d[:], want)
        assert f.Conventions == b"COARDS" and f.title == b"cmc-fluid-solver results"
        assert f.history == b"created by using cmc-fluid-solver"
        assert f.description == b"Test data" and f.platform == b"Model"


def test_layers_past_the_time_axis_and_a_subset_of_variables(adi_lib, tmp_path):
    from scipy.io import netcdf_file
    from adi_b200 import ncout
    path = str(tmp_path / "sub_res.nc")
    dims = (3, 4, 5)
    ncout.write_header(path, (0, 0, 0), (1, 1, 1), 0.5, 1.0, dims, ["u", "T"])
    vel = np.arange(np.prod(dims) * 3, dtype=np.float64).reshape(dims + (3,))
    T = -np.arange(np.prod(dims), dtype=np.float64).reshape(dims)
    ncout.write_layer(path, vel, T, 3, ["u", "T"])   # past the two records of the time axis
    with netcdf_file(path, "r", mmap=False) as f:
        assert list(f.variables) == ["x", "y", "z", "time", "u", "T"]
        assert f.variables["u"].shape == (4, 3, 4, 5)
        np.testing.assert_array_equal(f.variables["u"][3], vel[..., 0])
        np.testing.assert_array_equal(f.variables["T"][3], T)
        np.testing.assert_array_equal(f.variables["time"][:2], [0.0, 0.5])
        assert np.all(f.variables["time"][2:] == FILL)
    with pytest.raises(Exception):
        ncout.write_layer(path, vel[:2], T[:2], 0, ["u", "T"])   # dims differ from the file's


def test_header_arguments_the_format_cannot_hold_are_rejected(adi_lib, tmp_path):
    from adi_b200 import _abi, ncout
    path = tmp_path / "bad_res.nc"
    bad = [
        dict(timestep=0.1, time=-1.0, outdims=(2, 2, 2)),            # negative time
        dict(timestep=1e-9, time=1.0, outdims=(2, 2, 2)),            # 1e9 records
        dict(timestep=0.1, time=1.0, outdims=(1024, 1024, 1024)),    # 8 GiB per record of u
        dict(timestep=0.1, time=1.0, outdims=(0, 2, 2)),
    ]
    for kw in bad:
        with pytest.raises(_abi.AdiError):
            ncout.write_header(str(path), (0, 0, 0), (1, 1, 1), kw["timestep"], kw["time"], kw["outdims"], ["u"])
        assert not path.exists()


@pytest.mark.gpu
def test_driver_output_path_getlayer_to_result_file(adi_lib, tmp_path):
    """The reference driver's output path (FluidSolver3D.cpp:206, 248-258): header,
    then every out_time_steps-th step GetLayer on the output grid and one layer of
    the result file; the file holds exactly what GetLayer returned."""
    from scipy.io import netcdf_file
    from adi_b200 import geometry as G, ncout
    d = G.spheres_channel(dims=(40, 24, 28), n_spheres=3, rmin=3.0, rmax=5.0, seed=9)
    s = adi_lib.AdiSolver3D(d, Re=150.0, Pr=0.72, lam=1.4)
    s.CreateSegments()
    out_dims, out_vars, dt = (20, 12, 14), ["u", "v", "w", "T"], 5e-4
    path = str(tmp_path / "run_res.nc")
    ncout.write_header(path, (0.0, 0.0, 0.0), (1.0, 0.6, 0.7), 2 * dt, 6 * dt, out_dims, out_vars)
    layers = []
    for i in range(6):
        assert s.step(dt, 4, 2, i % 10 == 0) == 0
        if i % 2 == 0:
            v, T = s.GetLayer(*out_dims)
            ncout.write_layer(path, v, T, len(layers), out_vars)
            layers.append((v.copy(), T.copy()))
    with netcdf_file(path, "r", mmap=False) as f:
        for r, (v, T) in enumerate(layers):
            for c, k in enumerate("uvw"):
                np.testing.assert_array_equal(f.variables[k][r], v[..., c].astype(np.float64))
            np.testing.assert_array_equal(f.variables["T"][r], T)
