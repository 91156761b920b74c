"""NetCDF output of a block (snapy_linfel_b200.netcdf) read back with an
independent NetCDF-3 reader (scipy.io.netcdf_file): file name, dimensions,
coordinate variables and their attributes, the variables' layout
[time, x1, x3, x2] and values, the metadata table's units and long names
(src/output/netcdf.cpp, src/output/output_utils.cpp:28-70)."""
import os

import numpy as np
import pytest

from snapy_linfel_b200 import netcdf
from snapy_linfel_b200.config import make_config

scipy_io = pytest.importorskip("scipy.io")


def _arrays(c, seed=3):
    rng = np.random.default_rng(seed)
    w = rng.random(c.shape) + 0.5
    u = rng.random(c.shape) + 0.5
    s = rng.random((2,) + c.shape[1:])
    return w, u, s


def test_prim_cons_and_scalars_round_trip(tmp_path):
    c = make_config(nx1=6, nx2=5, nx3=4, x1=(0.0, 600.0), x2=(0.0, 1000.0), x3=(0.0, 800.0))
    w, u, s = _arrays(c)
    path = netcdf.write_block(c, w, u, str(tmp_path), "bubble", 7, 12.5,
                              variables=("prim", "cons"), rank=1, block_loc=(0, 1, 0),
                              blocks=(1, 2, 1), scalars=s)
    assert os.path.basename(path) == "bubble.block1.out1.00007.nc"
    with scipy_io.netcdf_file(path, "r", mmap=False) as f:
        assert f.dimensions["time"] is None
        assert (f.dimensions["x1"], f.dimensions["x1f"]) == (6, 7)
        assert (f.dimensions["x2"], f.dimensions["x3"]) == (5, 4)
        assert int(f.NumFilesInSet) == 2
        assert float(f.variables["time"][0]) == 12.5
        x1 = f.variables["x1"]
        assert x1.axis == b"Z" and x1.units == b"m"
        np.testing.assert_allclose(x1[:], 50.0 + 100.0 * np.arange(6), rtol=1e-6)
        np.testing.assert_allclose(f.variables["x1f"][:], 100.0 * np.arange(7), rtol=1e-6)
        # the block's position along x2 (second of two blocks)
        assert list(f.variables["x2"].domain_decomposition) == [1, 10, 6, 10]
        assert list(f.variables["x2f"].domain_decomposition) == [0, 10, 5, 10]
        rho = f.variables["rho"]
        assert rho.dimensions == ("time", "x1", "x3", "x2")
        assert rho.units == b"kg/m^3" and rho.long_name == b"density"
        assert f.variables["vel1"].long_name == b"vertical velocity"
        it = c.interior()
        for name, arr, v in (("rho", w, 0), ("press", w, 4), ("vel2", w, 2), ("dens", u, 0),
                             ("Etot", u, 4), ("mom3", u, 3), ("s1", s, 0), ("s2", s, 1)):
            want = np.transpose(arr[v][it], (2, 0, 1)).astype(np.float32)
            np.testing.assert_array_equal(f.variables[name][0], want, err_msg=name)


def test_two_dimensional_block_and_single_components(tmp_path):
    c = make_config(nx1=8, nx2=6, x1=(0.0, 6400.0), x2=(-25.6e3, 25.6e3))
    w, u, _ = _arrays(c, seed=5)
    path = netcdf.write_block(c, w, None, str(tmp_path), "straka", 0, 0.0, variables=("v1",))
    with scipy_io.netcdf_file(path, "r", mmap=False) as f:
        assert "x3f" not in f.dimensions and f.dimensions["x3"] == 1
        assert set(f.variables) >= {"time", "x1", "x1f", "x2", "x2f", "x3", "vel1"}
        assert "rho" not in f.variables
        assert f.variables["vel1"].shape == (1, 8, 1, 6)
    with pytest.raises(ValueError):
        netcdf.write_block(c, w, None, str(tmp_path), "straka", 1, 0.0, variables=("cons",))
    with pytest.raises(ValueError):
        netcdf.write_block(c, w, u, str(tmp_path), "straka", 1, 0.0, variables=("theta",))
