"""Output path on the CPU: the oracle's restatement of the lat-lon
interpolation and of the zonal / meridional velocity against the reference's
own outputs (tests/golden/make_golden_output.py), the drivers' output-grid
rule through the C ABI, and the netCDF classic writer read back by an
independent reader (scipy.io.netcdf_file).

Tolerances: the oracle matches the reference to <= 1e-14 relative (same
formulas, same libm); the output grid exactly; the written file exactly."""
import os

import numpy as np
import pytest

from conftest import GOLDEN

CASES = ("output_L3.npz", "output_L4_d2.npz")


def load(name):
    return dict(np.load(os.path.join(GOLDEN, name)))


@pytest.mark.parametrize("name", CASES)
def test_oracle_latlon_matches_reference(port, name):
    gd = load(name)
    g = port.build(int(gd["levels"]), int(gd["degree"]), None)
    for field, key in (("vor", "vor_ll"), ("u", "u_ll")):
        out = port.interp_to_latlon(g, gd[field], gd["lats"], gd["lons"])
        ref = gd[key]
        assert np.abs(out - ref).max() <= 1e-14 * np.abs(ref).max(), (name, field)
    out = port.interp_to_latlon(g, gd["vel"][0], gd["lats"], gd["lons"])
    assert np.abs(out - gd["velx_ll"]).max() <= 1e-14 * np.abs(gd["velx_ll"]).max()


@pytest.mark.parametrize("name", CASES)
def test_oracle_uv_matches_reference(port, name):
    gd = load(name)
    u, v = port.xyz_vel_to_uv_vel(gd["x"], gd["y"], gd["z"], *gd["vel"])
    assert np.abs(u - gd["u"]).max() <= 1e-14 * np.abs(gd["u"]).max()
    assert np.abs(v - gd["v"]).max() <= 1e-14 * np.abs(gd["v"]).max()


@pytest.mark.parametrize("name", CASES)
def test_output_grid_matches_driver(sb, name):
    gd = load(name)
    spacing, lats, lons = sb.output_grid(int(gd["point_count"]))
    assert spacing == float(gd["spacing"])
    assert np.array_equal(lats, gd["lats"]) and np.array_equal(lons, gd["lons"])


def test_output_grid_at_levels_7(sb):
    spacing, lats, lons = sb.output_grid(24576 * 9 + 2)  # 393,216 particles, degree 3
    assert spacing == 0.25 and len(lats) == 721 and len(lons) == 1440


def test_netcdf_writer_roundtrip(sb, tmp_path):
    from scipy.io import netcdf_file

    path = tmp_path / "output.nc"
    rng = np.random.default_rng(3)
    lats, lons = np.linspace(-90, 90, 5), np.arange(8) * 45.0
    vor = rng.standard_normal((3, 5, 8))
    with sb.NcFile(path) as nc:
        t = nc.def_dim("time", 3)
        la = nc.def_dim("latitude", 5)
        lo = nc.def_dim("longitude", 8)
        tv = nc.def_var("time", nc.INT, [t])
        lav = nc.def_var("latitude", nc.DOUBLE, [la])
        lov = nc.def_var("longitude", nc.DOUBLE, [lo])
        vv = nc.def_var("vor", nc.DOUBLE, [t, la, lo])
        nc.put_att(tv, "units", "s")
        nc.put_att(lav, "units", "degrees_north")
        nc.put_att(vv, "long name", "relative vorticity")
        nc.enddef()
        # global attributes after enddef, as the reference driver adds them
        nc.put_att(nc.GLOBAL, "initial condition", "rh4")
        nc.put_att(nc.GLOBAL, "tree levels", 3)
        nc.put_att(nc.GLOBAL, "fmm theta", 0.7)
        nc.put_vara(tv, np.array([0, 1800, 3600], np.int32))
        nc.put_vara(lav, lats)
        nc.put_vara(lov, lons)
        for k in (2, 0, 1):  # one time slab per call, out of order
            nc.put_vara(vv, vor[k:k + 1], start=[k, 0, 0])
        nc.put_vara(vv, np.full((1, 2, 3), 7.0), start=[1, 2, 4])  # an interior hyperslab
    expect = vor.copy()
    expect[1, 2:4, 4:7] = 7.0
    with netcdf_file(str(path), "r", mmap=False) as f:
        assert f.version_byte == 2
        assert f.dimensions == {"time": 3, "latitude": 5, "longitude": 8}
        assert np.array_equal(f.variables["time"][:], [0, 1800, 3600])
        assert np.array_equal(f.variables["latitude"][:], lats)
        assert np.array_equal(f.variables["longitude"][:], lons)
        assert np.array_equal(f.variables["vor"][:], expect)
        assert f.variables["latitude"].units == b"degrees_north"
        assert getattr(f.variables["vor"], "long name") == b"relative vorticity"
        assert getattr(f, "initial condition") == b"rh4"
        assert getattr(f, "tree levels") == 3 and getattr(f, "fmm theta") == 0.7


def test_netcdf_writer_rejects_misuse(sb, tmp_path):
    nc = sb.NcFile(tmp_path / "bad.nc")
    d = nc.def_dim("n", 4)
    v = nc.def_var("a", nc.DOUBLE, [d])
    with pytest.raises(sb.SbslpmError):
        nc.put_vara(v, np.zeros(4))  # before enddef
    nc.enddef()
    with pytest.raises(sb.SbslpmError):
        nc.put_vara(v, np.zeros(5))  # outside the variable
    with pytest.raises(sb.SbslpmError):
        nc.put_vara(v, np.zeros(4, np.int32))  # wrong type
    with pytest.raises(sb.SbslpmError):
        nc.def_dim("late", 2)  # after enddef
    nc.close()
