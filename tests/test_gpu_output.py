"""GPU parity of the output path, through the C ABI: the lat-lon
interpolation and the zonal / meridional velocity against the reference's own
outputs (tests/golden/make_golden_output.py) and the oracle, and one output
file written from a GPU step and read back.

Tolerances (relative L-infinity): <= 1e-13 for the interpolation (device and
host libm sin / cos / atan may differ in the last bit), <= 1e-14 for u, v."""
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

CASES = ("output_L3.npz", "output_L4_d2.npz")


def rel(a, b):
    a = a.detach().cpu().numpy() if hasattr(a, "detach") else np.asarray(a)
    s = np.abs(b).max()
    return float(np.abs(a - b).max() / (s if s > 0 else 1.0))


def cuda(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def ctx_for(sb, gd):
    return sb.Context(sb.config_default(levels=int(gd["levels"]), interp_degree=int(gd["degree"]), kernel_eps=1e-4,
                                        omega=2 * np.pi, dt=1.0))


@pytest.mark.parametrize("name", CASES)
def test_latlon_matches_reference(sb, port, name):
    gd = dict(np.load(os.path.join(GOLDEN, name)))
    ctx = ctx_for(sb, gd)
    lats, lons = cuda(gd["lats"]), cuda(gd["lons"])
    for field, key in (("vor", "vor_ll"), ("u", "u_ll")):
        out = ctx.interp_to_latlon(cuda(gd[field]), lats, lons)
        assert rel(out, gd[key]) <= 1e-13, (name, field, rel(out, gd[key]))
    out = ctx.interp_to_latlon(cuda(gd["vel"][0]), lats, lons)
    assert rel(out, gd["velx_ll"]) <= 1e-13
    # an off-grid set of points against the oracle (random latitudes and longitudes)
    rng = np.random.default_rng(7)
    la, lo = rng.uniform(-90, 90, 37), rng.uniform(-180, 360, 53)
    g = port.build(int(gd["levels"]), int(gd["degree"]), None)
    want = port.interp_to_latlon(g, gd["vor"], la, lo)
    assert rel(ctx.interp_to_latlon(cuda(gd["vor"]), cuda(la), cuda(lo)), want) <= 1e-13


@pytest.mark.parametrize("name", CASES)
def test_uv_matches_reference(sb, name):
    gd = dict(np.load(os.path.join(GOLDEN, name)))
    ctx = ctx_for(sb, gd)
    u, v = ctx.xyz_vel_to_uv_vel(cuda(gd["x"]), cuda(gd["y"]), cuda(gd["z"]), *[cuda(c) for c in gd["vel"]])
    assert rel(u, gd["u"]) <= 1e-14 and rel(v, gd["v"]) <= 1e-14


def test_step_output_file(sb, tmp_path):
    """The driver's per-step output (executables/bve_time_evo.cpp:300-350) from
    device fields: a GPU step, u / v, lat-lon interpolation, netCDF file."""
    from scipy.io import netcdf_file

    g = sb.build_grid(4, 3, exact_cc=True)
    cfg = sb.config_default(levels=4, interp_degree=3, kernel_eps=1e-4, omega=2 * np.pi, dt=0.005)
    ctx = sb.Context(cfg)
    x, y, z, area = (cuda(a) for a in (g.x, g.y, g.z, g.area))
    lat = torch.asin(z.clamp(-1, 1))
    vors = 2 * 0.5 * torch.sin(lat) - 0.5 * torch.sin(lat) * torch.cos(lat) ** 4 * 30 * torch.cos(4 * torch.atan2(y, x))
    vel = [torch.zeros_like(x) for _ in range(3)]
    spacing, lats, lons = sb.output_grid(g.x.size // 16 * 9 + 2)
    dl, dn = cuda(lats), cuda(lons)
    path = tmp_path / "output.nc"
    with sb.NcFile(path) as nc:
        t = nc.def_dim("time", 3)
        la, lo = nc.def_dim("latitude", len(lats)), nc.def_dim("longitude", len(lons))
        ids = {k: nc.def_var(k, nc.DOUBLE, [t, la, lo]) for k in ("vor", "u_vel", "v_vel")}
        lav, lov = nc.def_var("latitude", nc.DOUBLE, [la]), nc.def_var("longitude", nc.DOUBLE, [lo])
        nc.enddef()
        nc.put_vara(lav, lats)
        nc.put_vara(lov, lons)
        nc.put_vara(ids["vor"], ctx.interp_to_latlon(vors, dl, dn).cpu().numpy()[None], start=[0, 0, 0])
        kept = []
        for k in (1, 2):
            ctx.bve_back_rk4_step(x, y, z, area, vors, *vel)
            u, v = ctx.xyz_vel_to_uv_vel(x, y, z, *vel)
            for key, fld in (("vor", vors), ("u_vel", u), ("v_vel", v)):
                arr = ctx.interp_to_latlon(fld, dl, dn).cpu().numpy()
                nc.put_vara(ids[key], arr[None], start=[k, 0, 0])
                kept.append(arr)
    with netcdf_file(str(path), "r", mmap=False) as f:
        assert np.array_equal(f.variables["vor"][2], kept[3])
        assert np.array_equal(f.variables["u_vel"][1], kept[1])
        assert np.isfinite(f.variables["v_vel"][1:]).all() and np.abs(f.variables["u_vel"][2]).max() > 0
