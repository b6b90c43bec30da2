"""Generate the output-path golden vectors (tests/golden/output_L3.npz,
output_L4_d2.npz) from the reference itself.

Runs the reference's own unmodified code (oracle/_ref/libsbslpm_ref.so, built
by ``make -C oracle ref`` from the reference checkout) with one OpenMP thread:
the Rossby-Haurwitz vorticity and the velocity after one bve_back_rk4_step,
their zonal / meridional components by xyz_vel_to_uv_vel
(src/general_utils_impl.hpp:195-229), and interp_to_latlon_host
(src/interp_funcs.hpp:22-77) of the vorticity, u and vel_x onto the lat-lon
grid the reference's driver writes (executables/bve_time_evo.cpp:93-95,
206-211: spacing 2^floor(log2(sqrt(4 pi / point_count) * 180 / pi)) degrees,
latitudes -90..90 and longitudes 0..360-spacing), which puts points on the
poles and on cube-face edges.

Usage:  make -C oracle ref && python tests/golden/make_golden_output.py
"""
from __future__ import annotations

import os
import sys

os.environ["OMP_NUM_THREADS"] = "1"
HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import numpy as np  # noqa: E402

from oracle.pyoracle import Ref  # noqa: E402


def output_grid(point_count):
    spacing = 2.0 ** np.floor(np.log2(np.sqrt(4 * np.pi / point_count) * 180.0 / np.pi))
    nlat, nlon = int(180.0 / spacing + 1.0), int(360.0 / spacing)
    return spacing, -90.0 + spacing * np.arange(nlat), spacing * np.arange(nlon)


def case(ref, levels, degree):
    c = ref.create(levels, degree, 0.7, 1e-4, 2 * np.pi, 1, 0)
    ints, dbls = ref.panels(c)
    x, y, z, area, interp = ref.points(c)
    vor = ref.initialize(c, "rh4", True)
    v1, vel, _ = ref.bve_step(c, vor.copy(), None, nsteps=1)
    u, v = ref.xyz_vel_to_uv_vel(c, *vel)
    point_count = c["A"] * degree * degree + 2
    spacing, lats, lons = output_grid(point_count)
    out = dict(levels=levels, degree=degree, panel_ints=ints, panel_dbls=dbls, x=x, y=y, z=z, vor=vor,
               vel=np.stack(vel), u=u, v=v, point_count=point_count, spacing=spacing, lats=lats, lons=lons,
               vor_ll=ref.interp_to_latlon(c, vor, lats, lons), u_ll=ref.interp_to_latlon(c, u, lats, lons),
               velx_ll=ref.interp_to_latlon(c, vel[0], lats, lons))
    ref.destroy(c)
    return out


def main():
    ref = Ref()
    for name, levels, degree in (("output_L3", 3, 3), ("output_L4_d2", 4, 2)):
        out = case(ref, levels, degree)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        print(name, {k: np.shape(v) for k, v in out.items() if np.ndim(v)})


if __name__ == "__main__":
    main()
