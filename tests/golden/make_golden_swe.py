"""Generate the shallow-water (SWE v2) golden vectors in tests/golden/ from the
reference itself.

Runs the reference's own unmodified code (oracle/_ref/libsbslpm_ref.so, built
by ``make -C oracle ref`` from the reference checkout) with one OpenMP thread,
so that its atomics accumulate in a fixed order, and stores small cases as .npz:

  swe_L3.npz        levels=3, degree=3, theta=0.7: points, the grid-point map
                    (cubed_sphere_2d_to_1d), the driver's set-up (initial
                    velocity and base tendencies), swe_tendency_computation_2
                    and swe_vel_interactions_2 on seeded inputs,
                    unify_boundary_vals, one swe_back_rk4_step_2 with the base
                    tendencies, one with zero base tendencies, and two steps of
                    the driver loop (step + unify of vors/divs/height).
  swe_L4_d2.npz     levels=4, degree=2, theta=0.5: set-up and one step.
  swe_L3_direct.npz levels=3, theta=1e-6 (every pair leaf-leaf): one step.
  swe_L4_unit.npz   levels=4, theta=0.7: the unit-sphere steady geostrophic
                    flow with N(0, 1e-4^2) height noise (the 393,216-particle
                    benchmark configuration at 6,144 particles), time scaled
                    by 500 so that dt = 0.002 is one integer second; 20 steps
                    of the driver loop.

Units are the reference's: the unit sphere with time in integer seconds,
Omega = 2 pi / 86400, and the height Laplacian scaled by the reference's
hard-coded 9.81/6371000 (height in units of the radius).  The initial state is
Williamson test case 2 (steady zonal flow, one revolution in 12 days, g h0 =
2.94e4 m^2/s^2) with a vorticity bump, a divergence bump and a height bump
added, so that every term of the step is exercised.  kernel_eps = 1e-4.

Usage:  make -C oracle ref && python tests/golden/make_golden_swe.py
"""
from __future__ import annotations

import os
import sys

os.environ["OMP_NUM_THREADS"] = "1"
HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import numpy as np  # noqa: E402

from oracle.pyoracle import Ref  # noqa: E402

OMEGA = 2 * np.pi / 86400.0
EPS = 1e-4
DT = 1800
G_OVER_A = 9.81 / 6371000.0


def swe_ic(x, y, z):
    """Test case 2 plus bumps, in the reference's units."""
    lat = np.arcsin(np.clip(z, -1, 1))
    u0 = 2 * np.pi / (12 * 86400.0)
    def bump(lat0, lon0, w):
        c = np.array([np.cos(lat0) * np.cos(lon0), np.cos(lat0) * np.sin(lon0), np.sin(lat0)])
        return np.exp(-w * ((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2))
    vors = 2 * u0 * np.sin(lat) + 2e-6 * bump(0.5, 1.0, 8.0)
    divs = 1e-6 * bump(-0.3, 2.5, 10.0)
    height = 2.94e4 / (9.81 * 6371000.0) - (OMEGA * u0 + 0.5 * u0 * u0) * np.sin(lat) ** 2 / G_OVER_A
    height = height + 2e-5 * bump(0.2, -1.5, 12.0)
    return vors, divs, height


def case(ref: Ref, levels, degree, theta, tracer_count, full, rng):
    c = ref.create(levels, degree, theta, EPS, OMEGA, DT, tracer_count)
    x, y, z, area, interp = ref.points(c)
    smap = ref.swe_map(c)
    vors, divs, height = swe_ic(x, y, z)
    out = dict(levels=levels, degree=degree, theta=theta, eps=EPS, omega=OMEGA, dt=float(DT), g_over_a=G_OVER_A,
               x=x, y=y, z=z, area=area, map=smap[0], counts=smap[1], vors=vors, divs=divs, height=height)
    vel, base = ref.swe_init(c, vors, divs, height, smap)
    out["init_vel"], out["init_base"] = np.stack(vel), np.stack(base)
    tr = np.stack([z, x][:tracer_count], axis=2).copy() if tracer_count else None
    if tr is not None:
        out["tracers_in"] = tr
    v, d, h, vel1, tr1 = ref.swe_step(c, vors, divs, height, base, smap, tracers=tr)
    out["step_vors"], out["step_divs"], out["step_height"], out["step_vel"] = v, d, h, np.stack(vel1)
    if tr1 is not None:
        out["step_tracers"] = tr1
    if full:
        A, q, P = c["A"], c["q"], c["P"]
        zero = [np.zeros((A, q)) for _ in range(3)]
        v, d, h, vel1, _ = ref.swe_step(c, vors, divs, height, zero, smap, tracers=tr)
        out["step0_vors"], out["step0_divs"], out["step0_height"], out["step0_vel"] = v, d, h, np.stack(vel1)
        v, d, h, vel2, tr2 = ref.swe_step(c, vors, divs, height, base, smap, tracers=tr, nsteps=2,
                                          driver_unify=True)
        out["run2_vors"], out["run2_divs"], out["run2_height"], out["run2_vel"] = v, d, h, np.stack(vel2)
        out["run2_tracers"] = tr2
        # the tendencies alone, on a perturbed velocity and a surface that differs from the height
        tvel = np.stack(vel) * (1 + 0.1 * rng.standard_normal((3, A, q)))
        surface = height + 1e-5 * rng.standard_normal((A, q))
        out["tend_vel"], out["tend_surface"] = tvel, surface
        out["tend_out"] = np.stack(ref.swe_tendency(c, [tvel[k] for k in range(3)], vors, divs, height, surface))
        # the interactions alone, on seeded displacements and sources
        disp = rng.standard_normal((3, P, q)) * 1e-3
        sv = rng.standard_normal((P, q)) * 1e-3
        sd = rng.standard_normal((P, q)) * 1e-3
        out["vi_disp"], out["vi_src_vor"], out["vi_src_div"] = disp, sv, sd
        out["vi_out"] = np.stack(ref.swe_vel_interactions(c, disp[0], disp[1], disp[2], sv, sd))
        # unify on a field that differs between the copies of a point
        f = rng.standard_normal((A, q))
        out["unify_in"], out["unify_out"] = f, ref.unify(c, f, smap)
    ref.destroy(c)
    return out


def unit_sphere_case(ref: Ref, levels, nsteps):
    """Omega = 2 pi, u0 = 2 pi/12, g h = 2.94 - (Omega u0 + u0^2/2) sin^2 lat
    (+ noise), dt = 0.002 on the unit sphere, expressed in the reference's
    units: time t' = 500 t (dt' = 1 s), so Omega' = Omega/500, vorticity and
    divergence / 500, and the height h' = (g h)/500^2/(9.81/6371000), which
    makes the reference's (9.81/6371000) lap(h') the unit-sphere lap(g h)."""
    S = 500.0
    om, u0 = 2 * np.pi, 2 * np.pi / 12
    c = ref.create(levels, 3, 0.7, EPS, om / S, 1, 0)
    x, y, z, area, interp = ref.points(c)
    smap = ref.swe_map(c)
    lat = np.arcsin(np.clip(z, -1, 1))
    vors = 2 * u0 * np.sin(lat) / S
    divs = np.zeros_like(vors)
    gh = 2.94 - (om * u0 + 0.5 * u0 * u0) * np.sin(lat) ** 2 + 1e-4 * np.random.default_rng(4).standard_normal(vors.shape)
    height = gh / S ** 2 / G_OVER_A
    out = dict(levels=levels, degree=3, theta=0.7, eps=EPS, omega=om / S, dt=1.0, g_over_a=G_OVER_A, x=x, y=y, z=z,
               area=area, vors=vors, divs=divs, height=height, time_scale=S, nsteps=nsteps)
    vel, base = ref.swe_init(c, vors, divs, height, smap)
    out["init_base"] = np.stack(base)
    v, d, h, vel2, _ = ref.swe_step(c, vors, divs, height, base, smap, vel=vel, nsteps=nsteps, driver_unify=True)
    out["run_vors"], out["run_divs"], out["run_height"], out["run_vel"] = v, d, h, np.stack(vel2)
    ref.destroy(c)
    return out


def main():
    ref = Ref()
    rng = np.random.default_rng(20261204)
    np.savez_compressed(os.path.join(HERE, "swe_L3.npz"), **case(ref, 3, 3, 0.7, 2, True, rng))
    np.savez_compressed(os.path.join(HERE, "swe_L4_d2.npz"), **case(ref, 4, 2, 0.5, 1, False, rng))
    np.savez_compressed(os.path.join(HERE, "swe_L3_direct.npz"), **case(ref, 3, 3, 1e-6, 0, False, rng))
    np.savez_compressed(os.path.join(HERE, "swe_L4_unit.npz"), **unit_sphere_case(ref, 4, 20))
    print("SWE golden vectors written to", HERE)


if __name__ == "__main__":
    main()
