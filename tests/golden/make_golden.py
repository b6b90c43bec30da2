"""Generate the golden vectors in tests/golden/ from the reference itself.

Runs the reference's own unmodified code (oracle/_ref/libsbslpm_ref.so, built by
``make -C oracle ref`` from the reference checkout) with one OpenMP thread, so
that its atomics accumulate in a fixed order, and stores small cases as .npz:

  bve_L3.npz     levels=3, degree=3, theta=0.7: panel table, interaction list,
                 points/areas/interp table, the reference's rh4 and gv initial
                 conditions, two bve_back_rk4_step calls with two tracers, and
                 one call of each pass (upward_pass, bve_vel_interactions,
                 downward_pass_3, departure, remap) on seeded random inputs.
  bve_L3_direct.npz  levels=3, theta=1e-6 (every pair leaf-leaf: the
                 reference's Biot-Savart direct sum) one step.
  bve_L4_d2.npz  levels=4, degree=2, theta=0.5: tree, list and one step.
  bli.npz        interp_vals_bli on seeded points, degrees 1..10, and
                 point_locate_panel on seeded sphere points (levels=4).
  inv_lap.npz    direct_sum_inv_lap on 400 seeded points.

Time is in the reference's integer seconds: dt = 1 with Omega = 2*pi/200, i.e.
the unit-sphere configuration (Omega = 2*pi, dt = 0.005) with time scaled by
200 (the reference's RunConfig::delta_t is an int).  kernel_eps = 1e-4 as in
the reference's namelist.txt.

Usage:  make -C oracle ref && python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

os.environ["OMP_NUM_THREADS"] = "1"
HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import numpy as np  # noqa: E402

from oracle.pyoracle import Ref  # noqa: E402

OMEGA = 2 * np.pi / 200.0
EPS = 1e-4


def step_case(ref: Ref, levels, degree, theta, tracer_count, nsteps, seed):
    c = ref.create(levels, degree, theta, EPS, OMEGA, 1, tracer_count)
    ints, dbls = ref.panels(c)
    lst = ref.interactions(c)
    x, y, z, area, interp = ref.points(c)
    out = dict(levels=levels, degree=degree, theta=theta, eps=EPS, omega=OMEGA, dt=1.0, panel_ints=ints,
               panel_dbls=dbls, list=lst, x=x, y=y, z=z, area=area, interp=interp)
    vor = ref.initialize(c, "rh4", True)
    out["ic_rh4"] = vor
    out["ic_gv"] = ref.initialize(c, "gv", True)
    tr = np.stack([z, x][:tracer_count], axis=2).copy() if tracer_count else None
    if tr is not None:
        out["tracers_in"] = tr
    v, vel, tr2 = ref.bve_step(c, vor, tr, nsteps=1)
    out["step1_vors"], out["step1_vel"] = v, np.stack(vel)
    if tr2 is not None:
        out["step1_tracers"] = tr2
    if nsteps > 1:
        v2, vel2, tr3 = ref.bve_step(c, v, tr2, time=1.0, nsteps=nsteps - 1)
        out[f"step{nsteps}_vors"], out[f"step{nsteps}_vel"] = v2, np.stack(vel2)
        if tr3 is not None:
            out[f"step{nsteps}_tracers"] = tr3
    return c, out


def main():
    ref = Ref()
    rng = np.random.default_rng(20261203)

    c, out = step_case(ref, 3, 3, 0.7, 2, 2, 1)
    P, A, q = c["P"], c["A"], c["q"]
    # single passes on seeded random inputs
    pots = rng.standard_normal((A, q))
    out["up_pots"] = pots
    out["up_proxy"] = ref.upward_pass(c, pots)
    disp = rng.standard_normal((3, P, q)) * 1e-3
    src = rng.standard_normal((P, q)) * 1e-3
    out["vi_disp"], out["vi_src"] = disp, src
    out["vi_out"] = np.stack(ref.vel_interactions(c, disp[0].copy(), disp[1].copy(), disp[2].copy(), src))
    tin = rng.standard_normal((3, P, q))
    out["down_in"] = tin
    t1, t2, t3 = (tin[i].copy() for i in range(3))
    out["down_sols"] = np.stack(ref.downward_pass_3(c, t1, t2, t3))
    # random velocities of realistic size in the scaled units (|v| ~ 0.2 / 200)
    vel = rng.standard_normal((4, 3, A, q)) * (0.2 / 200.0)
    out["dep_vel"] = vel
    dep = ref.departure(c, *[vel[k].reshape(3 * A, q) for k in range(4)], 1.0)
    out["dep_out"] = np.stack(dep)
    out["remap_vors"] = out["ic_rh4"]
    nv, ntr = ref.remap(c, dep, out["ic_rh4"], out["tracers_in"])
    out["remap_new_vors"], out["remap_new_tracers"] = nv, ntr
    np.savez_compressed(os.path.join(HERE, "bve_L3.npz"), **out)
    ref.destroy(c)

    c, out = step_case(ref, 3, 3, 1e-6, 0, 1, 2)
    np.savez_compressed(os.path.join(HERE, "bve_L3_direct.npz"), **out)
    ref.destroy(c)

    c, out = step_case(ref, 4, 2, 0.5, 1, 1, 3)
    np.savez_compressed(os.path.join(HERE, "bve_L4_d2.npz"), **out)

    # BLI and point location
    bl = {}
    for d in range(1, 11):
        pts = []
        for _ in range(20):
            a, b = np.sort(rng.uniform(-np.pi / 4, np.pi / 4, 2))
            e, f = np.sort(rng.uniform(-np.pi / 4, np.pi / 4, 2))
            xi, eta = rng.uniform(a, b), rng.uniform(e, f)
            pts.append((xi, eta, a, b, e, f))
        # exact-node hits: a node in xi, a node in eta
        a, b, e, f = -0.3, 0.5, -0.7, 0.1
        node = np.cos(np.pi * 1 / d) * 0.5 * (b - a) + 0.5 * (b + a)
        pts.append((node, 0.2 * e + 0.8 * f, a, b, e, f))
        pts = np.array(pts)
        vals = np.stack([ref.bli(*p, d) for p in pts])
        bl[f"bli_pts_d{d}"], bl[f"bli_vals_d{d}"] = pts, vals
    xyz = rng.standard_normal((2000, 3))
    xyz /= np.linalg.norm(xyz, axis=1, keepdims=True)
    bl["loc_xyz"] = xyz
    bl["loc_leaf"] = np.array([ref.locate(c, *p) for p in xyz], np.int32)
    bl["loc_levels"] = 4
    np.savez_compressed(os.path.join(HERE, "bli.npz"), **bl)
    ref.destroy(c)

    n = 400
    xyz = rng.standard_normal((n, 3))
    xyz /= np.linalg.norm(xyz, axis=1, keepdims=True)
    area = rng.uniform(0.5, 1.5, n) * 4 * np.pi / n
    pots = rng.standard_normal(n)
    soln = ref.direct_sum_inv_lap(*[np.ascontiguousarray(xyz[:, i]) for i in range(3)], area, pots)
    np.savez_compressed(os.path.join(HERE, "inv_lap.npz"), xyz=xyz, area=area, pots=pots, soln=soln)
    print("golden vectors written to", HERE)


if __name__ == "__main__":
    main()
