"""Pin the C restatement oracle against golden vectors made by the reference.

The vectors in tests/golden/ come from the reference's own code (see
tests/golden/make_golden.py).  The restatement keeps the reference's operand
order and accumulation order, so agreement is expected to the last bit; the
tolerance below (1e-14 relative) only allows for a different libm.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from oracle.pyoracle import panels_to_arrays

TOL = 1e-14


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    s = np.abs(b).max()
    return np.abs(a - b).max() / (s if s > 0 else 1.0)


def load(name):
    return dict(np.load(os.path.join(GOLDEN, name)))


@pytest.fixture(scope="module")
def g3(port):
    gd = load("bve_L3.npz")
    g = port.build(int(gd["levels"]), int(gd["degree"]), float(gd["theta"]))
    return gd, g


def test_tree_and_list(g3):
    gd, g = g3
    ints, dbls = panels_to_arrays(g["panels"])
    assert (ints == gd["panel_ints"]).all()
    assert rel(dbls, gd["panel_dbls"]) <= TOL
    assert np.array_equal(g["list"], gd["list"])
    for k in ("x", "y", "z", "area", "interp"):
        assert rel(g[k], gd[k]) <= TOL, k


def test_tree_and_list_L4_d2(port):
    gd = load("bve_L4_d2.npz")
    g = port.build(4, 2, 0.5)
    ints, _ = panels_to_arrays(g["panels"])
    assert (ints == gd["panel_ints"]).all()
    assert np.array_equal(g["list"], gd["list"])
    assert rel(g["area"], gd["area"]) <= TOL


def test_interaction_counts_match_survey(port):
    # levels=5 (6 x 16 x 16 leaf panels), theta=0.7: 75,438 pairs, split
    # 53,376 pp / 9,984 pc / 0 cp / 12,078 cc in the reference's traversal.
    g = port.build(5, 3, 0.7)
    assert len(g["list"]) == 75438
    assert np.bincount(g["list"][:, 2], minlength=4).tolist() == [53376, 9984, 0, 12078]


def test_upward_pass(g3, port):
    gd, g = g3
    assert rel(port.upward_pass(g, gd["up_pots"]), gd["up_proxy"]) <= TOL


def test_vel_interactions(g3, port):
    gd, g = g3
    d = gd["vi_disp"]
    out = port.vel_interactions(g, d[0].copy(), d[1].copy(), d[2].copy(), gd["vi_src"], float(gd["eps"]))
    assert rel(np.stack(out), gd["vi_out"]) <= TOL


def test_downward_pass(g3, port):
    gd, g = g3
    t = gd["down_in"]
    s = port.downward_pass_3(g, t[0], t[1], t[2])
    assert rel(np.stack(s), gd["down_sols"]) <= TOL


def test_departure_and_remap(g3, port):
    gd, g = g3
    v = gd["dep_vel"]
    A, q = g["x"].shape
    dep = port.departure(g, *[v[k].reshape(3 * A, q) for k in range(4)], 1.0)
    assert rel(np.stack(dep), gd["dep_out"]) <= TOL
    nv, ntr = port.remap(g, gd["dep_out"], gd["remap_vors"], gd["tracers_in"], float(gd["omega"]))
    assert rel(nv, gd["remap_new_vors"]) <= TOL
    assert rel(ntr, gd["remap_new_tracers"]) <= TOL


@pytest.mark.parametrize("name", ["bve_L3.npz", "bve_L3_direct.npz", "bve_L4_d2.npz"])
def test_bve_step(port, name):
    gd = load(name)
    theta = float(gd["theta"])
    g = port.build(int(gd["levels"]), int(gd["degree"]), theta)
    tr = gd.get("tracers_in")
    v, vel, tr1 = port.bve_step(g, gd["ic_rh4"], tr, dt=float(gd["dt"]), omega=float(gd["omega"]),
                                eps=float(gd["eps"]), mode=0)
    assert rel(v, gd["step1_vors"]) <= TOL
    assert rel(np.stack(vel), gd["step1_vel"]) <= TOL
    if tr is not None:
        assert rel(tr1, gd["step1_tracers"]) <= TOL
    if "step2_vors" in gd:
        v2, vel2, _ = port.bve_step(g, v, tr1, dt=1.0, omega=float(gd["omega"]), eps=float(gd["eps"]), mode=0)
        assert rel(v2, gd["step2_vors"]) <= TOL
        assert rel(np.stack(vel2), gd["step2_vel"]) <= TOL


def test_direct_mode_equals_theta_to_zero(port):
    """The oracle's direct (all leaf pairs) mode reproduces the reference run
    at theta = 1e-6, whose list holds every leaf-leaf pair (in another order,
    hence a tolerance rather than bit equality)."""
    gd = load("bve_L3_direct.npz")
    g = port.build(3, 3, None)
    v, vel, _ = port.bve_step(g, gd["ic_rh4"], None, dt=1.0, omega=float(gd["omega"]), eps=float(gd["eps"]), mode=1)
    assert rel(np.stack(vel), gd["step1_vel"]) <= 1e-13
    assert rel(v, gd["step1_vors"]) <= 1e-13


def test_bli_and_locate(port):
    gd = load("bli.npz")
    for d in range(1, 11):
        for p, want in zip(gd[f"bli_pts_d{d}"], gd[f"bli_vals_d{d}"]):
            assert rel(port.bli(*p, d), want) <= TOL
    g = port.build(int(gd["loc_levels"]), 3, None)
    got = np.array([port.locate(g, *p) for p in gd["loc_xyz"]])
    assert np.array_equal(got, gd["loc_leaf"])


def test_inv_lap(port):
    gd = load("inv_lap.npz")
    xyz = gd["xyz"]
    out = port.direct_sum_inv_lap(*[np.ascontiguousarray(xyz[:, i]) for i in range(3)], gd["area"], gd["pots"])
    assert rel(out, gd["soln"]) <= TOL


def test_area_kat_exact_cc(port):
    """Known answer: with exact Clenshaw-Curtis weights the particle areas sum
    to the sphere's area 4*pi (to the accuracy of the panel areas)."""
    g = port.build(4, 3, None, exact_cc=True)
    assert abs(g["area"].sum() - 4 * np.pi) < 1e-10
    # the reference's weights miss the middle node for odd degree
    g = port.build(4, 3, None, exact_cc=False)
    assert abs(g["area"].sum() - 4 * np.pi * (10 / 9) ** 2 / 4) < 1e-10


def test_solid_body_rotation_is_steady(port):
    """Known answer from the reference's 'rot' IC: vorticity proportional to z
    (solid-body rotation) stays steady under the BVE step."""
    g = port.build(4, 4, 0.7, exact_cc=True)
    om, a = 2 * np.pi / 200, 1 / 400
    vor = 2 * a * g["z"]
    v, vel, _ = port.bve_step(g, vor, None, dt=1.0, omega=om, eps=1e-4, mode=0)
    assert rel(v, vor) < 1e-3
    # the velocity is the rigid rotation a * (z_hat x x)
    assert np.abs(vel[0] + a * g["y"]).max() / a < 2e-2
    assert np.abs(vel[1] - a * g["x"]).max() / a < 2e-2


@pytest.mark.parametrize("case", ["ssw_ramp", "ssw2_plateau", "ssw_down"])
def test_forced_step_matches_reference(port, case):
    """bve_back_rk4_step with the SSW forcing on (src/forcing_funcs.cpp:6-96)."""
    gd = load("bve_forcing_L3.npz")
    g = port.build(3, 3, 0.7)
    v, vel, _ = port.bve_step(g, gd["ic"], None, dt=1.0, omega=float(gd["omega"]), eps=float(gd["eps"]), mode=0,
                              nsteps=int(gd[case + "_n"]), forcing=int(gd[case + "_forcing"]),
                              time=float(gd[case + "_t0"]))
    assert rel(v, gd[case + "_vors"]) <= TOL
    assert rel(np.stack(vel), gd[case + "_vel"]) <= TOL
