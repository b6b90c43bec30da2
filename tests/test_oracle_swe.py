"""The C restatement of the shallow-water (SWE v2) step against the
reference's own outputs (CPU, no GPU).

oracle/bslpm_oracle.c restates swe_vel_interactions_2, the finite-difference
tendencies of swe_tendency_computation_2 (fd_deriv_xi / fd_deriv_eta,
spatial_filter_vals, single_panel_lap_fd, single_panel_curl_rad_comp_fd,
single_panel_div_fd, xietavec_from_xyzvec), unify_boundary_vals and the whole
swe_back_rk4_step_2.  The golden vectors come from the reference compiled
here (tests/golden/make_golden_swe.py, one OpenMP thread); the restatement
keeps the reference's operand order and single-thread summation order, so it
agrees bit for bit on this machine; the tolerance (1e-14 relative) only
allows for a different libm.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN

TOL = 1e-14
FIXTURES = ["swe_L3.npz", "swe_L4_d2.npz", "swe_L3_direct.npz"]


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    s = np.abs(b).max()
    return float(np.abs(a - b).max() / (s if s > 0 else 1.0))


def load(name):
    return dict(np.load(os.path.join(GOLDEN, name)))


def grid(port, gd):
    g = port.build(int(gd["levels"]), int(gd["degree"]), float(gd["theta"]))
    assert np.array_equal(g["x"], gd["x"]) and np.array_equal(g["area"], gd["area"])
    return g


def kw(gd):
    return dict(dt=float(gd["dt"]), omega=float(gd["omega"]), eps=float(gd["eps"]), g_over_a=float(gd["g_over_a"]))


def test_swe_tendencies_interactions_and_unify(port):
    gd = load("swe_L3.npz")
    g = grid(port, gd)
    t = port.swe_tendencies(g, gd["tend_vel"], gd["vors"], gd["divs"], gd["height"], gd["tend_surface"],
                            float(gd["omega"]), float(gd["g_over_a"]))
    for k in range(3):
        assert rel(t[k], gd["tend_out"][k]) <= TOL, k
    vi = port.swe_vel_interactions(g, *gd["vi_disp"], gd["vi_src_vor"], gd["vi_src_div"], float(gd["eps"]))
    assert rel(np.stack(vi), gd["vi_out"]) <= TOL
    # the mean of the copies of each point: the same additions in the same order
    assert np.array_equal(port.swe_unify(gd["unify_in"], gd["map"], gd["counts"]), gd["unify_out"])


@pytest.mark.parametrize("name", FIXTURES)
def test_swe_step_matches_reference(port, name):
    gd = load(name)
    g = grid(port, gd)
    tr = gd.get("tracers_in")
    v, d, h, vel, trr = port.swe_step(g, gd["vors"], gd["divs"], gd["height"], gd["init_base"], gd["map"],
                                      gd["counts"], tr, **kw(gd))
    assert rel(v, gd["step_vors"]) <= TOL
    assert rel(d, gd["step_divs"]) <= TOL
    assert rel(h, gd["step_height"]) <= TOL
    assert rel(np.stack(vel), gd["step_vel"]) <= TOL
    if tr is not None:
        assert rel(trr, gd["step_tracers"]) <= TOL


def test_swe_step_without_base_tendencies_and_driver_loop(port):
    gd = load("swe_L3.npz")
    g = grid(port, gd)
    tr = gd["tracers_in"]
    v, d, h, vel, _ = port.swe_step(g, gd["vors"], gd["divs"], gd["height"], np.zeros_like(gd["init_base"]),
                                    gd["map"], gd["counts"], tr, **kw(gd))
    for got, want in ((v, "step0_vors"), (d, "step0_divs"), (h, "step0_height"), (np.stack(vel), "step0_vel")):
        assert rel(got, gd[want]) <= TOL, want
    # two steps of the driver's loop: step, then unify vorticity, divergence and height
    v, d, h, vel, trr = port.swe_step(g, gd["vors"], gd["divs"], gd["height"], gd["init_base"], gd["map"],
                                      gd["counts"], tr, nsteps=2, driver_unify=True, **kw(gd))
    for got, want in ((v, "run2_vors"), (d, "run2_divs"), (h, "run2_height"), (np.stack(vel), "run2_vel"),
                      (trr, "run2_tracers")):
        assert rel(got, gd[want]) <= TOL, want
