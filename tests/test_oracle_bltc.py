"""Pin the oracle's treecode (decoupled proxy degree) against the reference.

tests/golden/bltc_*.npz hold the reference's own irregular-point FMM functions
(dual_tree_traversal_irreg, upward_pass_ll, swe_vel_interactions_ll with zero
divergence, downward_pass_3_ll; see tests/golden/make_golden_bltc.py) run on
the particle grid's truncated quadtree.  The oracle restates them in C
(oracle/bslpm_oracle.c, orc_bltc_*): its list must be identical, and its
passes and typed velocity agree to rounding (1e-13 relative; the strengths
are multiplied in another order).  The library's own treecode evaluates every
well-separated pair proxy x proxy; the oracle's untyped variant does the same,
and the last tests bound how far the two typings are apart, and how far both
are from the direct sum, on the headline's geometry (theta 0.7, degree-8
proxies, 256-particle leaves) at 24,576 particles.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from tests.golden.bltc_inputs import CASES, EPS, divs_of, down_in, pots_of

TOL = 1e-13


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.fixture(scope="module", params=sorted(CASES))
def case(request, port):
    gd = dict(np.load(os.path.join(GOLDEN, f"bltc_{request.param}.npz")))
    levels, degree, leaf, n, theta = CASES[request.param]
    g = port.build(levels, degree, None)
    return gd, g, (levels, degree, leaf, n, theta)


def test_tree_shape(case, port):
    gd, _, (levels, degree, leaf, _, _) = case
    assert port.bltc_shape(levels, degree, leaf) == (int(gd["tree_levels"]), int(gd["npl"]))


def test_list_is_the_irregular_traversal(case, port):
    gd, _, (levels, degree, leaf, n, theta) = case
    assert np.array_equal(port.bltc_list(levels, degree, leaf, n, theta), gd["list"])


def test_upward_pass(case, port):
    gd, g, (levels, degree, leaf, n, _) = case
    w = pots_of(g["x"], g["y"], g["z"]) * g["area"]
    assert rel(port.bltc_upward(levels, degree, leaf, n, g["x"], g["y"], g["z"], w), gd["upward"]) <= TOL


def test_downward_pass(case, port):
    gd, g, (levels, degree, leaf, n, _) = case
    T = np.stack(down_in(*gd["upward"].shape))
    _, u = port.bltc_downward(levels, degree, leaf, n, T, g["x"], g["y"], g["z"])
    assert rel(u, gd["down_out"].reshape(3, -1)) <= TOL


def test_typed_velocity(case, port):
    gd, g, (levels, degree, leaf, n, theta) = case
    p = (g["x"], g["y"], g["z"])
    w = pots_of(*p) * g["area"]
    u = port.bltc_velocity(levels, degree, leaf, n, theta, EPS, 1, p, p, w)
    assert rel(u, gd["vel"].reshape(3, -1)) <= TOL


def test_typed_shallow_water_velocity(case, port):
    """Both fields (vorticity and divergence at the grid points): the
    rotational and divergent parts of swe_vel_panel_interaction_ll."""
    gd, g, (levels, degree, leaf, n, theta) = case
    p = (g["x"], g["y"], g["z"])
    w = pots_of(*p) * g["area"]
    wd = divs_of(*p) * g["area"]
    u = port.bltc_velocity_swe(levels, degree, leaf, n, theta, EPS, 1, p, p, w, p, wd)
    assert rel(u, gd["vel_swe"].reshape(3, -1)) <= TOL


def test_untyped_velocity_within_the_treecode_error(case, port):
    """Proxy x proxy for every well-separated pair changes the result by the
    treecode's own approximation error, not more."""
    gd, g, (levels, degree, leaf, n, theta) = case
    p = (g["x"], g["y"], g["z"])
    w = pots_of(*p) * g["area"]
    u0 = port.bltc_velocity(levels, degree, leaf, n, theta, EPS, 0, p, p, w)
    assert rel(u0, gd["vel"].reshape(3, -1)) <= 1e-4


def test_headline_geometry_error_against_the_direct_sum(port):
    """theta 0.7, degree-8 proxies, 256-particle leaves at levels 5: both
    typings stay within 1e-6 of the float64 direct sum (velocity, relative
    L-infinity) and within a factor 2 of each other's error."""
    g = port.build(5, 3, None, exact_cc=True)
    p = (g["x"], g["y"], g["z"])
    w = pots_of(*p) * g["area"]
    P, q = len(g["panels"]), g["x"].shape[1]
    off = P - g["x"].shape[0]
    src = np.zeros((P, q))
    src[off:] = w
    zero = [np.zeros((P, q)) for _ in range(3)]
    ud = np.stack([t[off:].ravel() for t in port.direct_velocity(g, *zero, src, EPS)])
    err = [rel(port.bltc_velocity(5, 3, 256, 8, 0.7, EPS, typed, p, p, w.ravel()), ud) for typed in (0, 1)]
    assert max(err) <= 1e-6
    assert err[0] <= 2 * err[1] and err[1] <= 2 * err[0]
