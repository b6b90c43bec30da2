"""CPU tests of the product library: the C ABI loads, exports every symbol
include/sbslpm.h declares, and its host-side setup functions (tree,
interpolation table, points, traversal, BLI, point location, namelist)
reproduce the reference's golden vectors.  No compute call needs a GPU here."""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN, ROOT

HEADER = os.path.join(ROOT, "include", "sbslpm.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sbslpm_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(sb):
    path = sb.library_path()
    assert os.path.exists(path)
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (sbslpm_\w+)", out))
    missing = [s for s in declared_symbols() if s not in exported]
    assert not missing, missing
    assert len(declared_symbols()) >= 25


def test_library_is_sm100a(sb):
    out = subprocess.run(["/usr/local/cuda/bin/cuobjdump", "--list-elf", sb.library_path()], capture_output=True,
                         text=True)
    if out.returncode != 0:
        pytest.skip("cuobjdump unavailable")
    assert "sm_100a" in out.stdout


def load(name):
    return dict(np.load(os.path.join(GOLDEN, name)))


def panel_arrays(panels):
    ints = np.array([[p.id, p.id_top_edge, p.id_left_edge, p.id_bot_edge, p.id_right_edge, p.face, p.level,
                      p.parent_id, p.child1, p.child2, p.child3, p.child4, p.is_leaf] for p in panels], np.int32)
    dbls = np.array([[p.min_xi, p.max_xi, p.min_eta, p.max_eta, p.radius, p.area] for p in panels])
    return ints, dbls


@pytest.mark.parametrize("name", ["bve_L3.npz", "bve_L4_d2.npz"])
def test_setup_matches_reference(sb, name):
    gd = load(name)
    L, d = int(gd["levels"]), int(gd["degree"])
    panels = sb.cubed_sphere_panels_init(L)
    ints, dbls = panel_arrays(panels)
    assert (ints == gd["panel_ints"]).all()
    assert np.array_equal(dbls, gd["panel_dbls"])
    interp = sb.interp_init(d, exact_cc=False)
    assert np.array_equal(interp, gd["interp"])
    x, y, z, area = sb.cube_sphere_spec_points(L, d, panels, interp)
    for a, k in ((x, "x"), (y, "y"), (z, "z"), (area, "area")):
        assert np.array_equal(a, gd[k]), k
    lst = sb.dual_tree_traversal(L, panels, float(gd["theta"]))
    assert np.array_equal(lst, gd["list"])


def test_traversal_counts_levels7(sb):
    """393,216-particle tree (6 x 64 x 64 leaves), theta = 0.7."""
    panels = sb.cubed_sphere_panels_init(7)
    lst = sb.dual_tree_traversal(7, panels, 0.7)
    assert len(lst) == 1224342
    assert np.bincount(lst[:, 2], minlength=4).tolist() == [862560, 144648, 0, 217134]


def test_bli_and_locate_match_reference(sb):
    gd = load("bli.npz")
    for d in range(1, 11):
        for p, want in zip(gd[f"bli_pts_d{d}"], gd[f"bli_vals_d{d}"]):
            got = sb.interp_vals_bli(*p, d)
            assert np.abs(got - want).max() <= 1e-14 * max(1.0, np.abs(want).max())
    panels = sb.cubed_sphere_panels_init(int(gd["loc_levels"]))
    got = np.array([sb.point_locate_panel(panels, *p) for p in gd["loc_xyz"]])
    assert np.array_equal(got, gd["loc_leaf"])


def test_bli_out_of_panel_is_an_error(sb):
    with pytest.raises(sb.SbslpmError) as e:
        sb.interp_vals_bli(0.9, 0.0, -0.5, 0.5, -0.5, 0.5, 3)
    assert e.value.status == 3


def test_exact_cc_areas_sum_to_sphere(sb):
    g = sb.build_grid(4, 3, exact_cc=True)
    assert abs(g.area.sum() - 4 * np.pi) < 1e-10


def test_read_run_config(sb, tmp_path):
    nl = tmp_path / "namelist.txt"
    nl.write_text("out_path=../x\nlevels=7\ninterp_degree=12\ntheta=0.5\nkernel_eps=1e-4\ndelta_t=50\n"
                  "tracers=vor,z,x,y\nprecision=mixed\nvelocity=direct\nend\nlevels=3\n")
    cfg = sb.read_run_config(str(nl))
    assert cfg.levels == 7 and cfg.interp_degree == 10 and cfg.fmm_theta == 0.5
    assert cfg.dt == 50.0 and cfg.tracer_count == 4 and cfg.kernel_eps == 1e-4
    assert cfg.precision == sb.MIXED and cfg.velocity == sb.VEL_DIRECT
    bad = tmp_path / "bad.txt"
    bad.write_text("levels=abc\nend\n")
    with pytest.raises(sb.SbslpmError):
        sb.read_run_config(str(bad))
    with pytest.raises(sb.SbslpmError):
        sb.read_run_config(str(tmp_path / "missing.txt"))


def test_reference_namelist_keys_parse(sb, tmp_path):
    """The reference's shipped namelist format (key=value, 'end' terminator)."""
    nl = tmp_path / "namelist.txt"
    nl.write_text("out_path=../../run-output\nwrite_precision=16\nwrite_output=1\nlevels=7\ninterp_degree=10\n"
                  "grid_spacing=1\nend_time=432000\ndelta_t=50\noutput_vel=1\noutput_freq=1\n"
                  "initial_condition=galewsky\nbalance_ic=1\ntheta=0.5\ninterp_output=1\ntracers=vor,z,x,y\n"
                  "kernel_eps=1e-4\nforcing=0\nforcing_type=none\ntopo_type=none\nend")
    cfg = sb.read_run_config(str(nl))
    assert (cfg.levels, cfg.interp_degree, cfg.fmm_theta, cfg.dt, cfg.tracer_count) == (7, 10, 0.5, 50.0, 4)


def test_config_validation(sb):
    with pytest.raises(sb.SbslpmError):
        sb.Context(sb.config_default(levels=0))
    with pytest.raises(sb.SbslpmError):
        sb.Context(sb.config_default(precision=sb.MIXED, interp_degree=8))


@pytest.mark.parametrize("degree", [1, 2, 3, 4, 6, 8, 10])
def test_bli_reproduces_polynomials(sb, degree):
    """Known answer: the barycentric Lagrange basis on a panel's Chebyshev
    nodes (sbslpm_interp_vals_bli, src/interp_funcs_impl.hpp:11-142)
    reproduces every tensor-product polynomial of degree <= d exactly."""
    rng = np.random.default_rng(degree)
    it = sb.interp_init(degree)
    lo_x, hi_x, lo_y, hi_y = -0.3, 0.5, -0.2, 0.2
    X = lo_x + (it[:, 0] + 1) / 2 * (hi_x - lo_x)
    Y = lo_y + (it[:, 1] + 1) / 2 * (hi_y - lo_y)
    for _ in range(4):
        a = rng.standard_normal((degree + 1, degree + 1))

        def p(x, y):
            return sum(a[i, j] * x ** i * y ** j for i in range(degree + 1) for j in range(degree + 1))

        vals = p(X, Y)
        for _ in range(8):
            xi, eta = rng.uniform(lo_x, hi_x), rng.uniform(lo_y, hi_y)
            b = sb.interp_vals_bli(xi, eta, lo_x, hi_x, lo_y, hi_y, degree)
            assert abs(b @ vals - p(xi, eta)) <= 1e-12 * max(1.0, abs(p(xi, eta)))
