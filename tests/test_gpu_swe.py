"""GPU parity tests of the shallow-water (SWE v2) step, through the C ABI.

Checkers: golden vectors made by the reference itself (tests/golden/swe_*.npz,
tests/golden/make_golden_swe.py), and at 24,576 particles the oracle's C
restatement of swe_back_rk4_step_2 (oracle/bslpm_oracle.c, pinned bit for
bit to those vectors by tests/test_oracle_swe.py).  Tolerances (relative L-infinity, scaled by
the largest reference magnitude of the field):
  float64 path            <= 1e-12 (step, tendencies, interactions, set-up)
  unify_boundary_vals     bit-exact (same summation order, IEEE operations)
  mixed-precision path    <= 1e-6 against the float64 path (vorticity, height)
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

FP64_TOL = 1e-12
MIXED_TOL = 1e-6


def rel(a, b):
    a = a.detach().cpu().numpy() if hasattr(a, "detach") else np.asarray(a)
    b = b.detach().cpu().numpy() if hasattr(b, "detach") else np.asarray(b)
    s = np.abs(b).max()
    return float(np.abs(a - b).max() / (s if s > 0 else 1.0))


def cuda(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def load(name):
    return dict(np.load(os.path.join(GOLDEN, name)))


def golden_ctx(sb, gd, **kw):
    theta = float(gd["theta"])
    vel = sb.VEL_DIRECT if theta < 1e-3 else sb.VEL_FMM
    cfg = sb.config_default(levels=int(gd["levels"]), interp_degree=int(gd["degree"]), fmm_theta=theta,
                            kernel_eps=float(gd["eps"]), omega=float(gd["omega"]), dt=float(gd["dt"]),
                            tracer_count=int(gd["tracers_in"].shape[2]) if "tracers_in" in gd else 0, velocity=vel,
                            g_over_a=float(gd["g_over_a"]))
    for k, v in kw.items():
        setattr(cfg, k, v)
    return sb.Context(cfg)


class State:
    def __init__(self, gd, base=None):
        A, q = gd["x"].shape
        self.x, self.y, self.z, self.area = (cuda(gd[k]) for k in ("x", "y", "z", "area"))
        self.vors, self.divs, self.height = (cuda(gd[k]) for k in ("vors", "divs", "height"))
        self.vel = [torch.zeros(A, q, dtype=torch.float64, device="cuda") for _ in range(3)]
        self.tr = cuda(gd["tracers_in"]) if "tracers_in" in gd else None
        b = gd["init_base"] if base is None else base
        self.base = [cuda(b[k]) for k in range(3)]

    def args(self):
        return (self.x, self.y, self.z, self.area, self.vors, self.divs, self.height, *self.vel, self.tr, *self.base)


@pytest.mark.parametrize("name", ["swe_L3.npz", "swe_L4_d2.npz", "swe_L3_direct.npz"])
def test_swe_init_matches_reference(sb, name):
    gd = load(name)
    ctx = golden_ctx(sb, gd)
    s = State(gd)
    vel = [torch.empty_like(s.vors) for _ in range(3)]
    base = [torch.empty_like(s.vors) for _ in range(3)]
    ctx.swe_init(s.x, s.y, s.z, s.area, s.vors, s.divs, s.height, *vel, *base)
    assert rel(torch.stack(vel), gd["init_vel"]) <= FP64_TOL
    for k in range(3):
        assert rel(base[k], gd["init_base"][k]) <= FP64_TOL, k


@pytest.mark.parametrize("name", ["swe_L3.npz", "swe_L4_d2.npz", "swe_L3_direct.npz"])
def test_swe_step_matches_reference(sb, name):
    gd = load(name)
    ctx = golden_ctx(sb, gd)
    s = State(gd)
    ctx.swe_back_rk4_step_2(*s.args())
    assert rel(s.vors, gd["step_vors"]) <= FP64_TOL
    assert rel(s.divs, gd["step_divs"]) <= FP64_TOL
    assert rel(s.height, gd["step_height"]) <= FP64_TOL
    assert rel(torch.stack(s.vel), gd["step_vel"]) <= FP64_TOL
    if s.tr is not None:
        assert rel(s.tr, gd["step_tracers"]) <= FP64_TOL


def test_swe_step_with_zero_base_tendencies(sb):
    """Base tendencies of zero leave the full first-stage tendencies in the
    divergence and height updates (with the driver's base they cancel)."""
    gd = load("swe_L3.npz")
    ctx = golden_ctx(sb, gd)
    s = State(gd, base=np.zeros_like(gd["init_base"]))
    ctx.swe_back_rk4_step_2(*s.args())
    for k in ("vors", "divs", "height"):
        ref = gd[f"step0_{k}"]
        assert rel(getattr(s, k), ref) <= FP64_TOL, k
        # the update itself (a small change on a large field) also matches
        d0 = ref - gd[k]
        assert rel(getattr(s, k) - cuda(gd[k]), d0) <= 1e-9, k
    assert rel(torch.stack(s.vel), gd["step0_vel"]) <= FP64_TOL


@pytest.mark.parametrize("graph", [False, True])
def test_swe_driver_loop_two_steps(sb, graph):
    gd = load("swe_L3.npz")
    ctx = golden_ctx(sb, gd)
    s = State(gd)
    if graph:
        ctx.swe_run(*s.args(), nsteps=2)
    else:
        for _ in range(2):
            ctx.swe_back_rk4_step_2(*s.args())
            for f in (s.vors, s.divs, s.height):
                ctx.unify_boundary_vals(f)
    for k in ("vors", "divs", "height"):
        assert rel(getattr(s, k), gd[f"run2_{k}"]) <= FP64_TOL, k
    assert rel(torch.stack(s.vel), gd["run2_vel"]) <= FP64_TOL
    assert rel(s.tr, gd["run2_tracers"]) <= FP64_TOL


def test_swe_unit_sphere_twenty_steps_match_reference(sb):
    """The benchmark's steady geostrophic flow with height noise (time scaled
    to the reference's integer seconds), 20 driver steps.  The reference's
    forward-Euler divergence/height update amplifies grid-scale noise (by
    about 7% per step here), so roundoff differences grow with the steps:
    the tolerance is 1e-10 after 20 steps."""
    gd = load("swe_L4_unit.npz")
    ctx = golden_ctx(sb, gd)
    s = State(gd)
    base = [torch.empty_like(s.vors) for _ in range(3)]
    ctx.swe_init(s.x, s.y, s.z, s.area, s.vors, s.divs, s.height, *s.vel, *base)
    assert rel(torch.stack(base), gd["init_base"]) <= FP64_TOL
    s.base = base
    ctx.swe_run(*s.args(), nsteps=int(gd["nsteps"]))
    for k in ("vors", "divs", "height"):
        assert rel(getattr(s, k), gd[f"run_{k}"]) <= 1e-10, k
    assert rel(torch.stack(s.vel), gd["run_vel"]) <= 1e-10


def test_swe_tendencies_match_reference(sb):
    gd = load("swe_L3.npz")
    ctx = golden_ctx(sb, gd)
    s = State(gd)
    tv = cuda(gd["tend_vel"])
    out = [torch.empty_like(s.vors) for _ in range(3)]
    ctx.swe_tendencies(s.x, s.y, s.z, tv[0].contiguous(), tv[1].contiguous(), tv[2].contiguous(), s.vors, s.divs,
                       s.height, cuda(gd["tend_surface"]), *out)
    for k in range(3):
        assert rel(out[k], gd["tend_out"][k]) <= FP64_TOL, k


def test_swe_vel_interactions_match_reference(sb):
    gd = load("swe_L3.npz")
    ctx = golden_ctx(sb, gd)
    d = cuda(gd["vi_disp"])
    t = [torch.zeros(d.shape[1:], dtype=torch.float64, device="cuda") for _ in range(3)]
    ctx.swe_vel_interactions(d[0].contiguous(), d[1].contiguous(), d[2].contiguous(), cuda(gd["vi_src_vor"]),
                             cuda(gd["vi_src_div"]), *t)
    assert rel(torch.stack(t), gd["vi_out"]) <= FP64_TOL


def test_unify_is_bit_exact(sb):
    gd = load("swe_L3.npz")
    ctx = golden_ctx(sb, gd)
    f = cuda(gd["unify_in"])
    ctx.unify_boundary_vals(f)
    assert np.array_equal(f.cpu().numpy(), gd["unify_out"])


def test_swe_graph_replay_equals_steps(sb):
    gd = load("swe_L4_d2.npz")
    a, b = State(gd), State(gd)
    ctx_a, ctx_b = golden_ctx(sb, gd), golden_ctx(sb, gd)
    ctx_a.swe_run(*a.args(), nsteps=3)
    for _ in range(3):
        ctx_b.swe_back_rk4_step_2(*b.args())
        for f in (b.vors, b.divs, b.height):
            ctx_b.unify_boundary_vals(f)
    for k in ("vors", "divs", "height"):
        assert torch.equal(getattr(a, k), getattr(b, k)), k


def unit_sphere_state(sb, levels, precision, dt=0.002, seed=7, degree=3):
    """The steady geostrophic flow on the unit sphere (Omega = 2 pi, u0 = 2 pi/12,
    g h = 2.94 - (Omega u0 + u0^2/2) sin^2 lat, height holding g h, g/a = 1)
    with seeded N(0, 1e-4^2) noise on the height."""
    g = sb.build_grid(levels, degree, exact_cc=True)
    om, u0 = 2 * np.pi, 2 * np.pi / 12
    lat = np.arcsin(np.clip(g.z, -1, 1))
    vors = 2 * u0 * np.sin(lat)
    divs = np.zeros_like(vors)
    rng = np.random.default_rng(seed)
    height = 2.94 - (om * u0 + 0.5 * u0 * u0) * np.sin(lat) ** 2 + 1e-4 * rng.standard_normal(vors.shape)
    cfg = sb.config_default(levels=levels, interp_degree=degree, fmm_theta=0.7, kernel_eps=1e-4, omega=om, dt=dt,
                            precision=precision, g_over_a=1.0)
    ctx = sb.Context(cfg)
    gd = dict(x=g.x, y=g.y, z=g.z, area=g.area, vors=vors, divs=divs, height=height,
              init_base=np.zeros((3,) + vors.shape))
    s = State(gd)
    ctx.swe_init(s.x, s.y, s.z, s.area, s.vors, s.divs, s.height, *s.vel, *s.base)
    return ctx, s


def test_swe_mixed_close_to_fp64(sb):
    c64, s64 = unit_sphere_state(sb, 5, sb.FP64)
    c32, s32 = unit_sphere_state(sb, 5, sb.MIXED)
    c64.swe_run(*s64.args(), nsteps=5)
    c32.swe_run(*s32.args(), nsteps=5)
    assert rel(s32.vors, s64.vors) <= MIXED_TOL
    assert rel(s32.height, s64.height) <= MIXED_TOL


@pytest.mark.parametrize("degree", [2, 4])
def test_swe_mixed_close_to_fp64_other_degrees(sb, degree):
    """9 and 25 proxies per panel (odd counts) through the mixed two-field list
    kernel: within 1e-6 of float64 after 3 steps."""
    c64, s64 = unit_sphere_state(sb, 5, sb.FP64, degree=degree)
    c32, s32 = unit_sphere_state(sb, 5, sb.MIXED, degree=degree)
    c64.swe_run(*s64.args(), nsteps=3)
    c32.swe_run(*s32.args(), nsteps=3)
    assert rel(s32.vors, s64.vors) <= MIXED_TOL
    assert rel(s32.height, s64.height) <= MIXED_TOL


@pytest.mark.parametrize("precision,tol", [("FP64", FP64_TOL), ("MIXED", MIXED_TOL)])
def test_swe_steps_match_c_oracle_levels5(sb, port, precision, tol):
    """24,576 particles (beyond the golden fixtures), the benchmark's unit-sphere
    flow: one step, then two more of the driver's loop (step + unify), against
    the oracle's restatement on the same inputs and base tendencies.  The
    divergence of this balanced flow is the difference of nearly equal
    tendencies (a rounding-level field after the first step), so its error is
    measured on the vorticity's scale."""
    ctx, s = unit_sphere_state(sb, 5, getattr(sb, precision))
    g = port.build(5, 3, 0.7, exact_cc=True)
    host = lambda t: t.detach().cpu().numpy()
    assert np.array_equal(g["x"], host(s.x)) and np.array_equal(g["area"], host(s.area))
    smap, counts = sb.cubed_sphere_2d_to_1d(g["x"], g["y"], g["z"], 3)
    base = [host(b) for b in s.base]
    kw = dict(dt=0.002, omega=2 * np.pi, eps=1e-4, g_over_a=1.0)
    ov, od, oh, ovel, _ = port.swe_step(g, host(s.vors), host(s.divs), host(s.height), base, smap, counts, **kw)
    ctx.swe_back_rk4_step_2(*s.args())
    on_vor = lambda a, b: float(np.abs(host(a) - b).max() / np.abs(ov).max())
    errs = [rel(s.vors, ov), on_vor(s.divs, od), rel(s.height, oh), rel(torch.stack(s.vel), np.stack(ovel))]
    print(f"{precision} one step vs the C oracle: vorticity {errs[0]:.2e}, divergence {errs[1]:.2e}, "
          f"height {errs[2]:.2e}, velocity {errs[3]:.2e}")
    assert max(errs) <= tol
    for f in (s.vors, s.divs, s.height):
        ctx.unify_boundary_vals(f)
    ov, od, oh = (port.swe_unify(a, smap, counts) for a in (ov, od, oh))
    ctx.swe_run(*s.args(), nsteps=2)
    ov, od, oh, ovel, _ = port.swe_step(g, ov, od, oh, base, smap, counts, nsteps=2, driver_unify=True, **kw)
    assert rel(s.vors, ov) <= 10 * tol and rel(s.height, oh) <= 10 * tol and on_vor(s.divs, od) <= 10 * tol


def test_swe_steady_flow_stays_steady(sb):
    """Steady geostrophic flow: with the driver's base tendencies the height
    moves only by the noise's own evolution (L2 drift far below the noise)."""
    ctx, s = unit_sphere_state(sb, 5, sb.FP64)
    h0 = s.height.clone()
    ctx.swe_run(*s.args(), nsteps=20)
    w = s.area / s.area.sum()
    drift = float(torch.sqrt((w * (s.height - h0) ** 2).sum()) / torch.sqrt((w * h0 ** 2).sum()))
    assert drift < 1e-4, drift


def test_swe_nonfinite_input_reports_status(sb):
    gd = load("swe_L3.npz")
    ctx = golden_ctx(sb, gd)
    s = State(gd)
    s.vors[3, 5] = float("nan")
    with pytest.raises(sb.SbslpmError) as e:
        ctx.swe_back_rk4_step_2(*s.args())
    assert e.value.status in (3, 4)
    s2 = State(gd)  # the context stays usable
    ctx.swe_back_rk4_step_2(*s2.args())
    assert rel(s2.vors, gd["step_vors"]) <= FP64_TOL


def test_swe_needs_degree_two(sb):
    cfg = sb.config_default(levels=3, interp_degree=1)
    ctx = sb.Context(cfg)
    A, q = ctx.leaf_count, ctx.q
    z = torch.zeros(A, q, dtype=torch.float64, device="cuda")
    with pytest.raises(sb.SbslpmError):
        ctx.unify_boundary_vals(z)


@pytest.mark.parametrize("levels", [6, 7])
def test_height_drift_follows_the_reference(sb, levels):
    """The benchmark's SWE flow (steady geostrophic solid-body rotation with
    N(0, 1e-4^2) noise on g h, dt 0.002, spectral FMM at theta 0.7, exact
    Clenshaw-Curtis weights): the float64 path's relative L2 height drift
    every 10 steps against the reference's own step run to the same steps
    (tests/golden/swe_drift_reference_L<levels>.json, made by
    tests/golden/swe_drift_reference.py).  The reference's forward-Euler
    divergence and height update amplifies the noise until its point location
    meets a non-finite point, so both runs grow together; the drift values
    agree to 1e-8 relative while they are finite."""
    import json

    with open(os.path.join(GOLDEN, f"swe_drift_reference_L{levels}.json")) as f:
        ref = json.load(f)
    g = sb.build_grid(levels, 3, exact_cc=True)
    om, u0 = 2 * np.pi, 2 * np.pi / 12
    lat = np.arcsin(np.clip(g.z, -1, 1))
    h0 = 2.94 - (om * u0 + 0.5 * u0 * u0) * np.sin(lat) ** 2
    h0 = h0 + 1e-4 * np.random.default_rng(ref["noise_seed"]).standard_normal(h0.shape)
    ctx = sb.Context(sb.config_default(levels=levels, interp_degree=3, fmm_theta=ref["theta"],
                                       kernel_eps=ref["kernel_eps"], omega=om, dt=ref["dt"], g_over_a=1.0))
    f = [cuda(g.x), cuda(g.y), cuda(g.z), cuda(g.area), cuda(2 * u0 * np.sin(lat)), cuda(np.zeros_like(h0)),
         cuda(h0)]
    vel = [torch.zeros_like(f[0]) for _ in range(3)]
    base = [torch.zeros_like(f[0]) for _ in range(3)]
    ctx.swe_init(*f, *vel, *base)
    w = g.area / g.area.sum()
    l2 = lambda a: float(np.sqrt((w * a * a).sum()))
    done, checked = 0, 0
    for row in ref["curve"]:
        if row["height_l2_drift"] is None:
            break
        ctx.swe_run(*f, *vel, None, *base, nsteps=row["step"] - done)
        done = row["step"]
        d = l2(f[6].cpu().numpy() - h0) / l2(h0)
        print(f"levels {levels} step {done}: drift {d:.6e} (reference {row['height_l2_drift']:.6e})")
        assert abs(d - row["height_l2_drift"]) <= 1e-8 * row["height_l2_drift"]
        checked += 1
    assert checked >= 5
