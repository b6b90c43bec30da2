"""GPU parity tests of the BVE hot path, through the C ABI.

Checkers: the golden vectors made by the reference itself (tests/golden/) and
the C restatement oracle (oracle/), which is pinned to the reference bit for
bit by tests/test_oracle_golden.py.  Tolerances (relative L-infinity, scaled
by the largest reference magnitude):
  float64 path           <= 1e-12
  mixed-precision path   <= 1e-6 against the float64 path
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
                            tracer_count=int(gd["tracers_in"].shape[2]) if "tracers_in" in gd else 0, velocity=vel)
    for k, v in kw.items():
        setattr(cfg, k, v)
    return sb.Context(cfg)


def fields(gd):
    A, q = gd["x"].shape
    f = dict(x=cuda(gd["x"]), y=cuda(gd["y"]), z=cuda(gd["z"]), area=cuda(gd["area"]), vors=cuda(gd["ic_rh4"]))
    f["vel"] = [torch.zeros(A, q, dtype=torch.float64, device="cuda") for _ in range(3)]
    f["tr"] = cuda(gd["tracers_in"]) if "tracers_in" in gd else None
    return f


def step(ctx, f, n=1, graph=False):
    args = (f["x"], f["y"], f["z"], f["area"], f["vors"], *f["vel"], f["tr"])
    if graph:
        ctx.bve_run(*args, nsteps=n)
    else:
        for _ in range(n):
            ctx.bve_back_rk4_step(*args)


@pytest.mark.parametrize("name", ["bve_L3.npz", "bve_L3_direct.npz", "bve_L4_d2.npz"])
def test_step_matches_reference(sb, name):
    gd = load(name)
    ctx = golden_ctx(sb, gd)
    f = fields(gd)
    step(ctx, f)
    assert rel(f["vors"], gd["step1_vors"]) <= FP64_TOL
    assert rel(torch.stack(f["vel"]), gd["step1_vel"]) <= FP64_TOL
    if f["tr"] is not None:
        assert rel(f["tr"], gd["step1_tracers"]) <= FP64_TOL
    if "step2_vors" in gd:
        step(ctx, f)
        assert rel(f["vors"], gd["step2_vors"]) <= FP64_TOL
        assert rel(torch.stack(f["vel"]), gd["step2_vel"]) <= FP64_TOL
        assert rel(f["tr"], gd["step2_tracers"]) <= FP64_TOL


def test_graph_replay_equals_steps(sb):
    gd = load("bve_L3.npz")
    ctx = golden_ctx(sb, gd)
    f1, f2 = fields(gd), fields(gd)
    step(ctx, f1, 3)
    step(ctx, f2, 3, graph=True)
    assert torch.equal(f1["vors"], f2["vors"])
    assert torch.equal(f1["tr"], f2["tr"])
    assert all(torch.equal(a, b) for a, b in zip(f1["vel"], f2["vel"]))


def test_deterministic(sb):
    gd = load("bve_L4_d2.npz")
    ctx = golden_ctx(sb, gd)
    outs = []
    for _ in range(2):
        f = fields(gd)
        step(ctx, f, 2)
        outs.append(f["vors"].clone())
    assert torch.equal(outs[0], outs[1])


def test_upward_pass(sb):
    gd = load("bve_L3.npz")
    ctx = golden_ctx(sb, gd)
    out = torch.zeros(ctx.panel_count, ctx.q, dtype=torch.float64, device="cuda")
    ctx.upward_pass(cuda(gd["area"]), cuda(gd["up_pots"]), out)
    assert rel(out, gd["up_proxy"]) <= FP64_TOL


def test_vel_interactions(sb):
    gd = load("bve_L3.npz")
    ctx = golden_ctx(sb, gd)
    d = gd["vi_disp"]
    t = [torch.zeros(ctx.panel_count, ctx.q, dtype=torch.float64, device="cuda") for _ in range(3)]
    ctx.bve_vel_interactions(cuda(d[0]), cuda(d[1]), cuda(d[2]), cuda(gd["vi_src"]), *t)
    assert rel(torch.stack(t), gd["vi_out"]) <= FP64_TOL
    # accumulates into the targets, as the reference does
    ctx.bve_vel_interactions(cuda(d[0]), cuda(d[1]), cuda(d[2]), cuda(gd["vi_src"]), *t)
    assert rel(torch.stack(t), 2 * gd["vi_out"]) <= FP64_TOL


def test_downward_pass(sb):
    gd = load("bve_L3.npz")
    ctx = golden_ctx(sb, gd)
    t = [cuda(gd["down_in"][k]) for k in range(3)]
    s = [torch.zeros(ctx.leaf_count, ctx.q, dtype=torch.float64, device="cuda") for _ in range(3)]
    ctx.downward_pass_3(*t, *s)
    assert rel(torch.stack(s), gd["down_sols"]) <= FP64_TOL


def test_departure_and_remap(sb):
    gd = load("bve_L3.npz")
    ctx = golden_ctx(sb, gd)
    A, q = gd["x"].shape
    v = [cuda(gd["dep_vel"][k].reshape(3 * A, q)) for k in range(4)]
    dep = [torch.zeros(A, q, dtype=torch.float64, device="cuda") for _ in range(3)]
    ctx.bve_departure(cuda(gd["x"]), cuda(gd["y"]), cuda(gd["z"]), *v, 1.0, *dep)
    assert rel(torch.stack(dep), gd["dep_out"]) <= FP64_TOL
    nv = torch.zeros(A, q, dtype=torch.float64, device="cuda")
    ntr = torch.zeros_like(cuda(gd["tracers_in"]))
    ctx.bve_remap(cuda(gd["z"]), *[cuda(gd["dep_out"][k]) for k in range(3)], cuda(gd["remap_vors"]),
                  cuda(gd["tracers_in"]), nv, ntr)
    assert rel(nv, gd["remap_new_vors"]) <= FP64_TOL
    assert rel(ntr, gd["remap_new_tracers"]) <= FP64_TOL


def test_nonfinite_departure_is_reported(sb):
    """A NaN velocity makes point location fail; the kernel records it in the
    error word and the call returns SBSLPM_ERR_NONFINITE (no device trap)."""
    gd = load("bve_L3.npz")
    ctx = golden_ctx(sb, gd)
    A, q = gd["x"].shape
    v = [cuda(gd["dep_vel"][k].reshape(3 * A, q)) for k in range(4)]
    v[3][0, 0] = float("nan")
    dep = [torch.zeros(A, q, dtype=torch.float64, device="cuda") for _ in range(3)]
    with pytest.raises(sb.SbslpmError) as e:
        ctx.bve_departure(cuda(gd["x"]), cuda(gd["y"]), cuda(gd["z"]), *v, 1.0, *dep)
    assert e.value.status == 4
    # the context stays usable
    v[3][0, 0] = 0.0
    ctx.bve_departure(cuda(gd["x"]), cuda(gd["y"]), cuda(gd["z"]), *v, 1.0, *dep)
    assert rel(torch.stack(dep)[:, 1:], gd["dep_out"][:, 1:]) <= 1e-6


def test_inv_lap(sb):
    gd = load("inv_lap.npz")
    xyz = gd["xyz"]
    soln = torch.zeros(len(xyz), dtype=torch.float64, device="cuda")
    sb.direct_sum_inv_lap(*[cuda(xyz[:, i]) for i in range(3)], cuda(gd["area"]), cuda(gd["pots"]), soln)
    assert rel(soln, gd["soln"]) <= FP64_TOL


def numpy_bve_direct(t, s, w, eps):
    d = s[None, :, :] - t[:, None, :]
    r2 = (d * d).sum(-1)
    g = np.where(r2 > 0, w[None, :] / (0.5 * r2 + eps), 0.0)
    a = (g[:, :, None] * d).sum(1)
    return -0.07957747154594767 * np.cross(t, a)


def test_direct_sum_bve(sb):
    rng = np.random.default_rng(7)
    t = rng.standard_normal((1500, 3))
    t /= np.linalg.norm(t, axis=1, keepdims=True)
    s = rng.standard_normal((2100, 3))
    s /= np.linalg.norm(s, axis=1, keepdims=True)
    s[:10] = t[:10]  # coincident pairs contribute nothing
    w = rng.standard_normal(2100) * 1e-3
    want = numpy_bve_direct(t, s, w, 1e-4)
    args = [cuda(t[:, i]) for i in range(3)] + [cuda(s[:, i]) for i in range(3)] + [cuda(w)]
    got = torch.stack(sb.direct_sum_bve(*args, 1e-4, sb.FP64), dim=1)
    assert rel(got, want) <= FP64_TOL
    got32 = torch.stack(sb.direct_sum_bve(*args, 1e-4, sb.MIXED), dim=1)
    assert rel(got32, want) <= 1e-5


def unit_sphere_rh4(g):
    """Rossby-Haurwitz R=4 vorticity, omega0 = K = 0.5, minus its mean."""
    lat = np.arcsin(np.clip(g.z, -1, 1))
    lon = np.arctan2(g.y, g.x)
    R = 4
    vor = 2 * 0.5 * np.sin(lat) - 0.5 * np.sin(lat) * np.cos(lat) ** 4 * (R * R + 3 * R + 2) * np.cos(R * lon)
    return vor - (vor * g.area).sum() / (4 * np.pi)


def unit_ctx(sb, levels, **kw):
    cfg = sb.config_default(levels=levels, interp_degree=3, fmm_theta=0.7, kernel_eps=1e-4, omega=2 * np.pi,
                            dt=0.005, **kw)
    return sb.Context(cfg)


def unit_fields(g, vor):
    A, q = g.x.shape
    return dict(x=cuda(g.x), y=cuda(g.y), z=cuda(g.z), area=cuda(g.area), vors=cuda(vor),
                vel=[torch.zeros(A, q, dtype=torch.float64, device="cuda") for _ in range(3)], tr=None)


def test_fmm_step_matches_oracle_levels5(sb, port):
    """6 x 16 x 16 panels x 16 points (24,576 particles), unit sphere, dt=0.005:
    the float64 FMM step against the C oracle at the same size."""
    g = sb.build_grid(5, 3, exact_cc=True)
    vor = unit_sphere_rh4(g)
    og = port.build(5, 3, 0.7, exact_cc=True)
    ov, ovel, _ = port.bve_step(og, vor, None, dt=0.005, omega=2 * np.pi, eps=1e-4, mode=0)
    f = unit_fields(g, vor)
    step(unit_ctx(sb, 5), f)
    assert rel(torch.stack(f["vel"]), np.stack(ovel)) <= FP64_TOL
    assert rel(f["vors"], ov) <= FP64_TOL


def test_mixed_matches_fp64_levels6(sb):
    """98,304 particles: the mixed-precision step within 1e-6 of float64."""
    g = sb.build_grid(6, 3, exact_cc=True)
    vor = unit_sphere_rh4(g)
    f64, f32 = unit_fields(g, vor), unit_fields(g, vor)
    step(unit_ctx(sb, 6), f64, 2)
    step(unit_ctx(sb, 6, precision=sb.MIXED), f32, 2)
    assert rel(torch.stack(f32["vel"]), torch.stack(f64["vel"])) <= MIXED_TOL
    assert rel(f32["vors"], f64["vors"]) <= MIXED_TOL


@pytest.mark.parametrize("degree", [1, 2, 4])
def test_mixed_list_kernel_other_degrees(sb, degree):
    """The reference's FMM at interp degrees 1, 2 and 4 (4, 9 and 25 proxies:
    the mixed list kernel's pair staging with even and odd proxy counts, the
    odd one padded by a zero-strength partner): within 1e-6 of float64."""
    g = sb.build_grid(5, degree, exact_cc=True)
    vor = unit_sphere_rh4(g)
    out = {}
    for prec in (sb.FP64, sb.MIXED):
        cfg = sb.config_default(levels=5, interp_degree=degree, fmm_theta=0.7, kernel_eps=1e-4, omega=2 * np.pi,
                                dt=0.005, precision=prec)
        f = unit_fields(g, vor)
        step(sb.Context(cfg), f, 2)
        out[prec] = f
    assert rel(torch.stack(out[sb.MIXED]["vel"]), torch.stack(out[sb.FP64]["vel"])) <= MIXED_TOL
    assert rel(out[sb.MIXED]["vors"], out[sb.FP64]["vors"]) <= MIXED_TOL


@pytest.mark.parametrize("n", [2, 3, 4])
def test_treecode_mixed_low_proxy_degrees(sb, n):
    """Treecode proxies of degree 2, 3, 4 (9, 16, 25 per panel) run the
    well-separated list through the q <= 32 mixed list kernels (entry table
    of the tree's list): within 1e-6 of the float64 treecode of the same
    degree."""
    g = sb.build_grid(5, 3, exact_cc=True)
    vor = unit_sphere_rh4(g)
    f64, f32 = unit_fields(g, vor), unit_fields(g, vor)
    step(tree_ctx(sb, 5, n, leaf=64), f64)
    step(tree_ctx(sb, 5, n, precision=sb.MIXED, leaf=64), f32)
    assert rel(torch.stack(f32["vel"]), torch.stack(f64["vel"])) <= MIXED_TOL
    assert rel(f32["vors"], f64["vors"]) <= MIXED_TOL


def test_direct_mode_matches_oracle_levels4(sb, port):
    g = sb.build_grid(4, 3, exact_cc=True)
    vor = unit_sphere_rh4(g)
    og = port.build(4, 3, None, exact_cc=True)
    ov, ovel, _ = port.bve_step(og, vor, None, dt=0.005, omega=2 * np.pi, eps=1e-4, mode=1)
    for prec, tol in ((sb.FP64, FP64_TOL), (sb.MIXED, MIXED_TOL)):
        f = unit_fields(g, vor)
        step(unit_ctx(sb, 4, velocity=sb.VEL_DIRECT, precision=prec), f)
        assert rel(torch.stack(f["vel"]), np.stack(ovel)) <= tol
        assert rel(f["vors"], ov) <= tol


def test_solid_body_rotation_levels7(sb):
    """393,216 particles: solid-body rotation (vorticity 2 a z) stays steady
    and its velocity is a (z_hat x x), for both precisions."""
    g = sb.build_grid(7, 3, exact_cc=True)
    a = 0.25
    vor = 2 * a * g.z
    for prec in (sb.FP64, sb.MIXED):
        f = unit_fields(g, vor)
        step(unit_ctx(sb, 7, precision=prec), f)
        assert rel(f["vors"], vor) < 1e-4
        u = torch.stack(f["vel"]).cpu().numpy()
        assert np.abs(u[0] + a * g.y).max() / a < 1e-2
        assert np.abs(u[1] - a * g.x).max() / a < 1e-2


def tree_ctx(sb, levels, n, precision=0, theta=0.7, leaf=256):
    cfg = sb.config_default(levels=levels, interp_degree=3, fmm_theta=theta, kernel_eps=1e-4, omega=2 * np.pi,
                            dt=0.005, proxy_degree=n, leaf_size=leaf, precision=precision)
    return sb.Context(cfg)


def one_step(ctx, g, vor):
    f = unit_fields(g, vor)
    step(ctx, f)
    return f


@pytest.fixture(scope="module")
def direct_l5(sb):
    g = sb.build_grid(5, 3, exact_cc=True)
    vor = unit_sphere_rh4(g)
    return g, vor, one_step(unit_ctx(sb, 5, velocity=sb.VEL_DIRECT), g, vor)


def test_treecode_matches_direct_sum_levels5(sb, direct_l5):
    """24,576 particles, degree-8 proxies on 256-particle leaves, theta 0.7:
    within 1e-6 (vorticity) of the float64 direct sum after one step."""
    g, vor, fd = direct_l5
    ft = one_step(tree_ctx(sb, 5, 8), g, vor)
    ev = rel(torch.stack(ft["vel"]), torch.stack(fd["vel"]))
    ew = rel(ft["vors"], fd["vors"])
    print(f"treecode n=8: rel vel err {ev:.3e}, rel vort err {ew:.3e}")
    assert ew <= 1e-6
    assert ev <= 1e-4


def test_treecode_error_falls_with_degree(sb, direct_l5):
    g, vor, fd = direct_l5
    errs = []
    for n in (2, 4, 6, 8):
        ft = one_step(tree_ctx(sb, 5, n), g, vor)
        errs.append(rel(torch.stack(ft["vel"]), torch.stack(fd["vel"])))
    print("treecode velocity error by degree 2,4,6,8:", errs)
    assert errs[0] > errs[1] > errs[2] > errs[3]


def test_treecode_mixed_matches_fp64_levels6(sb):
    g = sb.build_grid(6, 3, exact_cc=True)
    vor = unit_sphere_rh4(g)
    f64 = one_step(tree_ctx(sb, 6, 8), g, vor)
    f32 = one_step(tree_ctx(sb, 6, 8, precision=sb.MIXED), g, vor)
    assert rel(torch.stack(f32["vel"]), torch.stack(f64["vel"])) <= MIXED_TOL
    assert rel(f32["vors"], f64["vors"]) <= MIXED_TOL


def test_treecode_graph_replay_and_determinism(sb):
    g = sb.build_grid(5, 3, exact_cc=True)
    vor = unit_sphere_rh4(g)
    ctx = tree_ctx(sb, 5, 6, precision=sb.MIXED)
    a, b = unit_fields(g, vor), unit_fields(g, vor)
    step(ctx, a, 2)
    step(ctx, b, 2, graph=True)
    assert torch.equal(a["vors"], b["vors"])


@pytest.mark.parametrize("case", ["ssw_ramp", "ssw2_plateau", "ssw_down"])
def test_forced_step_matches_reference(sb, case):
    """The SSW forcing (src/forcing_funcs.cpp:6-96) in the step, eager steps
    from the case's time and one graph-replayed run, against the reference.
    Tolerance 1e-11: the forcing term's tan / exp / atan2 / cos run in the
    device's libm (last-bit differences from the host's), and the forced
    flow is strong (the forcing moves the vorticity by 2.5 in one step)."""
    gd = load("bve_forcing_L3.npz")
    cfg = sb.config_default(levels=3, interp_degree=3, fmm_theta=0.7, kernel_eps=float(gd["eps"]),
                            omega=float(gd["omega"]), dt=1.0, forcing=int(gd[case + "_forcing"]))
    ctx = sb.Context(cfg)
    n, t0 = int(gd[case + "_n"]), float(gd[case + "_t0"])
    xyza = [cuda(gd[k]) for k in ("x", "y", "z", "area")]
    v = cuda(gd["ic"])
    vel = [torch.zeros_like(v) for _ in range(3)]
    for k in range(n):
        ctx.bve_back_rk4_step(*xyza, v, *vel, time=t0 + k)
    assert rel(v, gd[case + "_vors"]) <= 1e-11, rel(v, gd[case + "_vors"])
    assert rel(torch.stack(vel), gd[case + "_vel"]) <= 1e-11
    w = cuda(gd["ic"])
    wel = [torch.zeros_like(w) for _ in range(3)]
    ctx.bve_run(*xyza, w, *wel, nsteps=n, time=t0)
    assert torch.equal(w, v) and all(torch.equal(a, b) for a, b in zip(wel, vel))


def test_forcing_on_treecode_and_mixed(sb):
    """The forcing through the other velocity paths, at the benchmark's time
    step (dt 0.005; the golden case's dt = 1 turns the flow too far per step
    for the mixed-precision bar): mixed spectral FMM against the float64 one
    <= 1e-6, treecode and spectral FMM against the forced float64 direct sum."""
    g = sb.build_grid(4, 3, exact_cc=True)
    xyza = [cuda(a) for a in (g.x, g.y, g.z, g.area)]
    lat = np.arcsin(np.clip(g.z, -1, 1))
    vor0 = 2 * 0.5 * np.sin(lat) - 0.5 * np.sin(lat) * np.cos(lat) ** 4 * 30 * np.cos(4 * np.arctan2(g.y, g.x))
    out = {}
    for name, kw in (("direct", dict(velocity=sb.VEL_DIRECT)), ("fp64", {}), ("mixed", dict(precision=sb.MIXED)),
                     ("tree", dict(proxy_degree=8, leaf_size=64))):
        cfg = sb.config_default(levels=4, interp_degree=3, fmm_theta=0.7, kernel_eps=1e-4, omega=2 * np.pi,
                                dt=0.005, forcing=sb.FORCING_SSW2, **kw)
        ctx = sb.Context(cfg)
        v = cuda(vor0)
        vel = [torch.zeros_like(v) for _ in range(3)]
        ctx.bve_back_rk4_step(*xyza, v, *vel, time=6 * 86400.0)
        out[name] = v
    unforced = sb.Context(sb.config_default(levels=4, interp_degree=3, kernel_eps=1e-4, omega=2 * np.pi, dt=0.005,
                                            velocity=sb.VEL_DIRECT))
    u = cuda(vor0)
    unforced.bve_back_rk4_step(*xyza, u, *[torch.zeros_like(u) for _ in range(3)])
    assert rel(u, out["direct"].cpu().numpy()) > 1e-3  # the forcing acts
    assert rel(out["mixed"], out["fp64"].cpu().numpy()) <= MIXED_TOL
    assert rel(out["tree"], out["direct"].cpu().numpy()) <= 1e-7
    assert rel(out["fp64"], out["direct"].cpu().numpy()) <= 1e-4  # the spectral FMM's own error at theta 0.7
