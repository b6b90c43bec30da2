"""The treecode (decoupled proxy degree) against the oracle, through the C ABI.

Checkers (oracle/bslpm_oracle.c, pinned to the reference by
tests/test_oracle_bltc.py and tests/test_oracle_golden.py):
  * the oracle's treecode step (mode 2) with every well-separated pair proxy
    x proxy -- this library's design, built from the reference's
    irregular-point FMM functions (base_pots_ll, child_to_parent_ll,
    dual_tree_traversal_irreg, swe_vel_panel_interaction_ll,
    parent_to_child_3_ll, child_panel_interp_3_ll): the float64 GPU step must
    agree to 1e-12, the mixed-precision step to 1e-6;
  * the oracle's float64 direct-sum step (mode 1): the metric's bar, 1e-6
    relative L-infinity vorticity error after one step;
  * the oracle's treecode with the reference's pp / pc / cp / cc typing
    (typed = 1, the reference's own arithmetic at equal theta, proxy degree
    and leaf size): the GPU treecode's error against the direct sum must not
    exceed twice that error (plus the float32 rounding for mixed).
Plus the headline configuration itself (393,216 particles, theta 0.7,
degree-8 proxies, 256-particle leaves): one step within 1e-6 of the float64
direct sum, which is pinned to the oracle at 24,576 particles.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

FP64_TOL = 1e-12
MIXED_TOL = 1e-6
BAR = 1e-6
DT, OMEGA, EPS = 0.005, 2 * np.pi, 1e-4


def rel(a, b):
    a = a.detach().cpu().numpy() if hasattr(a, "detach") else np.asarray(a)
    b = b.detach().cpu().numpy() if hasattr(b, "detach") else np.asarray(b)
    return float(np.abs(a - b).max() / np.abs(b).max())


def cuda(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def rh4(x, y, z, area):
    lat, lon = np.arcsin(np.clip(z, -1, 1)), np.arctan2(y, x)
    vor = np.sin(lat) - 0.5 * np.sin(lat) * np.cos(lat) ** 4 * 30 * np.cos(4 * lon)
    return vor - (vor * area).sum() / (4 * np.pi)


def gpu_step(sb, g, vor, near_form=None, **kw):
    cfg = sb.config_default(levels=kw.pop("levels"), interp_degree=3, kernel_eps=EPS, omega=OMEGA, dt=DT, **kw)
    ctx = sb.Context(cfg)
    if near_form is not None:
        ctx.set_near_form(near_form)
    v = cuda(vor)
    vel = [torch.zeros_like(v) for _ in range(3)]
    ctx.bve_back_rk4_step(cuda(g.x), cuda(g.y), cuda(g.z), cuda(g.area), v, *vel)
    return v, torch.stack(vel)


@pytest.fixture(scope="module")
def grid5(sb, port):
    g = sb.build_grid(5, 3, exact_cc=True)
    og = port.build(5, 3, None, exact_cc=True)
    assert np.array_equal(og["x"], g.x) and np.array_equal(og["area"], g.area)
    vor = rh4(g.x, g.y, g.z, g.area)
    dv, dvel, _ = port.bve_step(og, vor, None, dt=DT, omega=OMEGA, eps=EPS, mode=1)
    return g, og, vor, dv, np.stack(dvel)


# (levels, leaf size, proxy degree, theta): the headline geometry at 24,576
# particles, the ensemble's (theta, degree) pairs, a deeper tree of 64-particle
# leaves, and leaves that are single grid panels
CASES = [(5, 256, 8, 0.7), (5, 256, 6, 0.5), (5, 256, 10, 0.8), (4, 64, 8, 0.7), (4, 16, 5, 0.6)]


@pytest.mark.parametrize("levels,leaf,n,theta", CASES)
def test_treecode_step_matches_oracle(sb, port, levels, leaf, n, theta):
    g = sb.build_grid(levels, 3, exact_cc=True)
    og = port.build(levels, 3, None, exact_cc=True)
    vor = rh4(g.x, g.y, g.z, g.area)
    ov, ovel, _ = port.bve_step(og, vor, None, dt=DT, omega=OMEGA, eps=EPS, mode=2, tree=(n, leaf, theta, 0))
    ovel = np.stack(ovel)
    for prec, tol in ((sb.FP64, FP64_TOL), (sb.MIXED, MIXED_TOL)):
        v, vel = gpu_step(sb, g, vor, levels=levels, fmm_theta=theta, proxy_degree=n, leaf_size=leaf,
                          precision=prec)
        assert rel(vel, ovel) <= tol, (prec, rel(vel, ovel))
        assert rel(v, ov) <= tol, (prec, rel(v, ov))


def test_treecode_step_with_tracers_matches_oracle(sb, port, grid5):
    """Two passive tracers carried by a treecode step (the remap of
    bve_departure_to_target at the treecode's departure points) against the
    oracle's treecode step with the same tracers."""
    g, og, vor, _, _ = grid5
    tr = np.ascontiguousarray(np.stack([g.z, g.x * g.y], axis=2))
    ov, _, otr = port.bve_step(og, vor, tr, dt=DT, omega=OMEGA, eps=EPS, mode=2, tree=(8, 256, 0.7, 0))
    for prec, tol in ((sb.FP64, FP64_TOL), (sb.MIXED, MIXED_TOL)):
        cfg = sb.config_default(levels=5, interp_degree=3, kernel_eps=EPS, omega=OMEGA, dt=DT, fmm_theta=0.7,
                                proxy_degree=8, leaf_size=256, precision=prec, tracer_count=2)
        ctx = sb.Context(cfg)
        v, t = cuda(vor), cuda(tr)
        vel = [torch.zeros_like(v) for _ in range(3)]
        ctx.bve_back_rk4_step(cuda(g.x), cuda(g.y), cuda(g.z), cuda(g.area), v, *vel, t)
        assert rel(v, ov) <= tol, prec
        assert rel(t, otr) <= tol, prec


@pytest.mark.parametrize("n,theta", [(8, 0.7), (6, 0.5), (10, 0.8)])
def test_treecode_error_against_the_direct_sum(sb, port, grid5, n, theta):
    """Vorticity after one step within the bar of the oracle's float64 direct
    sum, and no further from it than the reference's typed treecode."""
    g, og, vor, dv, dvel = grid5
    rv, _, _ = port.bve_step(og, vor, None, dt=DT, omega=OMEGA, eps=EPS, mode=2, tree=(n, 256, theta, 1))
    ref_err = rel(rv, dv)
    for prec, slack in ((sb.FP64, 1e-12), (sb.MIXED, 1e-8)):
        v, vel = gpu_step(sb, g, vor, levels=5, fmm_theta=theta, proxy_degree=n, leaf_size=256, precision=prec)
        err = rel(v, dv)
        print(f"n={n} theta={theta} prec={prec}: vorticity error {err:.3e} (reference typing {ref_err:.3e}), "
              f"velocity error {rel(vel, dvel):.3e}")
        assert err <= BAR
        assert err <= 2 * ref_err + slack


@pytest.mark.parametrize("levels,leaf,n,theta", [(6, 256, 8, 0.7), (6, 64, 8, 0.7)])
def test_expanded_near_form_matches_oracle(sb, port, levels, leaf, n, theta):
    """The mixed near field in the expanded pair form (8 float32 operations per
    pair: the denominator as (|s|^2 + eps) + |b|^2 + 2 b.s about the source
    leaf's centre), which set-up chooses at 98,304 particles: within the
    mixed-precision bar of the oracle's treecode, and of the difference
    form."""
    g = sb.build_grid(levels, 3, exact_cc=True)
    og = port.build(levels, 3, None, exact_cc=True)
    vor = rh4(g.x, g.y, g.z, g.area)
    ov, ovel, _ = port.bve_step(og, vor, None, dt=DT, omega=OMEGA, eps=EPS, mode=2, tree=(n, leaf, theta, 0))
    ovel = np.stack(ovel)
    kw = dict(levels=levels, fmm_theta=theta, proxy_degree=n, leaf_size=leaf, precision=sb.MIXED)
    v1, vel1 = gpu_step(sb, g, vor, **kw)  # set-up's choice: the expanded form
    v0, vel0 = gpu_step(sb, g, vor, near_form=False, **kw)
    print(f"levels {levels} leaf {leaf}: expanded vs oracle velocity {rel(vel1, ovel):.2e}, vorticity "
          f"{rel(v1, ov):.2e}; difference form {rel(vel0, ovel):.2e}, {rel(v0, ov):.2e}")
    assert rel(vel1, ovel) <= MIXED_TOL and rel(v1, ov) <= MIXED_TOL
    assert rel(vel1, vel0) <= MIXED_TOL and rel(v1, v0) <= MIXED_TOL


def test_near_form_chosen_at_set_up(sb):
    """Set-up keeps the difference form where eps does not dominate the
    expanded form's rounding (256-particle leaves at 24,576 particles) and
    takes the expanded one at the headline size; float64 never uses it, and
    eps = 0 refuses it."""
    def ctx(levels, **kw):
        return sb.Context(sb.config_default(levels=levels, interp_degree=3, omega=OMEGA, dt=DT, fmm_theta=0.7,
                                            proxy_degree=8, leaf_size=256, **kw))
    assert not ctx(5, kernel_eps=EPS, precision=sb.MIXED).near_form()
    assert ctx(6, kernel_eps=EPS, precision=sb.MIXED).near_form()
    assert ctx(7, kernel_eps=EPS, precision=sb.MIXED).near_form()
    assert not ctx(7, kernel_eps=EPS, precision=sb.FP64).near_form()
    assert not ctx(7, kernel_eps=0.0, precision=sb.MIXED).near_form()
    with pytest.raises(sb.SbslpmError):
        ctx(5, kernel_eps=0.0, precision=sb.MIXED).set_near_form(True)
    with pytest.raises(sb.SbslpmError):
        ctx(5, kernel_eps=EPS, precision=sb.FP64).set_near_form(True)


def test_headline_configuration_meets_the_bar(sb):
    """393,216 particles, theta 0.7, degree-8 proxies, 256-particle leaves:
    the mixed (both near-field pair forms) and float64 treecode steps within
    1e-6 (vorticity) of the float64 direct sum."""
    g = sb.build_grid(7, 3, exact_cc=True)
    vor = rh4(g.x, g.y, g.z, g.area)
    dv, dvel = gpu_step(sb, g, vor, levels=7, velocity=sb.VEL_DIRECT)
    for prec, form in ((sb.MIXED, True), (sb.MIXED, False), (sb.FP64, None)):
        v, vel = gpu_step(sb, g, vor, near_form=form, levels=7, fmm_theta=0.7, proxy_degree=8, leaf_size=256,
                          precision=prec)
        print(f"levels 7 prec={prec} expanded={form}: vorticity error {rel(v, dv):.3e}, "
              f"velocity error {rel(vel, dvel):.3e}")
        assert rel(v, dv) <= BAR


@pytest.mark.parametrize("levels", [5, 6])
def test_two_sided_first_stage_near_field(sb, port, levels):
    """The first stage's near field evaluated once per unordered leaf pair for
    both directions (sbslpm_set_near_mutual): the same step within the
    mixed-precision bar of the oracle's treecode and of the one-sided kernel,
    and deterministic."""
    g = sb.build_grid(levels, 3, exact_cc=True)
    vor = rh4(g.x, g.y, g.z, g.area)
    out = {}
    for on in (False, True, True):
        cfg = sb.config_default(levels=levels, interp_degree=3, kernel_eps=EPS, omega=OMEGA, dt=DT, fmm_theta=0.7,
                                proxy_degree=8, leaf_size=256, precision=sb.MIXED)
        ctx = sb.Context(cfg)
        ctx.set_near_tuning(128, 2, 4)
        ctx.set_near_mutual(on)
        assert ctx.near_mutual()[0] == on
        v = cuda(vor)
        vel = [torch.zeros_like(v) for _ in range(3)]
        ctx.bve_back_rk4_step(cuda(g.x), cuda(g.y), cuda(g.z), cuda(g.area), v, *vel)
        if on in out:
            assert torch.equal(v, out[on][0]) and torch.equal(torch.stack(vel), out[on][1])
        out[on] = (v, torch.stack(vel))
    assert rel(out[True][1], out[False][1]) <= MIXED_TOL
    assert rel(out[True][0], out[False][0]) <= MIXED_TOL
    if levels == 5:
        og = port.build(levels, 3, None, exact_cc=True)
        ov, ovel, _ = port.bve_step(og, vor, None, dt=DT, omega=OMEGA, eps=EPS, mode=2, tree=(8, 256, 0.7, 0))
        assert rel(out[True][1], np.stack(ovel)) <= MIXED_TOL
        assert rel(out[True][0], ov) <= MIXED_TOL


def test_two_sided_kernel_refused_where_it_does_not_apply(sb):
    for kw in (dict(precision=sb.FP64, leaf_size=256), dict(precision=sb.MIXED, leaf_size=64)):
        cfg = sb.config_default(levels=5, interp_degree=3, kernel_eps=EPS, omega=OMEGA, dt=DT, fmm_theta=0.7,
                                proxy_degree=8, **kw)
        ctx = sb.Context(cfg)
        with pytest.raises(sb.SbslpmError):
            ctx.set_near_mutual(True)
