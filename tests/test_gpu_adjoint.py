"""GPU tests of the hand-written adjoint: the Biot-Savart direct-sum VJP, one
reverse BVE step, and the gradient of a 20-step loss through the
torch.autograd.Function with per-step checkpoints, all against central
finite differences.

Tolerances: VJP dot-product test <= 1e-7 relative; one reverse step <= 1e-6;
the 20-step gradient <= 1e-5 in every one of 64 seeded directions (h = 1e-6),
the error of direction k measured relative to the root-mean-square
directional derivative over the 64 directions: a random direction can be
nearly orthogonal to the gradient (one of the 64 has a derivative 260 times
below the typical one), where the error relative to its own derivative says
nothing about the gradient.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def sphere_points(rng, n):
    p = rng.standard_normal((n, 3))
    p /= np.linalg.norm(p, axis=1, keepdims=True)
    return [torch.from_numpy(np.ascontiguousarray(p[:, k])).cuda() for k in range(3)]


def test_direct_sum_vjp_dot_product(sb):
    rng = np.random.default_rng(11)
    tx, ty, tz = sphere_points(rng, 700)
    sx, sy, sz = sphere_points(rng, 500)
    q = torch.from_numpy(rng.standard_normal(500)).cuda()
    ubar = [torch.from_numpy(rng.standard_normal(700)).cuda() for _ in range(3)]
    qb, (xb, yb, zb) = sb.direct_sum_bve_vjp(tx, ty, tz, ubar, sx, sy, sz, q, 1e-4)
    for seed in range(3):
        r = np.random.default_rng(100 + seed)
        dq, dx, dy, dz = (torch.from_numpy(r.standard_normal(500)).cuda() for _ in range(4))
        h = 1e-6

        def f(s):
            u = sb.direct_sum_bve(tx, ty, tz, sx + s * dx, sy + s * dy, sz + s * dz, q + s * dq, 1e-4)
            return sum(float((ubar[k] * u[k]).sum()) for k in range(3))

        fd = (f(h) - f(-h)) / (2 * h)
        ad = float((qb * dq).sum() + (xb * dx).sum() + (yb * dy).sum() + (zb * dz).sum())
        assert abs(fd - ad) <= 1e-7 * abs(ad), (fd, ad)


def test_direct_sum_autograd_gradcheck(sb):
    rng = np.random.default_rng(5)
    tx, ty, tz = sphere_points(rng, 12)
    sx, sy, sz = (t.clone().requires_grad_() for t in sphere_points(rng, 9))
    q = torch.from_numpy(rng.standard_normal(9)).cuda().requires_grad_()
    fn = lambda a, b, c, d: sb.direct_sum_bve_autograd(tx, ty, tz, a, b, c, d, 1e-2)
    assert torch.autograd.gradcheck(fn, (sx, sy, sz, q), eps=1e-6, atol=1e-7, rtol=1e-6)


def gaussian_vortex_state(sb, levels, dt, noise, seed=3):
    g = sb.build_grid(levels, 3, exact_cc=True)
    lat0, lon0 = np.deg2rad(30.0), 0.0
    c = np.array([np.cos(lat0) * np.cos(lon0), np.cos(lat0) * np.sin(lon0), np.sin(lat0)])
    r2 = (g.x - c[0]) ** 2 + (g.y - c[1]) ** 2 + (g.z - c[2]) ** 2
    w0 = np.exp(-r2 / (2 * 0.15 ** 2))
    wn = w0 + noise * np.random.default_rng(seed).standard_normal(w0.shape)
    cfg = sb.config_default(levels=levels, interp_degree=3, kernel_eps=1e-4, omega=2 * np.pi, dt=dt,
                            velocity=sb.VEL_DIRECT, precision=sb.FP64)
    ctx = sb.Context(cfg)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    return ctx, [T(g.x), T(g.y), T(g.z), T(g.area)], T(w0), T(wn)


def test_adjoint_step_dot_product(sb):
    ctx, f, w0, wn = gaussian_vortex_state(sb, 4, 0.01, 1e-2)
    rng = np.random.default_rng(8)
    wbar_next = torch.from_numpy(rng.standard_normal(tuple(wn.shape))).cuda()
    wbar = torch.empty_like(wn)
    ctx.bve_adjoint_step(*f, wn, wbar_next, wbar)

    def step(w):
        v = w.clone()
        vel = [torch.zeros_like(v) for _ in range(3)]
        ctx.bve_back_rk4_step(*f, v, *vel)
        return v

    for seed in range(3):
        d = torch.from_numpy(np.random.default_rng(50 + seed).standard_normal(tuple(wn.shape))).cuda()
        h = 1e-6
        fd = float((wbar_next * (step(wn + h * d) - step(wn - h * d))).sum()) / (2 * h)
        ad = float((wbar * d).sum())
        assert abs(fd - ad) <= 1e-6 * abs(ad), (seed, fd, ad)


def test_twenty_step_gradient_matches_finite_differences(sb):
    """The adjoint configuration: 24,576 particles, Gaussian vortex at 30N 0E
    (sigma 0.15) plus N(0, 1e-2^2) noise, J = 1/2 sum w (w(T) - w*(T))^2 with
    w* the run from the noiseless state and w the quadrature weights, 20 steps
    of dt = 0.01, gradient through the checkpointed adjoint, 64 central
    differences with h = 1e-6."""
    ctx, f, w0, wn = gaussian_vortex_state(sb, 5, 0.01, 1e-2)
    nsteps = 20
    area = f[3]

    def run(w):
        v = w.clone()
        vel = [torch.zeros_like(v) for _ in range(3)]
        ctx.bve_run(*f, v, *vel, nsteps=nsteps)
        return v

    wstar = run(w0)

    def J(w):
        return 0.5 * float((area * (run(w) - wstar) ** 2).sum())

    x = wn.clone().requires_grad_()
    out = sb.bve_rollout(ctx, *f, x, nsteps)
    loss = 0.5 * (area * (out - wstar) ** 2).sum()
    loss.backward()
    grad = x.grad
    assert abs(float(loss.detach()) - J(wn)) <= 1e-12 * abs(float(loss.detach()))
    h = 1e-6
    fds, ads = [], []
    for k in range(64):
        d = torch.from_numpy(np.random.default_rng(1000 + k).standard_normal(tuple(wn.shape))).cuda()
        fds.append((J(wn + h * d) - J(wn - h * d)) / (2 * h))
        ads.append(float((grad * d).sum()))
    fds, ads = np.array(fds), np.array(ads)
    rms = np.sqrt((ads ** 2).mean())
    errs = np.abs(fds - ads) / rms
    print("FD errors / rms derivative: median %.2e max %.2e" % (np.median(errs), errs.max()))
    assert errs.max() <= 1e-5, errs
    # and relative to its own derivative wherever that is not near zero
    big = np.abs(ads) >= 0.1 * rms
    assert big.sum() >= 56 and (np.abs(fds - ads)[big] / np.abs(ads[big])).max() <= 1e-5


def tree_ctx(sb, levels, dt, theta=0.7, degree=8, precision=None):
    cfg = sb.config_default(levels=levels, interp_degree=3, kernel_eps=1e-4, omega=2 * np.pi, dt=dt,
                            precision=sb.FP64 if precision is None else precision, fmm_theta=theta,
                            proxy_degree=degree, leaf_size=256)
    return sb.Context(cfg)


def test_treecode_adjoint_step_dot_product(sb):
    _, f, w0, wn = gaussian_vortex_state(sb, 5, 0.01, 1e-2)
    ctx = tree_ctx(sb, 5, 0.01)
    rng = np.random.default_rng(9)
    wbar_next = torch.from_numpy(rng.standard_normal(tuple(wn.shape))).cuda()
    wbar = torch.empty_like(wn)
    ctx.bve_adjoint_step(*f, wn, wbar_next, wbar)

    def step(w):
        v = w.clone()
        vel = [torch.zeros_like(v) for _ in range(3)]
        ctx.bve_back_rk4_step(*f, v, *vel)
        return v

    for seed in range(3):
        d = torch.from_numpy(np.random.default_rng(70 + seed).standard_normal(tuple(wn.shape))).cuda()
        h = 1e-6
        fd = float((wbar_next * (step(wn + h * d) - step(wn - h * d))).sum()) / (2 * h)
        ad = float((wbar * d).sum())
        assert abs(fd - ad) <= 1e-6 * abs(ad), (seed, fd, ad)


def test_treecode_gradient_matches_direct_sum_adjoint(sb):
    """The 20-step loss gradient through the treecode's adjoint against the
    float64 direct-sum adjoint's (the reference gradient): they differ by the
    treecode's approximation error."""
    ctxd, f, w0, wn = gaussian_vortex_state(sb, 5, 0.01, 1e-2)
    ctxt = tree_ctx(sb, 5, 0.01)
    area = f[3]
    grads = []
    for ctx in (ctxd, ctxt):
        v = w0.clone()
        vel = [torch.zeros_like(v) for _ in range(3)]
        ctx.bve_run(*f, v, *vel, nsteps=20)
        x = wn.clone().requires_grad_()
        out = sb.bve_rollout(ctx, *f, x, 20)
        (0.5 * (area * (out - v) ** 2).sum()).backward()
        grads.append(x.grad.clone())
    gd, gt = grads
    rel = float((gt - gd).norm() / gd.norm())
    print("treecode vs direct-sum adjoint gradient: relative L2 %.2e" % rel)
    assert rel <= 1e-5, rel


def test_mixed_treecode_adjoint_step_matches_float64(sb):
    """One reverse step on the mixed-precision treecode (the forward recomputed
    in mixed precision, the transposed pair sums in float32 on packed
    coordinates) against the same step in float64: the float32 rounding of
    the pair sums, 1e-6 relative L2 at most (measured ~1e-8)."""
    _, f, w0, wn = gaussian_vortex_state(sb, 5, 0.01, 1e-2)
    wbar_next = torch.from_numpy(np.random.default_rng(9).standard_normal(tuple(wn.shape))).cuda()
    out = []
    for prec in (sb.FP64, sb.MIXED):
        ctx = tree_ctx(sb, 5, 0.01, precision=prec)
        wbar = torch.empty_like(wn)
        ctx.bve_adjoint_step(*f, wn, wbar_next, wbar)
        out.append(wbar)
    rel = float((out[1] - out[0]).norm() / out[0].norm())
    print("mixed vs float64 treecode adjoint step: relative L2 %.2e" % rel)
    assert rel <= 1e-6, rel


def test_mixed_treecode_gradient_matches_direct_sum_adjoint(sb):
    """The 20-step loss gradient through the mixed-precision treecode's
    adjoint against the float64 direct-sum adjoint's: within the treecode's
    approximation error, as the float64 treecode."""
    ctxd, f, w0, wn = gaussian_vortex_state(sb, 5, 0.01, 1e-2)
    ctxm = tree_ctx(sb, 5, 0.01, precision=sb.MIXED)
    area = f[3]
    grads = []
    for ctx in (ctxd, ctxm):
        v = w0.clone()
        vel = [torch.zeros_like(v) for _ in range(3)]
        ctxd.bve_run(*f, v, *vel, nsteps=20)
        x = wn.clone().requires_grad_()
        out = sb.bve_rollout(ctx, *f, x, 20)
        (0.5 * (area * (out - v) ** 2).sum()).backward()
        grads.append(x.grad.clone())
    gd, gm = grads
    rel = float((gm - gd).norm() / gd.norm())
    print("mixed treecode vs direct-sum adjoint gradient: relative L2 %.2e" % rel)
    assert rel <= 1e-5, rel


def test_mixed_direct_sum_adjoint_matches_float64(sb):
    """The direct-sum velocity in mixed precision: one reverse step and the
    20-step gradient against the float64 direct sum's (float32 pairs on
    leaf-packed coordinates: 1e-6 relative L2 at most)."""
    ctxd, f, w0, wn = gaussian_vortex_state(sb, 5, 0.01, 1e-2)
    ctxm = sb.Context(sb.config_default(levels=5, interp_degree=3, kernel_eps=1e-4, omega=2 * np.pi, dt=0.01,
                                        velocity=sb.VEL_DIRECT, precision=sb.MIXED))
    wbar_next = torch.from_numpy(np.random.default_rng(5).standard_normal(tuple(wn.shape))).cuda()
    steps = []
    for ctx in (ctxd, ctxm):
        wbar = torch.empty_like(wn)
        ctx.bve_adjoint_step(*f, wn, wbar_next, wbar)
        steps.append(wbar)
    rel1 = float((steps[1] - steps[0]).norm() / steps[0].norm())
    area = f[3]
    v = w0.clone()
    vel = [torch.zeros_like(v) for _ in range(3)]
    ctxd.bve_run(*f, v, *vel, nsteps=20)
    grads = []
    for ctx in (ctxd, ctxm):
        x = wn.clone().requires_grad_()
        out = sb.bve_rollout(ctx, *f, x, 20)
        (0.5 * (area * (out - v) ** 2).sum()).backward()
        grads.append(x.grad.clone())
    rel20 = float((grads[1] - grads[0]).norm() / grads[0].norm())
    print("mixed vs float64 direct-sum adjoint: step %.2e, 20-step gradient %.2e" % (rel1, rel20))
    assert rel1 <= 1e-6 and rel20 <= 1e-6, (rel1, rel20)


def spectral_ctx(sb, levels, dt, theta=0.7):
    return sb.Context(sb.config_default(levels=levels, interp_degree=3, kernel_eps=1e-4, omega=2 * np.pi, dt=dt,
                                        precision=sb.FP64, fmm_theta=theta))


@pytest.mark.parametrize("levels", [3, 4])
def test_spectral_fmm_adjoint_step_dot_product(sb, levels):
    """One reverse step through the reference's own spectral FMM (displaced
    proxies on every panel, non-leaf displacements interpolated from the
    leaves) against central differences of the forward step."""
    _, f, w0, wn = gaussian_vortex_state(sb, levels, 0.01, 1e-2)
    ctx = spectral_ctx(sb, levels, 0.01)
    wbar_next = torch.from_numpy(np.random.default_rng(9).standard_normal(tuple(wn.shape))).cuda()
    wbar = torch.empty_like(wn)
    ctx.bve_adjoint_step(*f, wn, wbar_next, wbar)

    def step(w):
        v = w.clone()
        vel = [torch.zeros_like(v) for _ in range(3)]
        ctx.bve_back_rk4_step(*f, v, *vel)
        return v

    for seed in range(3):
        d = torch.from_numpy(np.random.default_rng(70 + seed).standard_normal(tuple(wn.shape))).cuda()
        h = 1e-6
        fd = float((wbar_next * (step(wn + h * d) - step(wn - h * d))).sum()) / (2 * h)
        ad = float((wbar * d).sum())
        print(f"levels {levels} seed {seed}: fd {fd:.10e} adjoint {ad:.10e}")
        assert abs(fd - ad) <= 1e-6 * abs(ad), (seed, fd, ad)


def test_spectral_fmm_gradient_close_to_direct_sum_adjoint(sb):
    """The 20-step loss gradient through the spectral FMM's adjoint against the
    float64 direct-sum adjoint's: they differ by the FMM's approximation
    error (theta 0.5 here; measured 1.3e-4 relative L2, bound 1e-3), which
    the forward runs show as well."""
    ctxd, f, w0, wn = gaussian_vortex_state(sb, 5, 0.01, 1e-2)
    ctxs = spectral_ctx(sb, 5, 0.01, theta=0.5)
    area = f[3]
    v = w0.clone()
    vel = [torch.zeros_like(v) for _ in range(3)]
    ctxd.bve_run(*f, v, *vel, nsteps=20)
    grads = []
    for ctx in (ctxd, ctxs):
        x = wn.clone().requires_grad_()
        out = sb.bve_rollout(ctx, *f, x, 20)
        (0.5 * (area * (out - v) ** 2).sum()).backward()
        grads.append(x.grad.clone())
    rel = float((grads[1] - grads[0]).norm() / grads[0].norm())
    fwd = []
    for ctx in (ctxd, ctxs):
        u = wn.clone()
        vel = [torch.zeros_like(u) for _ in range(3)]
        ctx.bve_run(*f, u, *vel, nsteps=20)
        fwd.append(u)
    rel_fwd = float((fwd[1] - fwd[0]).norm() / fwd[0].norm())
    print("spectral FMM vs direct sum after 20 steps: vorticity %.2e, adjoint gradient %.2e" % (rel_fwd, rel))
    assert rel <= 1e-3, rel


def test_mixed_spectral_fmm_adjoint_step_matches_float64(sb):
    """The spectral FMM's reverse step in mixed precision (forward recomputed in
    mixed precision, the transposed interactions in float32 on coordinates
    packed relative to the panels' centres) against the float64 one."""
    _, f, w0, wn = gaussian_vortex_state(sb, 5, 0.01, 1e-2)
    wbar_next = torch.from_numpy(np.random.default_rng(9).standard_normal(tuple(wn.shape))).cuda()
    out = []
    for prec in (sb.FP64, sb.MIXED):
        ctx = sb.Context(sb.config_default(levels=5, interp_degree=3, kernel_eps=1e-4, omega=2 * np.pi, dt=0.01,
                                           precision=prec, fmm_theta=0.7))
        wbar = torch.empty_like(wn)
        ctx.bve_adjoint_step(*f, wn, wbar_next, wbar)
        out.append(wbar)
    rel = float((out[1] - out[0]).norm() / out[0].norm())
    print("mixed vs float64 spectral FMM adjoint step: relative L2 %.2e" % rel)
    assert rel <= 1e-6, rel
