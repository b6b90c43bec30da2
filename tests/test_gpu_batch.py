"""GPU tests of the batched ensemble (sbslpm_batch): members with uneven trees
(different theta and proxy degree) stepped in one launch per phase must give
exactly what single contexts give member by member, and stay within the
accuracy bar against the float64 direct sum.

Tolerances: bit-exact against single contexts with the same near-field split
count and the CUDA-core well-separated interactions (the arithmetic per
target is the same; only the split count changes the order of the
near-field partial sums), <= 1e-12 with the autotuned split, mixed precision
<= 1e-6 relative L-infinity vorticity against the float64 direct sum after
one step.  The tensor-core well-separated interactions (3xTF32 GEMM over the
members) agree with the CUDA-core float32 pairs to <= 1e-6 relative
L-infinity in velocity, the single-pass TF32 GEMM to <= 1e-4.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

LEVELS, DEGREE, EPS, OMEGA, DT = 5, 3, 1e-4, 2 * np.pi, 0.005
THETA = [0.5, 0.8, 0.65, 0.7]
PDEG = [6, 8, 10, 8]


def rel(a, b):
    s = b.abs().max().item()
    return (a - b).abs().max().item() / (s if s > 0 else 1.0)


def grid_and_vors(sb, members):
    g = sb.build_grid(LEVELS, DEGREE, exact_cc=True)
    lat, lon = np.arcsin(np.clip(g.z, -1, 1)), np.arctan2(g.y, g.x)
    base = 2 * 0.5 * np.sin(lat) - 0.5 * np.sin(lat) * np.cos(lat) ** 4 * 30 * np.cos(4 * lon)
    vors = []
    for m in range(members):
        pert = 1e-3 * np.random.default_rng(m).standard_normal(3) @ np.stack([g.x, g.y, g.z]).reshape(3, -1)
        vors.append(base + pert.reshape(base.shape))
    vors = np.stack(vors)
    vors -= (vors * g.area).sum(axis=(1, 2), keepdims=True) / (4 * np.pi)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    return g, [T(g.x), T(g.y), T(g.z), T(g.area)], T(vors)


def base_cfg(sb, precision, **kw):
    return sb.config_default(levels=LEVELS, interp_degree=DEGREE, kernel_eps=EPS, omega=OMEGA, dt=DT,
                             precision=precision, leaf_size=256, **kw)


def single_step(sb, precision, theta, pdeg, xyza, vor, tuning=(128, 2, 2), near_form=None):
    ctx = sb.Context(base_cfg(sb, precision, fmm_theta=theta, proxy_degree=pdeg))
    if near_form is not None:
        ctx.set_near_form(near_form)  # the batch's near-field pair arithmetic
    if tuning:
        ctx.set_near_tuning(*tuning)
        ctx.set_cc_tuning(0, 0)  # one block per target panel, the batch's CUDA-core kernel
    v = vor.clone()
    vel = [torch.zeros_like(v) for _ in range(3)]
    ctx.bve_back_rk4_step(*xyza, v, *vel)
    return v, torch.stack(vel)


@pytest.mark.parametrize("precision,expanded", [("FP64", None), ("MIXED", None), ("MIXED", True)])
def test_batch_equals_single_contexts(sb, precision, expanded):
    """expanded = True forces the expanded near-field pair form on the batch
    (set-up keeps the difference form at this size); the single contexts
    follow the batch's form either way."""
    prec = getattr(sb, precision)
    g, xyza, vors = grid_and_vors(sb, len(THETA))
    batch = sb.Batch(base_cfg(sb, prec), THETA, PDEG)
    batch.set_tuning(128, 2, 2)  # the single context's near-field shape and split count
    if prec == sb.MIXED:
        batch.set_cc_mode(batch.CC_CUDA_CORES)  # the single context's float32 pair arithmetic
        batch.set_stage0_shared(False)  # and its per-member stage-0 near field
        if expanded is not None:
            batch.set_near_form(expanded)
            assert batch.near_form() == expanded
    v = vors.clone()
    vel = torch.zeros((len(THETA), 3) + v.shape[1:], dtype=torch.float64, device="cuda")
    batch.step(*xyza, v, vel)
    form = batch.near_form() if prec == sb.MIXED else None
    for m in range(len(THETA)):
        sv, svel = single_step(sb, prec, THETA[m], PDEG[m], xyza, vors[m].contiguous(), near_form=form)
        assert torch.equal(v[m], sv), m
        assert torch.equal(vel[m], svel), m


def test_stage0_shared_near_field_matches_per_member(sb):
    """The first stage's near field evaluated once per leaf pair for groups of
    members (theta-sorted, union lists with member bits) against every member's
    own near kernel: the same pairs, float32 sums in another order (one sum
    per member and component over a source leaf instead of two interleaved
    halves).  Both stay within the 1e-6 mixed-precision bar of the float64
    batch and of each other (measured: vorticity 1e-9, stage-0 velocity 5e-7,
    the float32 rounding of near-field sums whose terms largely cancel);
    graph replay equals eager steps."""
    g, xyza, vors = grid_and_vors(sb, 9)
    theta = [0.5, 0.8, 0.65, 0.7, 0.55, 0.75, 0.6, 0.52, 0.78]
    pdeg = [6, 8, 10, 8, 6, 10, 8, 6, 8]
    ref = sb.Batch(base_cfg(sb, sb.FP64), theta, pdeg)
    r = vors.clone()
    rel_ = torch.zeros((len(theta), 3) + r.shape[1:], dtype=torch.float64, device="cuda")
    ref.step(*xyza, r, rel_)
    out = []
    for shared in (False, True):
        batch = sb.Batch(base_cfg(sb, sb.MIXED), theta, pdeg)
        batch.set_tuning(128, 2, 2)
        batch.set_cc_mode(batch.CC_CUDA_CORES)
        batch.set_stage0_shared(shared)
        v = vors.clone()
        vel = torch.zeros((len(theta), 3) + v.shape[1:], dtype=torch.float64, device="cuda")
        batch.step(*xyza, v, vel)
        out.append((v, vel))
        if shared:
            w = vors.clone()
            wel = torch.zeros_like(vel)
            batch.run(*xyza, w, wel, nsteps=1)
            assert torch.equal(w, v) and torch.equal(wel, vel)
    assert rel(out[1][0], out[0][0]) <= 1e-8
    assert rel(out[1][1], out[0][1]) <= 1e-6
    for v, vel in out:
        assert rel(v, r) <= 1e-6 and rel(vel, rel_) <= 1e-6


@pytest.mark.parametrize("members", [1, 5])
def test_sharing_modes_with_partial_groups(sb, members):
    """One member, and five (a group of 4 plus a group of 1 in the shared
    well-separated kernel, one partial group of 8 in the stage-0 near field):
    the member-sharing modes against the per-member ones, within 1e-6."""
    g, xyza, vors = grid_and_vors(sb, members)
    theta = [0.5, 0.8, 0.65, 0.7, 0.55][:members]
    pdeg = [8] * members
    out = []
    for shared in (False, True):
        batch = sb.Batch(base_cfg(sb, sb.MIXED), theta, pdeg)
        batch.set_tuning(128, 2, 2)
        batch.set_cc_mode(batch.CC_SHARED if shared else batch.CC_CUDA_CORES)
        batch.set_stage0_shared(shared)
        out.append(batch_step(sb, batch, xyza, vors))
    assert rel(out[1][0], out[0][0]) <= 1e-6
    assert rel(out[1][1], out[0][1]) <= 1e-6


def test_stage0_shared_refused_in_float64(sb):
    g, xyza, vors = grid_and_vors(sb, 2)
    batch = sb.Batch(base_cfg(sb, sb.FP64), THETA[:2], PDEG[:2])
    with pytest.raises(sb.SbslpmError):
        batch.set_stage0_shared(True)
    batch.set_stage0_shared(False)
    with pytest.raises(sb.SbslpmError):  # nor the expanded near-field form
        batch.set_near_form(True)
    assert not batch.near_form()


def test_batch_autotuned_close_to_single(sb):
    g, xyza, vors = grid_and_vors(sb, len(THETA))
    batch = sb.Batch(base_cfg(sb, sb.FP64), THETA, PDEG)
    v = vors.clone()
    vel = torch.zeros((len(THETA), 3) + v.shape[1:], dtype=torch.float64, device="cuda")
    batch.step(*xyza, v, vel)
    nt, tpt, splits, cand, ms = batch.tuning()
    assert cand >= 4 and nt * tpt >= 256 and 1 <= splits <= 4 and ms > 0
    for m in range(len(THETA)):
        sv, svel = single_step(sb, sb.FP64, THETA[m], PDEG[m], xyza, vors[m].contiguous())
        assert rel(v[m], sv) <= 1e-12, m
        assert rel(vel[m], svel) <= 1e-12, m


def test_batch_graph_replay_equals_steps(sb):
    g, xyza, vors = grid_and_vors(sb, len(THETA))
    a = sb.Batch(base_cfg(sb, sb.MIXED), THETA, PDEG)
    b = sb.Batch(base_cfg(sb, sb.MIXED), THETA, PDEG)
    for x in (a, b):
        x.set_tuning(128, 2, 2)
    va, vb = vors.clone(), vors.clone()
    vela = torch.zeros((len(THETA), 3) + va.shape[1:], dtype=torch.float64, device="cuda")
    velb = torch.zeros_like(vela)
    a.run(*xyza, va, vela, nsteps=3)
    for _ in range(3):
        b.step(*xyza, vb, velb)
    assert torch.equal(va, vb) and torch.equal(vela, velb)


@pytest.mark.parametrize("mode", [-1, 0, 1, 2])
def test_batch_mixed_accuracy_vs_direct_sum(sb, mode):
    g, xyza, vors = grid_and_vors(sb, len(THETA))
    batch = sb.Batch(base_cfg(sb, sb.MIXED), THETA, PDEG)
    batch.set_cc_mode(mode)
    v = vors.clone()
    vel = torch.zeros((len(THETA), 3) + v.shape[1:], dtype=torch.float64, device="cuda")
    batch.step(*xyza, v, vel)
    for m in range(len(THETA)):
        ctx = sb.Context(base_cfg(sb, sb.FP64, velocity=sb.VEL_DIRECT))
        d = vors[m].clone()
        dvel = [torch.zeros_like(d) for _ in range(3)]
        ctx.bve_back_rk4_step(*xyza, d, *dvel)
        print("cc mode %d member %d: vorticity vs float64 direct sum %.2e" % (mode, m, rel(v[m], d)))
        assert rel(v[m], d) <= 1e-6, (m, rel(v[m], d))


def batch_step(sb, batch, xyza, vors):
    v = vors.clone()
    vel = torch.zeros((vors.shape[0], 3) + v.shape[1:], dtype=torch.float64, device="cuda")
    batch.step(*xyza, v, vel)
    return v, vel


@pytest.mark.parametrize("mode,tol", [(1, 1e-6), (2, 1e-4), (3, 1e-6)])
def test_tensor_core_cc_matches_cuda_core_pairs(sb, mode, tol):
    g, xyza, vors = grid_and_vors(sb, len(THETA))
    ref = sb.Batch(base_cfg(sb, sb.MIXED), THETA, PDEG)
    ref.set_tuning(128, 2, 2)
    ref.set_cc_mode(ref.CC_CUDA_CORES)
    tc = sb.Batch(base_cfg(sb, sb.MIXED), THETA, PDEG)
    tc.set_tuning(128, 2, 2)
    tc.set_cc_mode(mode)
    m, up, flops = tc.cc_info()
    near, far = tc.pairs()
    assert m == mode and (flops > 0) == (mode != 3) and up * 81 * 81 >= far / len(THETA)
    vr, velr = batch_step(sb, ref, xyza, vors)
    vt, velt = batch_step(sb, tc, xyza, vors)
    for k in range(len(THETA)):
        e = rel(velt[k], velr[k])
        print("member %d: tensor-core vs CUDA-core velocity %.2e" % (k, e))
        assert e <= tol, (k, e)
        assert rel(vt[k], vr[k]) <= tol, k


def test_tensor_core_wait_runs_out_and_the_batch_recovers(sb):
    """The tensor-core kernel's failure path: with one producer arrival
    withheld in every CTA (sbslpm_batch_set_wait_test), the MMA warp's
    bounded wait runs out before any MMA is issued, the CTA frees its tensor
    memory and returns, and the step reports SBSLPM_ERR_TIMEOUT.  The next
    step with the test off gives the normal result bit for bit."""
    g, xyza, vors = grid_and_vors(sb, len(THETA))
    tc = sb.Batch(base_cfg(sb, sb.MIXED), THETA, PDEG)
    tc.set_tuning(128, 2, 2)
    tc.set_cc_mode(1)
    v0, vel0 = batch_step(sb, tc, xyza, vors)  # a normal step first (and the first-step timing)
    tc.set_wait_test(True)
    with pytest.raises(sb.SbslpmError) as err:
        batch_step(sb, tc, xyza, vors)
    assert err.value.status == 7  # SBSLPM_ERR_TIMEOUT
    tc.set_wait_test(False)
    v1, vel1 = batch_step(sb, tc, xyza, vors)
    assert torch.equal(v1, v0) and torch.equal(vel1, vel0)


def test_cc_autotuner_times_every_mode(sb):
    g, xyza, vors = grid_and_vors(sb, len(THETA))
    batch = sb.Batch(base_cfg(sb, sb.MIXED), THETA, PDEG)
    assert batch.cc_info()[0] == batch.CC_AUTO
    batch_step(sb, batch, xyza, vors)
    groups = batch.cc_groups()
    assert sorted(gr["degree"] for gr in groups) == sorted(set(PDEG))
    assert sum(gr["members"] for gr in groups) == len(THETA)
    for gr in groups:
        t = {0: gr["ms_cuda_cores"], 1: gr["ms_tensor_cores"], 3: gr["ms_shared"]}
        assert min(t.values()) > 0
        assert gr["mode"] == min(t, key=t.get)


def test_tensor_core_cc_rejects_float64(sb):
    batch = sb.Batch(base_cfg(sb, sb.FP64), THETA, PDEG)
    assert batch.cc_info()[0] == 0
    with pytest.raises(sb.SbslpmError):
        batch.set_cc_mode(1)


def test_batch_rejects_bad_members(sb):
    with pytest.raises(sb.SbslpmError):
        sb.Batch(base_cfg(sb, sb.FP64), [0.7, 0.7], [8, 4])
    with pytest.raises(sb.SbslpmError):
        sb.Batch(base_cfg(sb, sb.FP64), [0.7, -1.0], [8, 8])
