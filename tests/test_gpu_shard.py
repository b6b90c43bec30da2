"""One treecode problem sharded over ranks: owner-computes over the tree leaves.

These tests get one GPU, so the ranks of a sharded problem are emulated as
separate contexts on it, each evaluating its own slice without a
communicator (no collective: nothing waits on anything).  Every rank's slice
of the velocity must be bit-identical to the unsharded context's, in float64
and in mixed precision, because each owned target sums the same list entries
in the same order.  A one-rank NCCL communicator runs whole steps with their
in-place all-gathers and must reproduce the unsharded steps bit for bit.  A
rank whose peer never joins ends its set-up with SBSLPM_ERR_TIMEOUT (a wait
on the host: no kernel is in flight) and the context stays usable.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

DT, OMEGA, EPS = 0.005, 2 * np.pi, 1e-4


def cuda(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def rh4(x, y, z, area):
    lat, lon = np.arcsin(np.clip(z, -1, 1)), np.arctan2(y, x)
    vor = np.sin(lat) - 0.5 * np.sin(lat) * np.cos(lat) ** 4 * 30 * np.cos(4 * lon)
    return vor - (vor * area).sum() / (4 * np.pi)


def make_ctx(sb, levels, leaf, n, theta, prec):
    cfg = sb.config_default(levels=levels, interp_degree=3, kernel_eps=EPS, omega=OMEGA, dt=DT, fmm_theta=theta,
                            proxy_degree=n, leaf_size=leaf, precision=prec)
    return sb.Context(cfg)


def fix_shapes(ctx, form):
    """The same launch shapes on every context (summation order is part of the result)."""
    ctx.set_near_tuning(128, 2, 2)
    ctx.set_near_mutual(False)
    if form == "bulk":
        ctx.set_cc_tuning_bulk(3, 3)
    else:
        ctx.set_cc_tuning(3, 3)


@pytest.fixture(scope="module")
def grids(sb):
    out = {}
    for levels in (4, 5):
        g = sb.build_grid(levels, 3, exact_cc=True)
        out[levels] = (g, rh4(g.x, g.y, g.z, g.area))
    return out


# (levels, leaf size, proxy degree, theta, ranks): 96 tree leaves in both trees
CASES = [(5, 256, 8, 0.7, 4), (5, 256, 8, 0.7, 3), (4, 64, 8, 0.7, 8), (5, 256, 6, 0.5, 2)]


@pytest.mark.parametrize("prec,form", [("fp64", "staged"), ("mixed", "staged"), ("mixed", "bulk")])
@pytest.mark.parametrize("levels,leaf,n,theta,ranks", CASES)
def test_rank_slices_are_the_whole_problems_velocity(sb, grids, levels, leaf, n, theta, ranks, prec, form):
    g, vor = grids[levels]
    p = sb.FP64 if prec == "fp64" else sb.MIXED
    f = [cuda(g.x), cuda(g.y), cuda(g.z), cuda(g.area), cuda(vor)]
    whole = make_ctx(sb, levels, leaf, n, theta, p)
    fix_shapes(whole, form)
    ref = [torch.zeros_like(f[0]) for _ in range(3)]
    whole.bve_velocity(*f, *ref)
    ref = torch.stack(ref).reshape(3, -1)
    N = ref.shape[1]
    covered = 0
    for r in range(ranks):
        ctx = make_ctx(sb, levels, leaf, n, theta, p)
        ctx.shard(r, ranks)
        fix_shapes(ctx, form)
        first, count = ctx.shard_range()
        assert (first, count) == sb.shard_slice(ctx.leaf_count, ctx.q, 96, r, ranks)
        vel = [torch.full_like(f[0], float("nan")) for _ in range(3)]
        ctx.bve_velocity(*f, *vel)
        vel = torch.stack(vel).reshape(3, -1)
        assert torch.equal(vel[:, first:first + count], ref[:, first:first + count]), r
        # nothing outside the slice is written
        assert torch.isnan(vel[:, :first]).all() and torch.isnan(vel[:, first + count:]).all()
        covered += count
        ctx.close()
    assert covered == N


def test_slice_timing_counts_the_slices_pairs(sb):
    """time_interactions on a rank times its own leaves' near field: the
    ranks' pair counts add up to the whole problem's."""
    whole = make_ctx(sb, 5, 256, 8, 0.7, sb.MIXED)
    fix_shapes(whole, "staged")
    _, total = whole.time_interactions(reps=1)
    parts = 0.0
    for r in range(4):
        ctx = make_ctx(sb, 5, 256, 8, 0.7, sb.MIXED)
        ctx.shard(r, 4)
        fix_shapes(ctx, "staged")
        parts += ctx.time_interactions(reps=1)[1]
    assert parts == total


def test_sharded_context_without_communicator_refuses_whole_steps(sb, grids):
    g, vor = grids[4]
    ctx = make_ctx(sb, 4, 64, 8, 0.7, sb.FP64)
    ctx.shard(1, 2)
    f = [cuda(g.x), cuda(g.y), cuda(g.z), cuda(g.area), cuda(vor)]
    vel = [torch.zeros_like(f[0]) for _ in range(3)]
    for call in (lambda: ctx.bve_back_rk4_step(*f, *vel), lambda: ctx.bve_run(*f, *vel, nsteps=2),
                 lambda: ctx.bve_adjoint_step(*f[:5], torch.ones_like(f[0]), torch.zeros_like(f[0]))):
        with pytest.raises(sb.SbslpmError) as e:
            call()
        assert e.value.status == 1  # SBSLPM_ERR_CONFIG
    ctx.shard(0, 1)  # one rank again: the whole problem
    ctx.bve_back_rk4_step(*f, *vel)


def test_bad_shard_arguments(sb):
    ctx = make_ctx(sb, 4, 64, 8, 0.7, sb.FP64)
    for rank, nranks in ((0, 0), (2, 2), (-1, 2), (0, 5)):  # 96 leaves: 5 does not divide them
        with pytest.raises(sb.SbslpmError) as e:
            ctx.shard(rank, nranks)
        assert e.value.status == 5  # SBSLPM_ERR_ARG
    spectral = sb.Context(sb.config_default(levels=4, interp_degree=3))
    with pytest.raises(sb.SbslpmError) as e:
        spectral.shard(0, 2)
    assert e.value.status == 1


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_one_rank_communicator_steps_are_the_unsharded_steps(sb, grids, prec):
    """Whole steps through NCCL (a one-rank communicator: the all-gather after
    every stage is a copy in place) against the same steps without sharding:
    bit-identical vorticity and velocity, for the single step and for a run
    (steps enqueued one by one when a communicator is present)."""
    g, vor = grids[5]
    p = sb.FP64 if prec == "fp64" else sb.MIXED
    out = []
    for sharded in (False, True):
        ctx = make_ctx(sb, 5, 256, 8, 0.7, p)
        if sharded:
            ctx.shard(0, 1, sb.shard_unique_id(), timeout=60.0)
        fix_shapes(ctx, "staged")
        f = [cuda(g.x), cuda(g.y), cuda(g.z), cuda(g.area), cuda(vor)]
        vel = [torch.zeros_like(f[0]) for _ in range(3)]
        ctx.bve_back_rk4_step(*f, *vel)
        ctx.bve_run(*f, *vel, nsteps=3)
        torch.cuda.synchronize()
        out.append((f[4].clone(), torch.stack(vel)))
        if sharded:
            ctx.shard_release()
        ctx.close()
    assert torch.equal(out[0][0], out[1][0])
    assert torch.equal(out[0][1], out[1][1])


NEVER_JOINS = r"""
import sys
import numpy as np
import torch
sys.path.insert(0, sys.argv[1])
from conftest import load_package
sb = load_package()
cfg = sb.config_default(levels=4, interp_degree=3, kernel_eps=1e-4, omega=2 * np.pi, dt=0.005, fmm_theta=0.7,
                        proxy_degree=8, leaf_size=64, precision=sb.FP64)
ctx = sb.Context(cfg)
try:
    ctx.shard(0, 2, sb.shard_unique_id(), timeout=3.0)
    print("joined")
except sb.SbslpmError as e:
    print("status", e.status)
print("range", *ctx.shard_range())
g = sb.build_grid(4, 3, exact_cc=True)
T = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()
v = T(g.z)
vel = [torch.zeros_like(v) for _ in range(3)]
ctx.bve_back_rk4_step(T(g.x), T(g.y), T(g.z), T(g.area), v, *vel)
print("stepped", bool(torch.isfinite(v).all()))
"""


def test_a_rank_that_never_joins_times_out(sb):
    """Rank 0 of 2 with no rank 1: the communicator's set-up is polled on the
    host and gives up after the limit with SBSLPM_ERR_TIMEOUT, leaving the
    context as it was (unsharded): it steps as before.  Run in a child
    process with its own time limit (the wait is on the host: no kernel is in
    flight while it lasts)."""
    import os
    import subprocess
    import sys

    from conftest import ROOT

    run = subprocess.run([sys.executable, "-c", NEVER_JOINS, os.path.join(ROOT, "tests")], capture_output=True,
                         text=True, timeout=180, cwd=ROOT)
    out = run.stdout.split("\n")
    assert run.returncode == 0, run.stdout + run.stderr
    assert "status 7" in out  # SBSLPM_ERR_TIMEOUT
    assert "range 0 6144" in out  # 384 leaves x 16 points: unsharded
    assert "stepped True" in out
