"""GPU tests of the treecode's well-separated (cluster-cluster) launch shapes:
every chunked shape (1..8 chunk slots per block, 1..4 list entries per
chunk) against the whole-panel kernel, for every proxy count with a chunked
kernel, in both precisions, and the barrier-free, bulk-copy (TMA) and
warp-per-chunk mixed-precision forms against the staged one, through the C
ABI (sbslpm_set_cc_tuning, sbslpm_set_cc_tuning_direct,
sbslpm_set_cc_tuning_bulk, sbslpm_set_cc_tuning_warp).

The shapes evaluate the same pairs with the same per-source-panel arithmetic
and differ only in the order in which a target's float64 sums are added, so
the step agrees to <= 1e-13 relative L-infinity; shapes with the same chunk
length agree bit for bit.  The treecode itself is checked against the
float64 direct sum in test_gpu_bve.py.
"""
import numpy as np
import pytest

from test_gpu_bve import rel, step, unit_fields, unit_sphere_rh4

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

ORDER_TOL = 1e-13
WARPS = (1, 2, 4, 8)  # warps per block of the warp-per-chunk form


def tree_ctx(sb, n, precision, leaf=64):
    cfg = sb.config_default(levels=5, interp_degree=3, fmm_theta=0.7, kernel_eps=1e-4, omega=2 * np.pi, dt=0.005,
                            proxy_degree=n, leaf_size=leaf, precision=precision)
    return sb.Context(cfg)


def shapes(q):
    """(slots, chunk length) of every chunked shape: slots in {1, 2, 3, 4, 6,
    8} whose blocks (slots x q threads rounded up to whole warps) hold at most
    512 threads with at most a fifth of them idle."""
    out = []
    for s in (1, 2, 3, 4, 6, 8):
        nt = -(-s * q // 32) * 32
        if nt <= 512 and 5 * s * q >= 4 * nt:
            out += [(s, k) for k in (1, 2, 3, 4)]
    return out


def direct_shapes(q, tpt):
    """(slots, chunk length) of the barrier-free form with tpt target proxies
    per thread: ceil(q / tpt) threads per slot, the same block rule."""
    qt = -(-q // tpt)
    out = []
    for s in (1, 2, 3, 4, 6, 8):
        nt = -(-s * qt // 32) * 32
        if nt <= 512 and 5 * s * qt >= 4 * nt:
            out += [(s, k) for k in (1, 2, 3, 4)]
    return out


@pytest.fixture(scope="module")
def grid(sb):
    g = sb.build_grid(5, 3, exact_cc=True)
    return g, unit_sphere_rh4(g)


@pytest.mark.parametrize("n", [5, 6, 7, 8, 9, 10])
@pytest.mark.parametrize("precision", ["FP64", "MIXED"])
def test_chunked_shapes_match_whole_panel_kernel(sb, grid, n, precision):
    g, vor = grid
    ctx = tree_ctx(sb, n, getattr(sb, precision))
    ctx.set_near_tuning(128, 2, 2)
    ctx.set_cc_tuning(0, 0)
    ref = unit_fields(g, vor)
    step(ctx, ref)
    q = (n + 1) ** 2
    by_len = {}
    for sl, k in shapes(q):
        ctx.set_cc_tuning(sl, k)
        assert ctx.cc_tuning()[:3] == (sl, k, -(-sl * q // 32) * 32)
        f = unit_fields(g, vor)
        step(ctx, f)
        assert rel(torch.stack(f["vel"]), torch.stack(ref["vel"])) <= ORDER_TOL, (sl, k)
        assert rel(f["vors"], ref["vors"]) <= ORDER_TOL, (sl, k)
        if k in by_len:  # the slot count does not change the arithmetic
            assert torch.equal(f["vors"], by_len[k]["vors"]), (sl, k)
            assert all(torch.equal(a, b) for a, b in zip(f["vel"], by_len[k]["vel"])), (sl, k)
        by_len.setdefault(k, f)


@pytest.mark.parametrize("n", [5, 6, 7, 8, 9, 10])
def test_barrier_free_form_matches_staged_form(sb, grid, n):
    """The barrier-free kernel (sources read through L1 from a pair-transposed
    copy, 1 or 2 target proxies per thread) runs the same per-source-panel
    float32 arithmetic in the same order as the staged kernel: with the same
    chunk length the step is bit-identical."""
    g, vor = grid
    ctx = tree_ctx(sb, n, sb.MIXED)
    ctx.set_near_tuning(128, 2, 2)
    q = (n + 1) ** 2
    staged = {}
    for k in (1, 2, 3, 4):
        ctx.set_cc_tuning(shapes(q)[0][0], k)
        staged[k] = unit_fields(g, vor)
        step(ctx, staged[k])
    for tpt in (1, 2):
        for sl, k in direct_shapes(q, tpt):
            ctx.set_cc_tuning_direct(sl, k, tpt)
            assert ctx.cc_form() == tpt
            assert ctx.cc_tuning()[:3] == (sl, k, -(-sl * -(-q // tpt) // 32) * 32)
            f = unit_fields(g, vor)
            step(ctx, f)
            assert torch.equal(f["vors"], staged[k]["vors"]), (tpt, sl, k)
            assert all(torch.equal(a, b) for a, b in zip(f["vel"], staged[k]["vel"])), (tpt, sl, k)
    # the bulk-copy form: the staged form's slots, each slot's source panels
    # copied into shared memory by cp.async.bulk (double-buffered)
    for sl, k in shapes(q):
        ctx.set_cc_tuning_bulk(sl, k)
        assert ctx.cc_form() == 3
        assert ctx.cc_tuning()[:3] == (sl, k, -(-sl * q // 32) * 32)
        f = unit_fields(g, vor)
        step(ctx, f)
        assert torch.equal(f["vors"], staged[k]["vors"]), ("bulk", sl, k)
        assert all(torch.equal(a, b) for a, b in zip(f["vel"], staged[k]["vel"])), ("bulk", sl, k)
    # the warp-per-chunk form: ceil(q / 32) target proxies per lane, warp-private
    # cp.async staging, __syncwarp only
    for w in WARPS:
        for k in (1, 2, 3, 4):
            ctx.set_cc_tuning_warp(w, k)
            assert ctx.cc_form() == 4
            assert ctx.cc_tuning()[:3] == (w, k, 32 * w)
            f = unit_fields(g, vor)
            step(ctx, f)
            assert torch.equal(f["vors"], staged[k]["vors"]), ("warp", w, k)
            assert all(torch.equal(a, b) for a, b in zip(f["vel"], staged[k]["vel"])), ("warp", w, k)


def test_autotuner_times_every_shape(sb, grid):
    g, vor = grid
    ctx = tree_ctx(sb, 8, sb.MIXED)
    f = unit_fields(g, vor)
    step(ctx, f)
    sl, k, threads, cand, ms = ctx.cc_tuning()
    assert cand == (1 + 2 * len(shapes(81)) + len(direct_shapes(81, 1)) + len(direct_shapes(81, 2))
                    + 4 * len(WARPS)) and ms > 0
    tpt = ctx.cc_form()
    if tpt in (1, 2):
        assert (sl, k) in direct_shapes(81, tpt) and threads == -(-sl * -(-81 // tpt) // 32) * 32
    elif tpt == 4:
        assert sl in WARPS and 1 <= k <= 4 and threads == 32 * sl
    else:  # staged or bulk copies: the same shapes
        assert (sl, k, threads) == (0, 0, 128) or ((sl, k) in shapes(81) and threads == -(-sl * 81 // 32) * 32)
    again = unit_fields(g, vor)
    step(ctx, again)
    assert torch.equal(again["vors"], f["vors"])  # a fixed shape is deterministic


def test_graph_replay_with_chunked_shape(sb, grid):
    g, vor = grid
    ctx = tree_ctx(sb, 6, sb.MIXED)
    ctx.set_near_tuning(128, 2, 2)
    ctx.set_cc_tuning(3, 3)
    a, b = unit_fields(g, vor), unit_fields(g, vor)
    step(ctx, a, 2)
    step(ctx, b, 2, graph=True)
    assert torch.equal(a["vors"], b["vors"])


def test_rejects_unsupported_shapes(sb):
    ctx = tree_ctx(sb, 6, sb.MIXED)  # 49 proxies: slots 3, 4, 6, 8
    for sl, k in ((1, 1), (2, 2), (5, 1), (3, 0), (3, 5), (9, 1), (0, 1), (-1, 1)):
        with pytest.raises(sb.SbslpmError):
            ctx.set_cc_tuning(sl, k)
    for sl, k, tpt in ((1, 1, 3), (3, 1, 0), (3, 0, 1), (5, 1, 1)):
        with pytest.raises(sb.SbslpmError):
            ctx.set_cc_tuning_direct(sl, k, tpt)
    with pytest.raises(sb.SbslpmError):  # float64: no barrier-free form
        tree_ctx(sb, 6, sb.FP64).set_cc_tuning_direct(6, 1, 1)
    with pytest.raises(sb.SbslpmError):  # nor a bulk-copy one
        tree_ctx(sb, 6, sb.FP64).set_cc_tuning_bulk(3, 1)
    with pytest.raises(sb.SbslpmError):
        ctx.set_cc_tuning_bulk(1, 1)  # 49 proxies: slots 3, 4, 6, 8
    for w, k in ((3, 1), (0, 1), (16, 1), (4, 0), (4, 5)):
        with pytest.raises(sb.SbslpmError):
            ctx.set_cc_tuning_warp(w, k)
    with pytest.raises(sb.SbslpmError):  # float64: no warp-per-chunk form
        tree_ctx(sb, 6, sb.FP64).set_cc_tuning_warp(4, 1)
    small = tree_ctx(sb, 3, sb.MIXED)  # 16 proxies: whole-panel kernel only
    with pytest.raises(sb.SbslpmError):
        small.set_cc_tuning(1, 1)
    assert small.cc_tuning()[:3] == (0, 0, 128)
    spectral = sb.Context(sb.config_default(levels=4, interp_degree=3, fmm_theta=0.7, kernel_eps=1e-4))
    with pytest.raises(sb.SbslpmError):
        spectral.set_cc_tuning(0, 0)
