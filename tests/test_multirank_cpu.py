"""The multi-rank path of bench.py on the CPU with the gloo backend
(world size 2): every rank steps an independent replica (no data-path
collective), the job's time is the maximum over ranks and the rate counts
every rank's steps; the reference arm runs on rank 0 alone."""
import importlib.util
import os
import socket

import numpy as np
import pytest

from conftest import ROOT

torch = pytest.importorskip("torch")


def load_bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=30))
    try:
        bench = load_bench()
        # rank-specific device times; the job's time is their maximum
        t = bench.job_time(dist, torch, [30.0, 45.0][rank], "cpu")
        z = np.linspace(-1, 1, 16)
        v = bench.replica_vorticity(np.ones(16), z, rank, world)
        vs = [torch.zeros(16, dtype=torch.float64) for _ in range(world)]
        dist.all_gather(vs, torch.from_numpy(v))
        out.put((rank, t, [x.numpy().tolist() for x in vs]))
    finally:
        dist.destroy_process_group()


def test_two_ranks_gloo():
    ctx = torch.multiprocessing.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, t0, v0), (r1, t1, v1) = res
    assert t0 == t1 == 45.0  # max over ranks, the same on every rank
    assert v0 == v1 and v0[0] != v0[1]  # the two replicas differ (independent members)
    bench = load_bench()
    steps, world = 10, 2
    assert world * steps / (t0 * 1e-3) == pytest.approx(444.444, rel=1e-5)


def test_single_rank_is_the_benchmark_state():
    bench = load_bench()
    v = np.arange(5.0)
    assert bench.replica_vorticity(v, np.ones(5), 0, 1) is v


def test_reference_arm_other_ranks_do_nothing(capsys):
    bench = load_bench()

    class Args:
        steps, warmup, gpus = 1, 0, 2

    bench.run_reference(Args(), 1)  # rank 1 returns without work or output
    assert capsys.readouterr().out == ""


def _lists_rank(rank, world, port, thetas, out):
    """An ensemble sharded over ranks: each rank builds the treecode lists of
    its members (every world-th theta) through the library's host API, and
    the ranks gather them."""
    import datetime

    import torch.distributed as dist

    from conftest import load_package

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=30))
    try:
        sb = load_package()
        panels = sb.cubed_sphere_panels_init(4)
        mine = {m: sb.dual_tree_traversal_flagged(4, panels, th) for m, th in enumerate(thetas) if m % world == rank}
        mine = {m: (l.tolist(), n.tolist()) for m, (l, n) in mine.items()}
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        out.put((rank, gathered))
    finally:
        dist.destroy_process_group()


def test_ensemble_lists_sharded_over_two_ranks():
    """The library's host traversal called on two gloo ranks, members split
    between them: the gathered lists equal one process's build of every
    member, and the same on both ranks."""
    from conftest import load_package

    thetas = [0.5, 0.55, 0.6, 0.65, 0.7, 0.8]
    ctx = torch.multiprocessing.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_lists_rank, args=(r, 2, port, thetas, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=120) for _ in procs), key=lambda r: r[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0][1] == res[1][1]
    merged = {m: v for part in res[0][1] for m, v in part.items()}
    sb = load_package()
    panels = sb.cubed_sphere_panels_init(4)
    for m, th in enumerate(thetas):
        lst, near = sb.dual_tree_traversal_flagged(4, panels, th)
        assert merged[m] == (lst.tolist(), near.tolist())
        assert np.array_equal(lst, sb.dual_tree_traversal(4, panels, th))


def _shard_id_rank(rank, world, port, out):
    """The host side of a sharded problem: the group's first rank makes the
    NCCL id through the library, every rank receives it, and each takes its
    slice of the particles."""
    import datetime

    import torch.distributed as dist

    from conftest import load_package

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=30))
    try:
        sb = load_package()
        ident = sb.exchange_shard_id()
        out.put((rank, ident, sb.shard_slice(24576, 16, 1536, rank, world)))
    finally:
        dist.destroy_process_group()


def test_shard_id_and_slices_over_two_ranks():
    ctx = torch.multiprocessing.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_shard_id_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=120) for _ in procs), key=lambda r: r[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, id0, s0), (_, id1, s1) = res
    assert len(id0) == 128 and id0 == id1  # one communicator id for both ranks
    assert s0 == (0, 196608) and s1 == (196608, 196608)  # disjoint, covering 24,576 x 16 particles


def test_shard_slices_partition_the_particles():
    from conftest import load_package

    sb = load_package()
    for ranks in (1, 2, 3, 4, 6, 8):
        s = [sb.shard_slice(384, 16, 96, r, ranks) for r in range(ranks)]
        assert s[0][0] == 0 and all(a[0] + a[1] == b[0] for a, b in zip(s, s[1:]))
        assert s[-1][0] + s[-1][1] == 384 * 16
    with pytest.raises(ValueError):
        sb.shard_slice(384, 16, 96, 0, 5)
