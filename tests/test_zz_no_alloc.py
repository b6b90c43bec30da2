"""The direct-sum entry point that allocates no device memory.

sbslpm_direct_sum_bve_noalloc serves callers that may not let a library
allocate device memory (a host model with a device footprint fixed at
start-up, or one that routes all device memory through its own allocator).
Its scratch is a fixed array inside the library instead of a per-call
allocation.  These tests call it through the C ABI and check it against the
allocating entry point, sbslpm_direct_sum_bve, on two calls in a row with
different inputs (so leftovers of the first call in the shared scratch would
show) and on a target count that leaves room for fewer source groups, and
check that a size beyond its fixed scratch and host arrays are refused.

This file is collected last, so a run that stops at the first failure has
run every other test first; it also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

TOL = 1e-12  # float64 path tolerance used by the other GPU parity tests
MAX_TARGETS = (1 << 21) // 3


def points(rng, n):
    p = rng.standard_normal((n, 3))
    p /= np.linalg.norm(p, axis=1, keepdims=True)
    return [torch.from_numpy(np.ascontiguousarray(p[:, i])).cuda() for i in range(3)]


def call_noalloc(sb, t, s, w, eps, precision):
    """Direct C-ABI call of sbslpm_direct_sum_bve_noalloc."""
    out = [torch.full_like(t[0], float("nan")) for _ in range(3)]
    status = sb.lib().sbslpm_direct_sum_bve_noalloc(
        ctypes.c_long(t[0].numel()), *[ctypes.c_void_p(a.data_ptr()) for a in t], ctypes.c_long(s[0].numel()),
        *[ctypes.c_void_p(a.data_ptr()) for a in (*s, w)], ctypes.c_double(eps), ctypes.c_int(precision),
        *[ctypes.c_void_p(a.data_ptr()) for a in out], ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert status == 0, sb.lib().sbslpm_last_error().decode()
    return torch.stack(out)


def rel(a, b):
    return float((a - b).abs().max() / b.abs().max())


@pytest.mark.parametrize("precision", [0, 1])
def test_noalloc_matches_allocating_entry_point(sb, precision):
    rng = np.random.default_rng(11 + precision)
    for nt, ns in ((3000, 5000), (1234, 777)):  # two calls in a row, different sizes and inputs
        t, s = points(rng, nt), points(rng, ns)
        w = torch.from_numpy(rng.standard_normal(ns) * 1e-3).cuda()
        want = torch.stack(sb.direct_sum_bve(*t, *s, w, 1e-4, precision))
        got = call_noalloc(sb, t, s, w, 1e-4, precision)
        assert torch.isfinite(got).all()
        assert rel(got, want) <= TOL


def test_noalloc_with_fewer_groups_than_the_allocating_path(sb):
    """200,000 targets leave room for 3 source groups in the fixed scratch
    where the allocating entry point uses 4: the same sums in another
    order, so the results agree to rounding."""
    rng = np.random.default_rng(29)
    t, s = points(rng, 200_000), points(rng, 8192)
    w = torch.from_numpy(rng.standard_normal(8192) * 1e-3).cuda()
    want = torch.stack(sb.direct_sum_bve(*t, *s, w, 1e-4, 0))
    got = call_noalloc(sb, t, s, w, 1e-4, 0)
    assert rel(got, want) <= TOL


@pytest.mark.parametrize("name", ["sbslpm_direct_sum_bve_noalloc", "sbslpm_direct_sum_bve"])
def test_direct_sums_refuse_host_arrays(sb, name):
    """Host arrays are refused before any copy or launch, with a message."""
    n = 64
    host = [np.zeros(n) for _ in range(6)]
    L = sb.lib()
    ptr = [ctypes.c_void_p(a.ctypes.data) for a in host]
    for ns in (0, 16):  # no sources: the path that only clears the outputs
        status = getattr(L, name)(ctypes.c_long(n), *ptr[:3], ctypes.c_long(ns), *ptr[:3], ptr[3],
                                  ctypes.c_double(1e-4), ctypes.c_int(0), *ptr[3:], ctypes.c_void_p(0))
        assert status == 5
        assert "host memory" in L.sbslpm_last_error().decode()


def test_noalloc_refuses_sizes_beyond_its_scratch(sb):
    n = MAX_TARGETS + 1
    # buffers of the full size, so the call would stay in bounds even if it ran
    t = [torch.zeros(n, dtype=torch.float64, device="cuda") for _ in range(3)]
    out = [torch.zeros(n, dtype=torch.float64, device="cuda") for _ in range(3)]
    w = torch.zeros(4, dtype=torch.float64, device="cuda")
    L = sb.lib()
    status = L.sbslpm_direct_sum_bve_noalloc(
        ctypes.c_long(n), *[ctypes.c_void_p(a.data_ptr()) for a in t], ctypes.c_long(4),
        *[ctypes.c_void_p(a.data_ptr()) for a in (*t, w)], ctypes.c_double(1e-4), ctypes.c_int(0),
        *[ctypes.c_void_p(a.data_ptr()) for a in out], ctypes.c_void_p(0))
    assert status == 5
    assert "at most" in L.sbslpm_last_error().decode()
