"""The dual tree traversal on the GPU (sbslpm_dual_tree_traversal_device)
against the host traversal, whose list is the reference's in the reference's
order (tests/test_cabi_host.py pins it to the reference's own output): the
same pairs, types and order, bit for bit, over tree depths and MAC
parameters, including the levels-7 list of the benchmark (1,224,342 pairs at
theta 0.7)."""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
pytest.importorskip("torch")


@pytest.mark.parametrize("levels,theta", [(1, 0.7), (3, 0.5), (4, 0.7), (5, 0.3), (5, 0.9), (6, 0.7), (7, 0.7)])
def test_device_traversal_equals_reference_order(sb, levels, theta):
    panels = sb.cubed_sphere_panels_init(levels)
    t0 = time.perf_counter()
    host = sb.dual_tree_traversal(levels, panels, theta)
    t1 = time.perf_counter()
    dev = sb.dual_tree_traversal(levels, panels, theta, device=True)
    t2 = time.perf_counter()
    print("levels %d theta %.1f: %d pairs, host %.3f s, device %.3f s" % (levels, theta, len(host), t1 - t0, t2 - t1))
    assert dev.shape == host.shape
    assert np.array_equal(dev, host)
    if (levels, theta) == (7, 0.7):
        assert len(host) == 1224342


@pytest.mark.parametrize("levels", [3, 4, 5])
def test_treecode_lists_of_many_members_in_one_launch_series(sb, levels):
    """The treecode's traversal (its tree is the grid's quadtree truncated at
    the leaf size: levels 3..5 here, the ensemble's tree at 98,304 particles
    being levels 4) for 128 members with their own theta, on the GPU in one
    launch series: every member's list, order and near flags equal the host
    traversal's, bit for bit."""
    panels = sb.cubed_sphere_panels_init(levels)
    thetas = np.random.default_rng(2026).uniform(0.5, 0.8, 128)
    t0 = time.perf_counter()
    dev = sb.dual_tree_traversal_device_multi(levels, panels, thetas)
    t1 = time.perf_counter()
    host = [sb.dual_tree_traversal_flagged(levels, panels, th) for th in thetas]
    t2 = time.perf_counter()
    print("levels %d, 128 members: %d pairs, device %.3f s, host %.3f s"
          % (levels, sum(len(h[0]) for h in host), t1 - t0, t2 - t1))
    for (dl, dn), (hl, hn), th in zip(dev, host, thetas):
        assert np.array_equal(dl, hl), th
        assert np.array_equal(dn, hn), th
        assert np.array_equal(hl, sb.dual_tree_traversal(levels, panels, th))  # the same list as the unflagged one
