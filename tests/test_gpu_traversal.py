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
