"""The Poisson FMM on the CPU: the oracle's restatement of
poisson_fmm_interactions and downward_pass against the reference's own outputs
(tests/golden/make_golden_poisson.py).  Tolerance <= 1e-13 relative (the
reference accumulates with atomics, the oracle in list order)."""
import os

import numpy as np
import pytest

from conftest import GOLDEN

CASES = ("poisson_L4.npz", "poisson_L3_d2.npz")


def rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.mark.parametrize("name", CASES)
def test_oracle_poisson_interactions_match_reference(port, name):
    gd = dict(np.load(os.path.join(GOLDEN, name)))
    g = port.build(int(gd["levels"]), int(gd["degree"]), float(gd["theta"]))
    assert np.array_equal(g["list"], gd["list"])
    out = port.poisson_fmm_interactions(g, gd["rand_source"], gd["rand_target_in"])
    assert rel(out, gd["rand_target_out"]) <= 1e-13
    tgt = port.poisson_fmm_interactions(g, gd["proxy_source"], np.zeros_like(gd["proxy_source"]))
    _, soln = port.downward_pass(g, tgt)
    assert rel(soln, gd["soln"]) <= 1e-13
