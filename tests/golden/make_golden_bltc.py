"""Golden vectors of the treecode (decoupled proxy degree) from the reference.

Runs the reference's own irregular-point FMM functions (the "_ll" variants:
dual_tree_traversal_irreg, upward_pass_ll, swe_vel_interactions_ll with zero
divergence, downward_pass_3_ll; harness oracle/ref_harness_ll.cpp, library
oracle/_ref/libsbslpm_ref.so) with one OpenMP thread on the BVE particle grid
whose quadtree is truncated so that a leaf holds at most leaf_size particles,
and stores small cases as tests/golden/bltc_<name>.npz:

  list       the interaction list (target, source, type) of
             dual_tree_traversal_irreg on the truncated tree
  upward     proxy source strengths (tree panels x (n+1)^2) of the smooth
             field pots below, times the grid's quadrature weights
  down_out   downward_pass_3_ll of the proxy targets down_in() below, added
             into zero particle values (3 x A x q)
  vel        the velocity of the vorticity pots (3 x A x q): upward pass,
             typed interactions, downward pass
  vel_swe    the same with the divergence divs_of as the second source
             field (the rotational and divergent parts)

The inputs are smooth functions of the grid (pots) and of the panel and
proxy indices (down_in), defined in tests/golden/bltc_inputs.py and
recomputed by the tests from there.

Usage:  make -C oracle ref REF=<checkout> && python tests/golden/make_golden_bltc.py
"""
from __future__ import annotations

import os
import sys

os.environ["OMP_NUM_THREADS"] = "1"
HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import numpy as np  # noqa: E402

from oracle.pyoracle import Ref  # noqa: E402
from tests.golden.bltc_inputs import CASES, EPS, divs_of, down_in, pots_of  # noqa: E402

def main():
    ref = Ref()
    for name, (levels, degree, leaf, n, theta) in CASES.items():
        c = ref.create(levels, degree, 0.7, EPS, 1.0, 1, 0)
        x, y, z, area, _ = ref.points(c)
        ref.destroy(c)
        ll = ref.ll_create(levels, degree, leaf, n, theta, EPS)
        pots = pots_of(x, y, z)
        out = dict(levels=levels, degree=degree, leaf_size=leaf, proxy_degree=n, theta=theta, eps=EPS,
                   tree_levels=ll["Lf"], npl=ll["npl"], list=ref.ll_list(ll), upward=ref.ll_upward(ll, pots),
                   down_out=np.stack(ref.ll_downward(ll, *down_in(ll["Pf"], ll["qx"]))),
                   vel=np.stack(ref.ll_velocity(ll, pots)),
                   vel_swe=np.stack(ref.ll_velocity(ll, pots, divs_of(x, y, z))))
        ref.ll_destroy(ll)
        np.savez_compressed(os.path.join(HERE, f"bltc_{name}.npz"), **out)
        print(name, {k: getattr(v, "shape", v) for k, v in out.items()})


if __name__ == "__main__":
    main()
