"""Generate the Poisson FMM golden vectors (tests/golden/poisson_L4.npz,
poisson_L3_d2.npz) from the reference itself.

Runs the reference's own unmodified code (oracle/_ref/libsbslpm_ref.so, built
by ``make -C oracle ref`` from the reference checkout) with one OpenMP thread:
the solve of executables/poisson_eq_fmm.cpp:128-160 (upward_pass,
poisson_fmm_interactions, downward_pass) on the sh43 potential
(src/initial_conditions.cpp:52-66: 3/4 sqrt(35/(2 pi)) x (x^2 - 3 y^2) z, a
degree-4 spherical harmonic whose inverse Laplacian is -f/20), and
poisson_fmm_interactions alone on seeded random proxy values.

Usage:  make -C oracle ref && python tests/golden/make_golden_poisson.py
"""
from __future__ import annotations

import os
import sys

os.environ["OMP_NUM_THREADS"] = "1"
HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import numpy as np  # noqa: E402

from oracle.pyoracle import Ref  # noqa: E402


def case(ref, levels, degree, theta, seed):
    c = ref.create(levels, degree, theta, 1e-4, 2 * np.pi, 1, 0)
    x, y, z, area, interp = ref.points(c)
    pots = 1.770130769779931 * x * (x * x - 3.0 * y * y) * z
    src, tgt, soln = ref.poisson_fmm(c, pots)
    rng = np.random.default_rng(seed)
    r_src, r_tgt = rng.standard_normal((c["P"], c["q"])), rng.standard_normal((c["P"], c["q"]))
    out = dict(levels=levels, degree=degree, theta=theta, x=x, y=y, z=z, area=area, list=ref.interactions(c),
               pots=pots, proxy_source=src, proxy_target=tgt, soln=soln, rand_source=r_src, rand_target_in=r_tgt,
               rand_target_out=ref.poisson_fmm_interactions(c, r_src, r_tgt))
    ref.destroy(c)
    return out


def main():
    ref = Ref()
    for name, levels, degree, theta, seed in (("poisson_L4", 4, 3, 0.7, 1), ("poisson_L3_d2", 3, 2, 0.5, 2)):
        out = case(ref, levels, degree, theta, seed)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        rel = np.abs(out["soln"] + out["pots"] / 20).max() / np.abs(out["pots"] / 20).max()
        print(name, "soln vs -f/20: %.2e" % rel)


if __name__ == "__main__":
    main()
