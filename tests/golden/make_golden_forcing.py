"""Generate the forced-BVE golden vectors (tests/golden/bve_forcing_L3.npz)
from the reference itself.

Runs the reference's own unmodified code (oracle/_ref/libsbslpm_ref.so, built
by ``make -C oracle ref`` from the reference checkout) with one OpenMP thread:
bve_back_rk4_step with RunConfig::forcing on (src/forcing_funcs.cpp:82-96),
levels 3, degree 3, theta 0.7, dt = 1 s, Omega = 2 pi, from the
Rossby-Haurwitz state:
  ssw  from t = 2 days, two steps (the ramp-up, src/forcing_funcs.cpp:27-28)
  ssw2 at t = 6 days, one step (the plateau)
  ssw  at t = 13.5 days, one step (the ramp-down)

Usage:  make -C oracle ref && python tests/golden/make_golden_forcing.py
"""
from __future__ import annotations

import os
import sys

os.environ["OMP_NUM_THREADS"] = "1"
HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import numpy as np  # noqa: E402

from oracle.pyoracle import Ref  # noqa: E402

DAY = 86400.0


def main():
    ref = Ref()
    c = ref.create(3, 3, 0.7, 1e-4, 2 * np.pi, 1, 0)
    x, y, z, area, interp = ref.points(c)
    vor = ref.initialize(c, "rh4", True)
    out = dict(levels=3, degree=3, theta=0.7, eps=1e-4, omega=2 * np.pi, dt=1.0, x=x, y=y, z=z, area=area,
               list=ref.interactions(c), ic=vor)
    for name, forcing, t0, n in (("ssw_ramp", 1, 2 * DAY, 2), ("ssw2_plateau", 2, 6 * DAY, 1),
                                 ("ssw_down", 1, 13.5 * DAY, 1)):
        ref.set_forcing(c, forcing)
        v, vel, _ = ref.bve_step(c, vor.copy(), None, time=t0, nsteps=n)
        out[name + "_forcing"], out[name + "_t0"], out[name + "_n"] = forcing, t0, n
        out[name + "_vors"], out[name + "_vel"] = v, np.stack(vel)
    ref.set_forcing(c, 0)
    v, vel, _ = ref.bve_step(c, vor.copy(), None, time=6 * DAY)
    out["unforced_vors"] = v
    ref.destroy(c)
    np.savez_compressed(os.path.join(HERE, "bve_forcing_L3.npz"), **out)
    print({k: np.shape(v) for k, v in out.items() if np.ndim(v)})
    print("forced vs unforced at 6 days: %.3e" % np.abs(out["ssw2_plateau_vors"] - v).max())


if __name__ == "__main__":
    main()
