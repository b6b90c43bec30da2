"""Height drift of the reference's own shallow-water step on the benchmark flow.

Runs the reference's unmodified swe_back_rk4_step_2 (oracle/_ref/libsbslpm_ref.so,
src/swe_time_step_2.cpp:785-1035, plus the driver's unify of vorticity,
divergence and height after each step, executables/swe_time_evo.cpp:415-418)
on the benchmark's unit-sphere flow: steady geostrophic solid-body rotation
(Omega = 2 pi, u0 = 2 pi/12, g h = 2.94 - (Omega u0 + u0^2/2) sin^2 lat) with
seeded N(0, 1e-4^2) noise on g h (numpy default_rng(4), the benchmark's draw),
dt = 0.002, spectral FMM at theta 0.7 with degree-3 panels, kernel_eps 1e-4,
and the exact Clenshaw-Curtis quadrature weights the benchmark uses (set
through ref_set_area; the reference's own weights for degree 3 sum to 3.88).
Time is scaled by 500 so that dt is one integer second (the reference keeps
delta_t an int): Omega' = Omega/500, vorticity and divergence /500, height
h' = (g h)/500^2/(9.81/6371000).  The relative L2 drift of the height is
scale-free, so it compares directly with the unit-sphere run.

Prints, every 10 steps, the area-weighted relative L2 height drift
|h - h0| / |h0| until the run becomes non-finite or reaches the last step,
and writes the curve so far to tests/golden/swe_drift_reference_L<levels>.json
after every 10 steps (the reference stops the process with Kokkos::abort when
a non-finite departure point reaches its point location, so the file holds
the curve up to the last finite state; "stopped" records the abort).

Usage:  make -C oracle ref REF=<checkout> &&
        OMP_NUM_THREADS=<n> python tests/golden/swe_drift_reference.py <levels> [<steps>]
"""
from __future__ import annotations

import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import numpy as np  # noqa: E402

from oracle.pyoracle import Port, Ref  # noqa: E402

S = 500.0
G_OVER_A = 9.81 / 6371000.0
EPS = 1e-4


def unit_flow(z):
    om, u0 = 2 * np.pi, 2 * np.pi / 12
    lat = np.arcsin(np.clip(z, -1, 1))
    vors = 2 * u0 * np.sin(lat)
    gh = 2.94 - (om * u0 + 0.5 * u0 * u0) * np.sin(lat) ** 2
    gh = gh + 1e-4 * np.random.default_rng(4).standard_normal(gh.shape)
    return vors, gh


def main():
    levels = int(sys.argv[1]) if len(sys.argv) > 1 else 6
    nsteps = int(sys.argv[2]) if len(sys.argv) > 2 else 100
    ref = Ref()
    c = ref.create(levels, 3, 0.7, EPS, 2 * np.pi / S, 1, 0)
    x, y, z, area, _ = ref.points(c)
    exact = Port().build(levels, 3, None, exact_cc=True)
    assert np.array_equal(exact["x"], x) and np.array_equal(exact["z"], z)
    area = exact["area"]
    ref.set_area(c, area)
    smap = ref.swe_map(c)
    vors, gh = unit_flow(z)
    vors, divs, height = vors / S, np.zeros_like(vors), gh / S ** 2 / G_OVER_A
    vel, base = ref.swe_init(c, vors, divs, height, smap)
    w = area / area.sum()
    h0 = height.copy()
    l2 = lambda a: float(np.sqrt((w * a * a).sum()))
    out = {"levels": levels, "particles": int(x.size), "threads": ref.lib.ref_num_threads(), "dt": 0.002,
           "time_scale": S, "theta": 0.7, "degree": 3, "kernel_eps": EPS, "noise_seed": 4, "curve": []}
    path = os.path.join(HERE, f"swe_drift_reference_L{levels}.json")
    done, t0 = 0, time.time()
    while done < nsteps:
        # what the file says if the reference stops the process in this chunk
        out["stopped"] = (f"Kokkos::abort (point location of a non-finite departure point) after step {done}, "
                          f"before step {done + 10}")
        with open(path, "w") as f:
            json.dump(out, f, indent=1)
        vors, divs, height, vel, _ = ref.swe_step(c, vors, divs, height, base, smap, vel=vel, time=float(done),
                                                   nsteps=10, driver_unify=True)
        done += 10
        finite = bool(np.isfinite(height).all())
        drift = l2(height - h0) / l2(h0) if finite else None
        out["curve"].append({"step": done, "height_l2_drift": drift})
        if done >= nsteps or not finite:
            out["stopped"] = None if finite else f"non-finite height at step {done}"
        print(f"levels {levels} step {done}: drift {drift}  ({time.time() - t0:.0f} s)", flush=True)
        with open(path, "w") as f:
            json.dump(out, f, indent=1)
        if not finite:
            break
    ref.destroy(c)


if __name__ == "__main__":
    main()
