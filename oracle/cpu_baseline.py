"""Time the reference's own CPU BVE step (test infrastructure: bench.py's
CPU-baseline leg and its ``--impl reference`` arm).

Runs bve_back_rk4_step from oracle/_ref/libsbslpm_ref.so (the reference's
unmodified sources built against the shim headers, OpenMP on every host
thread) -- or, where that library was not built, the C restatement
oracle/liboracle_port.so -- on the 6 x 4^(levels-1) panel cubed sphere with
4 x 4 points per panel (interp_degree 3), the Rossby-Haurwitz R=4 initial
condition, theta, kernel_eps 1e-4, and Omega = 2*pi, dt = 0.005 expressed in
the reference's integer seconds (time scaled by 200: dt = 1 s,
Omega = 2*pi/200, vorticity / 200).  Prints one JSON line.

    python -m oracle.cpu_baseline --levels 7 --steps 2 --warmup 1
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--levels", type=int, default=7)
    ap.add_argument("--theta", type=float, default=0.7)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--budget-s", type=float, default=240.0, help="stop timing steps after this much wall time")
    ap.add_argument("--kind", choices=["auto", "reference", "port"], default="auto")
    a = ap.parse_args(argv)

    threads = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    os.environ.setdefault("OMP_PROC_BIND", "close")
    os.environ.setdefault("OMP_PLACES", "cores")
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import numpy as np

    from oracle import pyoracle

    kind = a.kind
    if kind == "auto":
        kind = "reference" if os.path.exists(pyoracle.REF_PATH) else "port"
    omega_s = 2 * np.pi / 200.0
    d = 3
    if kind == "reference":
        ref = pyoracle.Ref()
        c = ref.create(a.levels, d, a.theta, 1e-4, omega_s, 1, 0)
        x, y, z, area, _ = ref.points(c)
        nthreads = int(ref.lib.ref_num_threads())

        def step(v):
            return ref.bve_step(c, v, None, nsteps=1)[0]
    else:
        port = pyoracle.Port()
        g = port.build(a.levels, d, a.theta, exact_cc=True)
        x, y, z, area = g["x"], g["y"], g["z"], g["area"]
        nthreads = int(os.environ["OMP_NUM_THREADS"])

        def step(v):
            return port.bve_step(g, v, None, dt=1.0, omega=omega_s, eps=1e-4, mode=0)[0]

    lat, lon = np.arcsin(np.clip(z, -1, 1)), np.arctan2(y, x)
    vor = (np.sin(lat) - 0.5 * np.sin(lat) * np.cos(lat) ** 4 * 30 * np.cos(4 * lon)) / 200.0
    vor -= (vor * area).sum() / (4 * np.pi)

    for _ in range(a.warmup):
        vor = step(vor)
    times = []
    t_all = time.perf_counter()
    for _ in range(a.steps):
        t0 = time.perf_counter()
        vor = step(vor)
        times.append(time.perf_counter() - t0)
        if time.perf_counter() - t_all > a.budget_s:
            break
    per = float(np.median(times))
    cpu = "unknown"
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                cpu = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    print(json.dumps({
        "kind": kind, "levels": a.levels, "particles": 6 * 4 ** (a.levels - 1) * (d + 1) ** 2,
        "steps_timed": len(times), "steps_requested": a.steps, "s_per_step_median": per,
        "steps_per_s": 1.0 / per, "threads": nthreads, "cpu": cpu, "finite": bool(np.isfinite(vor).all()),
    }))


if __name__ == "__main__":
    main()
