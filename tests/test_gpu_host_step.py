"""GPU tests of the step on host arrays (sbslpm_bve_step_host): the same
kernels as the device-pointer step, so the results are bit-identical to it,
whether the host arrays are pageable numpy arrays or pinned tensors, with
and without tracers, for the treecode and the spectral FMM; and the C++
drop-in header on HostSpace Views (the reference's OpenMP build) routes
through it."""
import os
import shutil
import subprocess
import textwrap

import numpy as np
import pytest

from conftest import ROOT
from test_gpu_bve import unit_sphere_rh4

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

ERR_ARG = 5  # SBSLPM_ERR_ARG


def device_step(ctx, g, vor, tracers=None, time=0.0):
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    v = T(vor)
    vel = [torch.zeros_like(v) for _ in range(3)]
    tr = T(tracers) if tracers is not None else None
    ctx.bve_back_rk4_step(T(g.x), T(g.y), T(g.z), T(g.area), v, *vel, tr, time=time)
    return v.cpu().numpy(), [u.cpu().numpy() for u in vel], (tr.cpu().numpy() if tr is not None else None)


def host_step(ctx, g, vor, tracers=None, pinned=False, time=0.0):
    if pinned:  # a fresh pinned copy (pin_memory() of memory that is pinned already returns it)
        H = lambda a: torch.from_numpy(np.array(a, dtype=np.float64, order="C", copy=True)).pin_memory()
        out = lambda t: t.numpy().copy()
    else:
        H = lambda a: np.ascontiguousarray(a, dtype=np.float64).copy()
        out = lambda a: a
    v = H(vor)
    vel = [H(np.zeros_like(vor)) for _ in range(3)]
    tr = H(tracers) if tracers is not None else None
    ctx.bve_back_rk4_step_host(H(g.x), H(g.y), H(g.z), H(g.area), v, *vel, tr, time=time)
    return out(v), [out(u) for u in vel], (out(tr) if tr is not None else None)


@pytest.mark.parametrize("pinned", [False, True])
@pytest.mark.parametrize("case", ["treecode_mixed", "spectral_fp64_tracers", "direct_fp64"])
def test_host_step_is_the_device_step(sb, case, pinned):
    levels = 5 if case == "treecode_mixed" else 4
    g = sb.build_grid(levels, 3, exact_cc=True)
    vor = unit_sphere_rh4(g)
    kw = dict(levels=levels, interp_degree=3, fmm_theta=0.7, kernel_eps=1e-4, omega=2 * np.pi, dt=0.005)
    tracers = None
    if case == "treecode_mixed":
        kw.update(precision=sb.MIXED, proxy_degree=8, leaf_size=256)
    elif case == "spectral_fp64_tracers":
        kw.update(tracer_count=2)
        tracers = np.stack([g.z, g.x * g.y], axis=-1)
    else:
        kw.update(velocity=sb.VEL_DIRECT)
    ctx = sb.Context(sb.config_default(**kw))
    if case == "treecode_mixed":
        ctx.set_near_tuning(128, 2, 2)
        ctx.set_cc_tuning(3, 2)
    a = device_step(ctx, g, vor, tracers)
    b = host_step(ctx, g, vor, tracers, pinned)
    assert np.array_equal(a[0], b[0])
    assert all(np.array_equal(x, y) for x, y in zip(a[1], b[1]))
    if tracers is not None:
        assert np.array_equal(a[2], b[2])
    # a second call reuses the context's host-step buffers
    again = b[0].copy()
    c = host_step(ctx, g, again, tracers, pinned)
    d = device_step(ctx, g, again, tracers)
    assert np.array_equal(c[0], d[0])


@pytest.mark.parametrize("case", ["treecode_mixed", "spectral_fp64_tracers"])
def test_repeated_pinned_host_steps_replay_as_a_graph(sb, case):
    """The same pinned arrays stepped again and again: after the first (eager)
    call the step and its copies replay as one captured CUDA graph; every
    step stays bit-identical to the device step, also after the launch shape
    changes (the captured graph is dropped and captured again)."""
    levels = 5 if case == "treecode_mixed" else 4
    g = sb.build_grid(levels, 3, exact_cc=True)
    vor = unit_sphere_rh4(g)
    kw = dict(levels=levels, interp_degree=3, fmm_theta=0.7, kernel_eps=1e-4, omega=2 * np.pi, dt=0.005)
    tracers = None
    if case == "treecode_mixed":
        kw.update(precision=sb.MIXED, proxy_degree=8, leaf_size=256)
    else:
        kw.update(tracer_count=2)
        tracers = np.stack([g.z, g.x * g.y], axis=-1)
    ctx = sb.Context(sb.config_default(**kw))
    if case == "treecode_mixed":
        ctx.set_near_tuning(128, 2, 2)
        ctx.set_cc_tuning(3, 2)
    P = lambda a: torch.from_numpy(np.array(a, dtype=np.float64, order="C", copy=True)).pin_memory()
    hv, hvel = P(vor), [P(np.zeros_like(vor)) for _ in range(3)]
    htr = P(tracers) if tracers is not None else None
    hx = [P(a) for a in (g.x, g.y, g.z, g.area)]
    dv, dtr = vor.copy(), (tracers.copy() if tracers is not None else None)
    launches = []
    for k in range(4):
        if k == 2 and case == "treecode_mixed":
            ctx.set_near_tuning(256, 1, 3)
        l0 = sb.kernel_launches()
        ctx.bve_back_rk4_step_host(*hx, hv, *hvel, htr)
        launches.append(sb.kernel_launches() - l0)
        dv, dvel, dtr = device_step(ctx, g, dv, dtr)
        assert np.array_equal(hv.numpy(), dv), k
        assert all(np.array_equal(h.numpy(), u) for h, u in zip(hvel, dvel)), k
        if tracers is not None:
            assert np.array_equal(htr.numpy(), dtr), k
    assert launches[1] == launches[0] > 0  # a replay counts the captured kernels


def test_host_step_rejects_device_and_misshaped_arrays(sb):
    g = sb.build_grid(3, 3, exact_cc=True)
    ctx = sb.Context(sb.config_default(levels=3, interp_degree=3, kernel_eps=1e-4))
    H = lambda a: np.ascontiguousarray(a, dtype=np.float64).copy()
    args = [H(g.x), H(g.y), H(g.z), H(g.area), H(unit_sphere_rh4(g))] + [H(np.zeros_like(g.x)) for _ in range(3)]
    bad = list(args)
    bad[0] = torch.from_numpy(args[0]).cuda()
    with pytest.raises(TypeError):
        ctx.bve_back_rk4_step_host(*bad)
    bad = list(args)
    bad[4] = args[4][:, :8].copy()
    with pytest.raises(ValueError):
        ctx.bve_back_rk4_step_host(*bad)


def test_device_entry_points_refuse_host_memory(sb):
    """sbslpm_bve_step / _run given host arrays return SBSLPM_ERR_ARG instead
    of handing host memory to the kernels; the context stays usable."""
    import ctypes

    g = sb.build_grid(3, 3, exact_cc=True)
    ctx = sb.Context(sb.config_default(levels=3, interp_degree=3, kernel_eps=1e-4))
    H = lambda a: np.ascontiguousarray(a, dtype=np.float64).copy()
    host = [H(g.x), H(g.y), H(g.z), H(g.area), H(unit_sphere_rh4(g))] + [H(np.zeros_like(g.x)) for _ in range(3)]
    L = sb.lib()
    st = L.sbslpm_bve_step(ctx._h, *[a.ctypes.data for a in host], None, ctypes.c_double(0.0))
    assert st == ERR_ARG and b"host memory" in L.sbslpm_last_error()
    st = L.sbslpm_bve_run(ctx._h, *[a.ctypes.data for a in host], None, ctypes.c_double(0.0), 1)
    assert st == ERR_ARG
    a = device_step(ctx, g, unit_sphere_rh4(g))  # still steps on device memory
    assert np.isfinite(a[0]).all()


def test_pointer_on_device(sb):
    d = torch.zeros(8, dtype=torch.float64, device="cuda")
    h = np.zeros(8)
    p = torch.zeros(8, dtype=torch.float64).pin_memory()
    assert sb.pointer_on_device(d.data_ptr()) == 1
    assert sb.pointer_on_device(h.ctypes.data) == 0
    assert sb.pointer_on_device(p.data_ptr()) == 0


PROGRAM = textwrap.dedent(r"""
    #include <Kokkos_Core.hpp>
    #include <cstdio>
    #include "sbslpm_kokkos.hpp"

    struct RunConfig {
      int levels = 4, interp_degree = 3, delta_t = 1, tracer_count = 0;
      double fmm_theta = 0.7, kernel_eps = 1e-4, omega = 0.0314;
    };
    struct CubedSpherePanel { int id; };
    struct interact_pair { int target_panel, source_panel, interact_type; };

    int main(int argc, char** argv) {
      const int A = 384, q = 16, P = 510;
      using V2 = Kokkos::View<double**, Kokkos::LayoutRight>;
      V2 x("x", A, q), y("y", A, q), z("z", A, q), area("a", A, q), vors("v", A, q), proxy("p", P, q),
         interp("i", q, 4), vx("vx", A, q), vy("vy", A, q), vz("vz", A, q);
      Kokkos::View<CubedSpherePanel*> panels("panels", P);
      Kokkos::View<interact_pair*> list("list", 1);
      Kokkos::View<double***, Kokkos::LayoutRight> tracers("t", A, q, 1);
      FILE* f = std::fopen(argv[1], "rb");
      for (V2* v : {&x, &y, &z, &area, &vors})
        if (std::fread(v->data(), sizeof(double), A * q, f) != (size_t)(A * q)) return 2;
      std::fclose(f);
      RunConfig rc;
      sbslpm_kokkos::bve_back_rk4_step(rc, x, y, z, area, vors, proxy, interp, panels, list, vx, vy, vz, tracers,
                                       0.0);
      f = std::fopen(argv[2], "wb");
      for (V2* v : {&vors, &vx, &vy, &vz}) std::fwrite(v->data(), sizeof(double), A * q, f);
      std::fclose(f);
      std::printf("stepped\n");
      return 0;
    }
""")


def test_cpp_dropin_steps_host_views(sb, tmp_path):
    """The reference's call on HostSpace Views, through the drop-in header:
    the same result as the device step of a context with the same RunConfig
    (levels 4, degree 3, theta 0.7, eps 1e-4, omega 0.0314, dt 1 s)."""
    gxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else shutil.which("g++")
    src = tmp_path / "dropin_host.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "dropin_host"
    libdir = os.path.dirname(sb.library_path())
    subprocess.run([gxx, "-std=c++17", "-O1", "-w", f"-I{ROOT}/include", f"-I{ROOT}/oracle/shim", str(src),
                    f"-L{libdir}", "-lsbslpm", f"-Wl,-rpath,{libdir}", "-o", str(exe)], check=True)
    g = sb.build_grid(4, 3, exact_cc=True)
    vor = unit_sphere_rh4(g)
    inp, outp = tmp_path / "in.bin", tmp_path / "out.bin"
    np.concatenate([np.ascontiguousarray(a, dtype=np.float64).ravel() for a in (g.x, g.y, g.z, g.area, vor)]).tofile(
        inp)
    run = subprocess.run([str(exe), str(inp), str(outp)], capture_output=True, text=True, timeout=300)
    assert run.returncode == 0 and "stepped" in run.stdout, run.stdout + run.stderr
    got = np.fromfile(outp, dtype=np.float64).reshape(4, *g.x.shape)
    ctx = sb.Context(sb.config_default(levels=4, interp_degree=3, fmm_theta=0.7, kernel_eps=1e-4, omega=0.0314,
                                       dt=1.0))
    v, vel, _ = device_step(ctx, g, vor)
    assert np.array_equal(got[0], v)
    assert all(np.array_equal(got[1 + k], vel[k]) for k in range(3))
