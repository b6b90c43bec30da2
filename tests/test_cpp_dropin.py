"""The C++ drop-in header compiles against a Kokkos-style View type and a
RunConfig with the reference's field names, links against libsbslpm.so and
reaches the C ABI.  Runs on the CPU: without a GPU the context creation
reports SBSLPM_ERR_NO_DEVICE, which the header turns into an exception."""
import os
import shutil
import subprocess
import textwrap

import pytest

from conftest import ROOT

PROGRAM = textwrap.dedent(r"""
    #include <Kokkos_Core.hpp>
    #include <cstdio>
    #include <string>
    #include "sbslpm_kokkos.hpp"

    // The reference's RunConfig fields used by the hot path (src/run_config.hpp).
    struct RunConfig {
      int levels = 3, interp_degree = 3, delta_t = 1, tracer_count = 0, oned_lb = 0, oned_ub = 0;
      double fmm_theta = 0.7, kernel_eps = 1e-4, omega = 0.0314;
    };
    struct CubedSpherePanel { int id; };
    struct interact_pair { int target_panel, source_panel, interact_type; };

    int main() {
      RunConfig rc;
      using V2 = Kokkos::View<double**, Kokkos::LayoutRight>;
      V2 x("x", 96, 16), y("y", 96, 16), z("z", 96, 16), area("a", 96, 16), vors("v", 96, 16),
         proxy("p", 126, 16), interp("i", 16, 4), vx("vx", 96, 16), vy("vy", 96, 16), vz("vz", 96, 16);
      Kokkos::View<CubedSpherePanel*> panels("panels", 126);
      Kokkos::View<interact_pair*> list("list", 1);
      Kokkos::View<double***, Kokkos::LayoutRight> tracers("t", 96, 16, 1);
      try {
        sbslpm_kokkos::bve_back_rk4_step(rc, x, y, z, area, vors, proxy, interp, panels, list, vx, vy, vz,
                                         tracers, 0.0);
        std::printf("stepped\n");
      } catch (const std::exception& e) {
        std::printf("exception: %s\n", e.what());
      }
      // swe_back_rk4_step_2 with the reference's argument list
      V2 divs("d", 96, 16), height("h", 96, 16), bv("bv", 96, 16), bd("bd", 96, 16), bh("bh", 96, 16);
      Kokkos::View<int*> counts("counts", 96 * 9 + 2);
      Kokkos::View<int**, Kokkos::LayoutRight> map("map", 96, 16);
      try {
        sbslpm_kokkos::swe_back_rk4_step_2(rc, x, y, z, area, vors, divs, height, interp, panels, list, vx, vy, vz,
                                           tracers, bv, bd, bh, counts, map, 0.0);
        std::printf("swe stepped\n");
      } catch (const std::exception& e) {
        std::printf("swe exception: %s\n", e.what());
      }
      // the Poisson FMM driver's calls (executables/poisson_eq_fmm.cpp:148-156)
      V2 ptgt("pt", 126, 16), psrc("ps", 126, 16), soln("s", 96, 16);
      try {
        sbslpm_kokkos::poisson_fmm_interactions(rc, ptgt, psrc, list, panels, interp);
        sbslpm_kokkos::downward_pass(rc, interp, panels, ptgt, soln);
        std::printf("poisson solved\n");
      } catch (const std::exception& e) {
        std::printf("poisson exception: %s\n", e.what());
      }
      return 0;
    }
""")


def test_cpp_dropin_header_compiles_and_reaches_the_abi(sb, tmp_path):
    gxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else shutil.which("g++")
    src = tmp_path / "dropin.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "dropin"
    libdir = os.path.dirname(sb.library_path())
    subprocess.run([gxx, "-std=c++17", "-O1", "-w", f"-I{ROOT}/include", f"-I{ROOT}/oracle/shim", str(src),
                    f"-L{libdir}", "-lsbslpm", f"-Wl,-rpath,{libdir}", "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present; this test checks the CPU-side path only")
    assert "exception: sbslpm_create" in out.stdout and "no CUDA device" in out.stdout, out.stdout
    assert "swe exception: sbslpm_create" in out.stdout, out.stdout
    assert "poisson exception: sbslpm_create" in out.stdout, out.stdout
