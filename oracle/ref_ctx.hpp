// Shared context of the reference harness translation units (test
// infrastructure only): the reference's grid, tree and interaction list built
// once per configuration, held in the shim's host Views.
#pragma once

#include <Kokkos_Core.hpp>
#include <cstring>

#include "run_config.hpp"
#include "initialize_cubed_sphere.hpp"
#include "fmm_funcs.hpp"

namespace refh {
using V2 = Kokkos::View<double**, Kokkos::LayoutRight>;
using V2H = Kokkos::View<double**, Kokkos::LayoutRight, Kokkos::HostSpace>;
using V3 = Kokkos::View<double***, Kokkos::LayoutRight>;

struct RefCtx {
  RunConfig rc;
  Kokkos::View<CubedSpherePanel*, Kokkos::HostSpace> panels_h;
  Kokkos::View<CubedSpherePanel*> panels;
  V2H interp_h;
  V2 interp;
  V2H xcos_h, ycos_h, zcos_h, area_h;
  V2 xcos, ycos, zcos, area;
  Kokkos::View<interact_pair*, Kokkos::HostSpace> list_h;
  Kokkos::View<interact_pair*> list;
  V2 proxy_source;
  int q;
};

inline void copy_in(const V2& v, const double* src) { std::memcpy(v.data(), src, sizeof(double) * v.size()); }
inline void copy_out(const V2& v, double* dst) { std::memcpy(dst, v.data(), sizeof(double) * v.size()); }
}  // namespace refh
