// sbslpm_kokkos.hpp -- C++ drop-in for the reference's BVE hot-path entry
// points, over the C ABI in sbslpm.h.
//
// The functions keep the reference's names and argument order and accept the
// caller's own View and RunConfig types (anything with data(), extent(i) and
// the reference's RunConfig field names), so a driver that calls
//   bve_back_rk4_step(run_config, xcos, ycos, zcos, area, vors,
//                     proxy_source_vors, interp_vals, cubed_sphere_panels,
//                     interaction_list, vel_x, vel_y, vel_z,
//                     passive_tracers, time);
// (reference: src/bve_time_step.hpp:7-13, called from
// executables/bve_time_evo.cpp:305) switches by including this header and
// `using sbslpm_kokkos::bve_back_rk4_step;`.  The Views are LayoutRight, in
// device memory (CudaSpace / CudaUVMSpace) or, for bve_back_rk4_step, in host
// memory (HostSpace: the reference's OpenMP build), where the step copies
// through sbslpm_bve_step_host; all Views of one call in the same space.  The
// other drop-ins take device Views only and throw on host ones.
//
// The panel table, interaction list and interpolation table the reference
// passes are rebuilt inside the library from run_config (they are functions
// of levels, interp_degree and fmm_theta alone) and only their sizes are
// checked.  proxy_source_vors is workspace in the reference and is not
// touched.  Errors throw std::runtime_error carrying sbslpm_last_error().
#pragma once

#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <tuple>

#include "sbslpm.h"

namespace sbslpm_kokkos {

struct CtxDeleter {
  void operator()(sbslpm_ctx* c) const { sbslpm_destroy(c); }
};

inline void check(sbslpm_status s, const char* where) {
  if (s != SBSLPM_OK)
    throw std::runtime_error(std::string(where) + ": " + sbslpm_status_string(s) + " (" + sbslpm_last_error() + ")");
}

// One context per distinct configuration, created on first use.
template <class RunConfig>
sbslpm_ctx* context_for(const RunConfig& rc, double dt, int velocity = SBSLPM_VEL_FMM,
                        int precision = SBSLPM_FP64) {
  using Key = std::tuple<int, int, double, double, double, double, int, int, int>;
  static std::map<Key, std::unique_ptr<sbslpm_ctx, CtxDeleter>> cache;
  Key k{rc.levels, rc.interp_degree, rc.fmm_theta, rc.kernel_eps, rc.omega, dt, rc.tracer_count, velocity,
        precision};
  auto it = cache.find(k);
  if (it != cache.end()) return it->second.get();
  sbslpm_config cfg;
  check(sbslpm_config_default(&cfg), "sbslpm_config_default");
  cfg.levels = rc.levels;
  cfg.interp_degree = rc.interp_degree;
  cfg.fmm_theta = rc.fmm_theta;
  cfg.kernel_eps = rc.kernel_eps;
  cfg.omega = rc.omega;
  cfg.dt = dt;
  cfg.tracer_count = rc.tracer_count;
  cfg.velocity = velocity;
  cfg.precision = precision;
  sbslpm_ctx* c = nullptr;
  check(sbslpm_create(&cfg, &c), "sbslpm_create");
  cache.emplace(k, std::unique_ptr<sbslpm_ctx, CtxDeleter>(c));
  return c;
}

// bve_back_rk4_step (src/bve_time_step.cpp:311-419).
template <class RunConfig, class V2, class VPanels, class VList, class V3>
void bve_back_rk4_step(const RunConfig& run_config, V2& xcos, V2& ycos, V2& zcos, V2& area, V2& vors,
                       V2& /*proxy_source_vors*/, V2& interp_vals, VPanels& cubed_sphere_panels,
                       VList& /*interaction_list*/, V2& vel_x, V2& vel_y, V2& vel_z, V3& passive_tracers,
                       double time) {
  sbslpm_ctx* c = context_for(run_config, static_cast<double>(run_config.delta_t));
  long sizes[4];
  check(sbslpm_get_sizes(c, sizes), "sbslpm_get_sizes");
  if ((long)cubed_sphere_panels.extent(0) != sizes[0] || (long)xcos.extent(0) != sizes[1] ||
      (long)xcos.extent(1) != sizes[2] || (long)interp_vals.extent(0) != sizes[2])
    throw std::runtime_error("bve_back_rk4_step: view sizes do not match run_config");
  double* tr = run_config.tracer_count > 0 ? passive_tracers.data() : nullptr;
  if (sbslpm_pointer_on_device(vors.data()) == 0)
    check(sbslpm_bve_step_host(c, xcos.data(), ycos.data(), zcos.data(), area.data(), vors.data(), vel_x.data(),
                               vel_y.data(), vel_z.data(), tr, time),
          "sbslpm_bve_step_host");
  else
    check(sbslpm_bve_step(c, xcos.data(), ycos.data(), zcos.data(), area.data(), vors.data(), vel_x.data(),
                          vel_y.data(), vel_z.data(), tr, time),
          "sbslpm_bve_step");
}

// swe_back_rk4_step_2 (src/swe_time_step_2.cpp:785-1035; declared in
// src/swe_time_step_2.hpp:7-14, called from executables/swe_time_evo.cpp:415).
// The grid-point map the reference passes (one_d_no_of_points, two_d_to_1d)
// is rebuilt inside the library from the same grid; only its size is checked.
// The library's g/a is the reference's hard-coded 9.81/6371000.
template <class RunConfig, class V2, class VPanels, class VList, class V3, class VI1, class VI2>
void swe_back_rk4_step_2(const RunConfig& run_config, V2& xcos, V2& ycos, V2& zcos, V2& area, V2& vors, V2& divs,
                         V2& height, V2& interp_vals, VPanels& cubed_sphere_panels, VList& /*interaction_list*/,
                         V2& vel_x, V2& vel_y, V2& vel_z, V3& passive_tracers, V2& base_vor_tend, V2& base_div_tend,
                         V2& base_h_tend, VI1& one_d_no_of_points, VI2& two_d_to_1d, double time) {
  sbslpm_ctx* c = context_for(run_config, static_cast<double>(run_config.delta_t));
  long sizes[4];
  check(sbslpm_get_sizes(c, sizes), "sbslpm_get_sizes");
  if ((long)cubed_sphere_panels.extent(0) != sizes[0] || (long)xcos.extent(0) != sizes[1] ||
      (long)xcos.extent(1) != sizes[2] || (long)interp_vals.extent(0) != sizes[2] ||
      (long)two_d_to_1d.extent(0) != sizes[1] || (long)one_d_no_of_points.extent(0) < 1)
    throw std::runtime_error("swe_back_rk4_step_2: view sizes do not match run_config");
  double* tr = run_config.tracer_count > 0 ? passive_tracers.data() : nullptr;
  check(sbslpm_swe_step(c, xcos.data(), ycos.data(), zcos.data(), area.data(), vors.data(), divs.data(),
                        height.data(), vel_x.data(), vel_y.data(), vel_z.data(), tr, base_vor_tend.data(),
                        base_div_tend.data(), base_h_tend.data(), time),
        "sbslpm_swe_step");
}

// unify_boundary_vals (src/initialize_cubed_sphere.cpp:364-370).
template <class RunConfig, class VI1, class VI2, class V2>
void unify_boundary_vals(const RunConfig& run_config, VI1& /*one_d_no_of_points*/, VI2& /*two_d_to_1d*/, V2& vals) {
  sbslpm_ctx* c = context_for(run_config, static_cast<double>(run_config.delta_t));
  check(sbslpm_unify_boundary_vals(c, vals.data()), "sbslpm_unify_boundary_vals");
}

// direct_sum_inv_lap (src/direct_sum.cpp:8-15) over the caller's row block
// [oned_lb, oned_ub) as the reference does; with one GPU the block is usually
// all points.  The reference then all-reduces soln across ranks.
template <class RunConfig, class V1>
void direct_sum_inv_lap(const RunConfig& run_config, V1 xcos, V1 ycos, V1 zcos, V1 area, V1 pots, V1 soln) {
  long n = (long)xcos.extent(0);
  if (run_config.oned_lb != 0 || run_config.oned_ub != n)
    throw std::runtime_error("direct_sum_inv_lap: one-GPU version sums all rows; set oned_lb=0, oned_ub=n");
  check(sbslpm_direct_sum_inv_lap(n, xcos.data(), ycos.data(), zcos.data(), area.data(), pots.data(), soln.data(),
                                  nullptr),
        "sbslpm_direct_sum_inv_lap");
}

// poisson_fmm_interactions (src/fmm_interactions/inverse_poisson.cpp:9-34,
// called from executables/poisson_eq_fmm.cpp:148): target_pots += the log
// kernel over the interaction list, which the library rebuilds from run_config.
template <class RunConfig, class V2, class VList, class VPanels>
void poisson_fmm_interactions(const RunConfig& run_config, V2& target_pots, V2& source_vals,
                              VList& /*interaction_list*/, VPanels cubed_sphere_panels, V2& interp_vals) {
  sbslpm_ctx* c = context_for(run_config, 1.0);
  long sizes[4];
  check(sbslpm_get_sizes(c, sizes), "sbslpm_get_sizes");
  if ((long)cubed_sphere_panels.extent(0) != sizes[0] || (long)target_pots.extent(0) != sizes[0] ||
      (long)interp_vals.extent(0) != sizes[2])
    throw std::runtime_error("poisson_fmm_interactions: view sizes do not match run_config");
  check(sbslpm_poisson_fmm_interactions(c, source_vals.data(), target_pots.data()),
        "sbslpm_poisson_fmm_interactions");
}

// downward_pass (src/fmm_funcs.cpp:357-372, called from
// executables/poisson_eq_fmm.cpp:156).
template <class RunConfig, class V2, class VPanels>
void downward_pass(const RunConfig& run_config, V2& interp_vals, VPanels cubed_sphere_panels, V2& proxy_target_pots,
                   V2& sols) {
  sbslpm_ctx* c = context_for(run_config, 1.0);
  long sizes[4];
  check(sbslpm_get_sizes(c, sizes), "sbslpm_get_sizes");
  if ((long)cubed_sphere_panels.extent(0) != sizes[0] || (long)sols.extent(0) != sizes[1] ||
      (long)interp_vals.extent(0) != sizes[2])
    throw std::runtime_error("downward_pass: view sizes do not match run_config");
  check(sbslpm_downward_pass(c, proxy_target_pots.data(), sols.data()), "sbslpm_downward_pass");
}

}  // namespace sbslpm_kokkos
