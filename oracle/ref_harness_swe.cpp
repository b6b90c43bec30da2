// Harness around the reference's own shallow-water (SWE v2) hot-path code
// (test infrastructure only).  Compiled with the reference's unmodified
// src/*.cpp against oracle/shim/ into oracle/_ref/libsbslpm_ref.so (recipe:
// oracle/Makefile).  Entry points:
//   cubed_sphere_2d_to_1d, unify_boundary_vals
//                                  (src/initialize_cubed_sphere.cpp:290-370)
//   swe_vel_interactions_2         (src/fmm_interactions/swe_vel.cpp:39-67)
//   swe_tendency_computation_2     (src/swe_time_step_2_impl.hpp:10-128)
//   the driver's initial velocity + base tendencies
//                                  (executables/swe_time_evo.cpp:352-410)
//   swe_back_rk4_step_2 (+ the driver's unify of vors/divs/height)
//                                  (src/swe_time_step_2.cpp:785-1035,
//                                   executables/swe_time_evo.cpp:415-418)
// src/swe_time_step_2.cpp is included textually (unmodified) so that its
// file-local functors are visible.  The reference prints to stdout inside the
// step (a device View at src/swe_time_step_2.cpp:821-823) and in
// cubed_sphere_2d_to_1d; those calls run with stdout sent to /dev/null.
#include <fcntl.h>
#include <unistd.h>

#include <cstdio>
#include <iostream>

#include "swe_time_step_2.cpp"
#include "ref_ctx.hpp"

using namespace refh;

namespace {
struct Quiet {
  int saved;
  Quiet() {
    std::cout.flush();
    std::fflush(stdout);
    saved = dup(1);
    int fd = open("/dev/null", O_WRONLY);
    dup2(fd, 1);
    close(fd);
  }
  ~Quiet() {
    std::cout.flush();
    std::fflush(stdout);
    dup2(saved, 1);
    close(saved);
  }
};

struct Map {
  Kokkos::View<int*> counts;
  Kokkos::View<int**, Kokkos::LayoutRight> two_d;
};

Map make_map(RefCtx* c, const int* two_d_to_1d, const int* counts) {
  Map m;
  int A = c->rc.active_panel_count, U = c->rc.point_count;
  m.counts = Kokkos::View<int*>("counts", U);
  m.two_d = Kokkos::View<int**, Kokkos::LayoutRight>("map", A, c->q);
  std::memcpy(m.counts.data(), counts, sizeof(int) * U);
  std::memcpy(m.two_d.data(), two_d_to_1d, sizeof(int) * A * c->q);
  return m;
}
}  // namespace

extern "C" {

// cubed_sphere_2d_to_1d over the grid: two_d_to_1d (A x q) and counts (U).
// Returns U, the number of distinct points.
int ref_swe_map(void* h, int* two_d_to_1d, int* counts) {
  RefCtx* c = static_cast<RefCtx*>(h);
  int A = c->rc.active_panel_count, U = c->rc.point_count;
  Kokkos::View<double*, Kokkos::HostSpace> x1("x1", U), y1("y1", U), z1("z1", U);
  Kokkos::View<int*, Kokkos::HostSpace> n1("n1", U);
  Kokkos::View<int**, Kokkos::LayoutRight, Kokkos::HostSpace> m("m", A, c->q);
  {
    Quiet quiet;
    cubed_sphere_2d_to_1d(c->rc, x1, y1, z1, n1, m, c->xcos_h, c->ycos_h, c->zcos_h);
  }
  std::memcpy(two_d_to_1d, m.data(), sizeof(int) * A * c->q);
  std::memcpy(counts, n1.data(), sizeof(int) * U);
  return U;
}

void ref_unify(void* h, double* vals, const int* two_d_to_1d, const int* counts) {
  RefCtx* c = static_cast<RefCtx*>(h);
  Map m = make_map(c, two_d_to_1d, counts);
  V2 v("v", c->rc.active_panel_count, c->q);
  copy_in(v, vals);
  unify_boundary_vals(c->rc, m.counts, m.two_d, v);
  copy_out(v, vals);
}

// One pass of swe_vel_interactions_2 over the whole list.  disp_* and the two
// source fields: P x q; out_1..3 (P x q) are accumulated into.
void ref_swe_vel_interactions(void* h, const double* disp_x, const double* disp_y, const double* disp_z,
                              const double* src_vor, const double* src_div, double* out_1, double* out_2,
                              double* out_3) {
  RefCtx* c = static_cast<RefCtx*>(h);
  int P = c->rc.panel_count, q = c->q;
  V2 dx("dx", P, q), dy("dy", P, q), dz("dz", P, q), sv("sv", P, q), sd("sd", P, q), t1("t1", P, q),
      t2("t2", P, q), t3("t3", P, q);
  copy_in(dx, disp_x);
  copy_in(dy, disp_y);
  copy_in(dz, disp_z);
  copy_in(sv, src_vor);
  copy_in(sd, src_div);
  copy_in(t1, out_1);
  copy_in(t2, out_2);
  copy_in(t3, out_3);
  swe_vel_interactions_2(c->rc, dx, dy, dz, t1, t2, t3, sv, sd, c->list, c->panels, c->interp);
  copy_out(t1, out_1);
  copy_out(t2, out_2);
  copy_out(t3, out_3);
}

// swe_tendency_computation_2 over every leaf panel (all A x q).
void ref_swe_tendency(void* h, const double* vel_x, const double* vel_y, const double* vel_z, const double* vors,
                      const double* divs, const double* height, const double* surface, double* vor_tend,
                      double* div_tend, double* h_tend) {
  RefCtx* c = static_cast<RefCtx*>(h);
  int A = c->rc.active_panel_count, q = c->q;
  V2 vx("vx", A, q), vy("vy", A, q), vz("vz", A, q), v("v", A, q), d("d", A, q), hh("h", A, q), s("s", A, q),
      vt("vt", A, q), dt("dt", A, q), ht("ht", A, q);
  copy_in(vx, vel_x);
  copy_in(vy, vel_y);
  copy_in(vz, vel_z);
  copy_in(v, vors);
  copy_in(d, divs);
  copy_in(hh, height);
  copy_in(s, surface);
  int offset = c->rc.panel_count - A;
  Kokkos::parallel_for(A, swe_tendency_computation_2(c->xcos, c->ycos, c->zcos, vx, vy, vz, v, vt, d, dt, hh, s, ht,
                                                     c->panels, c->rc.omega, c->rc.interp_degree, offset));
  copy_out(vt, vor_tend);
  copy_out(dt, div_tend);
  copy_out(ht, h_tend);
}

// The driver's set-up before the time loop (executables/swe_time_evo.cpp:352-410):
// velocity of the undisplaced vorticity and divergence, unified; base
// tendencies from it, unified.  vel_* receive the unified velocity (the
// driver zeroes them afterwards; the step does not read them).
void ref_swe_init(void* h, const double* vors, const double* divs, const double* height, double* vel_x,
                  double* vel_y, double* vel_z, double* base_vor, double* base_div, double* base_h,
                  const int* two_d_to_1d, const int* counts) {
  RefCtx* c = static_cast<RefCtx*>(h);
  const RunConfig& rc = c->rc;
  int A = rc.active_panel_count, P = rc.panel_count, q = c->q;
  Map m = make_map(c, two_d_to_1d, counts);
  V2 v("v", A, q), d("d", A, q), hh("h", A, q);
  copy_in(v, vors);
  copy_in(d, divs);
  copy_in(hh, height);
  V2 psv("psv", P, q), psd("psd", P, q), dx("dx", P, q), dy("dy", P, q), dz("dz", P, q), eff("eff", A, q);
  apply_topography(rc, c->xcos, c->ycos, c->zcos, dx, dy, dz, hh, eff);
  upward_pass(rc, c->interp, c->panels, c->area, v, psv);
  upward_pass(rc, c->interp, c->panels, c->area, d, psd);
  V2 t1("t1", P, q), t2("t2", P, q), t3("t3", P, q);
  swe_vel_interactions_2(rc, dx, dy, dz, t1, t2, t3, psv, psd, c->list, c->panels, c->interp);
  V2 vx("vx", A, q), vy("vy", A, q), vz("vz", A, q);
  downward_pass_3(rc, c->interp, c->panels, t1, t2, t3, vx, vy, vz);
  unify_boundary_vals(rc, m.counts, m.two_d, vx);
  unify_boundary_vals(rc, m.counts, m.two_d, vy);
  unify_boundary_vals(rc, m.counts, m.two_d, vz);
  V2 bv("bv", A, q), bd("bd", A, q), bh("bh", A, q);
  int offset = P - A;
  Kokkos::parallel_for(A, swe_tendency_computation_2(c->xcos, c->ycos, c->zcos, vx, vy, vz, v, bv, d, bd, eff, eff, bh,
                                                     c->panels, rc.omega, rc.interp_degree, offset));
  unify_boundary_vals(rc, m.counts, m.two_d, bv);
  unify_boundary_vals(rc, m.counts, m.two_d, bd);
  unify_boundary_vals(rc, m.counts, m.two_d, bh);
  copy_out(vx, vel_x);
  copy_out(vy, vel_y);
  copy_out(vz, vel_z);
  copy_out(bv, base_vor);
  copy_out(bd, base_div);
  copy_out(bh, base_h);
}

// nsteps calls of swe_back_rk4_step_2; vors / divs / height / vel / tracers
// are in-out (A x q [x T]).  With driver_unify, each step is followed by the
// driver's unify_boundary_vals of vors, divs and height
// (executables/swe_time_evo.cpp:416-418).
void ref_swe_step(void* h, double* vors, double* divs, double* height, double* vel_x, double* vel_y,
                  double* vel_z, double* tracers, const double* base_vor, const double* base_div,
                  const double* base_h, const int* two_d_to_1d, const int* counts, double time, int nsteps,
                  int driver_unify) {
  RefCtx* c = static_cast<RefCtx*>(h);
  int A = c->rc.active_panel_count, q = c->q, T = c->rc.tracer_count;
  Map m = make_map(c, two_d_to_1d, counts);
  V2 v("vors", A, q), d("divs", A, q), hh("height", A, q), vx("vel_x", A, q), vy("vel_y", A, q),
      vz("vel_z", A, q), bv("bv", A, q), bd("bd", A, q), bh("bh", A, q);
  V3 tr("tracers", A, q, T);
  copy_in(v, vors);
  copy_in(d, divs);
  copy_in(hh, height);
  copy_in(vx, vel_x);
  copy_in(vy, vel_y);
  copy_in(vz, vel_z);
  copy_in(bv, base_vor);
  copy_in(bd, base_div);
  copy_in(bh, base_h);
  if (T > 0) std::memcpy(tr.data(), tracers, sizeof(double) * A * q * T);
  for (int s = 0; s < nsteps; s++) {
    {
      Quiet quiet;
      swe_back_rk4_step_2(c->rc, c->xcos, c->ycos, c->zcos, c->area, v, d, hh, c->interp, c->panels, c->list, vx,
                          vy, vz, tr, bv, bd, bh, m.counts, m.two_d, time + s * c->rc.delta_t);
    }
    if (driver_unify) {
      unify_boundary_vals(c->rc, m.counts, m.two_d, v);
      unify_boundary_vals(c->rc, m.counts, m.two_d, d);
      unify_boundary_vals(c->rc, m.counts, m.two_d, hh);
    }
  }
  copy_out(v, vors);
  copy_out(d, divs);
  copy_out(hh, height);
  copy_out(vx, vel_x);
  copy_out(vy, vel_y);
  copy_out(vz, vel_z);
  if (T > 0) std::memcpy(tracers, tr.data(), sizeof(double) * A * q * T);
}

}  // extern "C"
