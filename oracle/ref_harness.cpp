// Harness around the reference's own BVE hot-path code (test infrastructure only).
//
// This translation unit is compiled together with the reference's unmodified
// src/*.cpp against the project-written shim headers in oracle/shim/, into
// oracle/_ref/libsbslpm_ref.so (recipe: oracle/Makefile).  It exposes plain C
// entry points so that the golden-vector script and the CPU-baseline leg of the
// benchmark can drive the reference's functions:
//   cubed_sphere_panels_init / interp_init / cube_sphere_spec_points
//       (src/initialize_cubed_sphere.cpp:185-234, 280-288; src/interp_funcs.cpp:24-73)
//   dual_tree_traversal            (src/fmm_funcs.cpp:17-123)
//   upward_pass / downward_pass_3  (src/fmm_funcs.cpp:341-355, 374-392)
//   bve_vel_interactions           (src/fmm_interactions/bve_vel.cpp:9-37)
//   bve_back_rk4_step              (src/bve_time_step.cpp:311-419)
//   bve_find_departure_points, bve_departure_to_target
//                                  (src/bve_time_step.cpp:172-309, 15-67)
//   interp_vals_bli / point_locate_panel (src/interp_funcs_impl.hpp:11-142)
//   bve_initialize                 (src/initial_conditions.cpp:358-385)
//   direct_sum_inv_lap             (src/direct_sum.cpp:8-15)
//   poisson_fmm_interactions, downward_pass
//                                  (src/fmm_interactions/inverse_poisson.cpp:9-34, src/fmm_funcs.cpp:357-372)
//   interp_to_latlon_host          (src/interp_funcs.hpp:22-77)
//   xyz_vel_to_uv_vel              (src/general_utils_impl.hpp:195-229)
// The reference's bve_time_step.cpp is included textually (unmodified) so that
// its file-local departure / remap functors can be called one at a time.
#include <Kokkos_Core.hpp>
#include <cstring>
#include <string>

#include "run_config.hpp"
#include "initialize_cubed_sphere.hpp"
#include "interp_funcs.hpp"
#include "fmm_funcs.hpp"
#include "fmm_interactions/bve_vel.hpp"
#include "initial_conditions.hpp"
#include "direct_sum.hpp"
#include "fmm_interactions/inverse_poisson.hpp"
#include "bve_time_step.cpp"
#include "ref_ctx.hpp"

using namespace refh;

extern "C" {

// Builds the grid, tree and interaction list exactly as the reference driver
// does (executables/bve_time_evo.cpp:48-76, 255-257).  delta_t is an integer
// number of seconds as in the reference's RunConfig (src/run_config.hpp:20-21).
void* ref_create(int levels, int degree, double theta, double kernel_eps, double omega, int delta_t,
                 int tracer_count) {
  RefCtx* c = new RefCtx();
  RunConfig& rc = c->rc;
  rc.levels = levels;
  rc.interp_degree = degree > 10 ? 10 : degree;
  rc.fmm_theta = theta;
  rc.kernel_eps = kernel_eps;
  rc.omega = omega;
  rc.delta_t = delta_t;
  rc.end_time = delta_t;
  rc.time_steps = 1;
  rc.tracer_count = tracer_count;
  rc.forcing = false;
  rc.mpi_p = 1;
  rc.mpi_id = 0;
  // derived sizes, as read_run_config computes them (src/io_utils.cpp:83-90)
  rc.fmm_cluster_thresh = 4 * (rc.interp_degree + 1) * (rc.interp_degree + 1);
  rc.point_count = 6 * (int)std::pow(4, rc.levels);
  rc.panel_count = 2 * ((int)std::pow(4, rc.levels) - 1);
  rc.active_panel_count = 6 * (int)std::pow(4, rc.levels - 1);
  c->q = (rc.interp_degree + 1) * (rc.interp_degree + 1);
  int q = c->q, A = rc.active_panel_count;

  c->panels_h = Kokkos::View<CubedSpherePanel*, Kokkos::HostSpace>("panels", rc.panel_count);
  cubed_sphere_panels_init(rc, c->panels_h);
  rc.point_count = rc.active_panel_count * rc.interp_degree * rc.interp_degree + 2;
  c->interp_h = V2H("interp vals", q, 4);
  interp_init(rc, c->interp_h);
  c->xcos_h = V2H("xcos", A, q);
  c->ycos_h = V2H("ycos", A, q);
  c->zcos_h = V2H("zcos", A, q);
  c->area_h = V2H("area", A, q);
  cube_sphere_spec_points(rc, c->panels_h, c->interp_h, c->xcos_h, c->ycos_h, c->zcos_h, c->area_h);
  c->list_h = Kokkos::View<interact_pair*, Kokkos::HostSpace>("interaction list", 1);
  dual_tree_traversal(rc, c->panels_h, c->list_h);
  // one memory space in this build: device views alias the host views
  c->panels = c->panels_h;
  c->interp = c->interp_h;
  c->xcos = c->xcos_h;
  c->ycos = c->ycos_h;
  c->zcos = c->zcos_h;
  c->area = c->area_h;
  c->list = c->list_h;
  c->proxy_source = V2("proxy source", rc.panel_count, q);
  return c;
}

void ref_destroy(void* h) { delete static_cast<RefCtx*>(h); }

// sizes[0..4] = panel_count, active_panel_count, q, interaction_count, level_count
void ref_sizes(void* h, int* sizes) {
  RefCtx* c = static_cast<RefCtx*>(h);
  sizes[0] = c->rc.panel_count;
  sizes[1] = c->rc.active_panel_count;
  sizes[2] = c->q;
  sizes[3] = c->rc.fmm_interaction_count;
  sizes[4] = c->rc.levels;
}

// ints: P x 13 = id, top, left, bot, right, face, level, parent, child1..4, is_leaf
// dbls: P x 6  = min_xi, max_xi, min_eta, max_eta, radius, area
void ref_get_panels(void* h, int* ints, double* dbls) {
  RefCtx* c = static_cast<RefCtx*>(h);
  for (int i = 0; i < c->rc.panel_count; i++) {
    const CubedSpherePanel& p = c->panels_h(i);
    int* o = ints + 13 * i;
    o[0] = p.id; o[1] = p.id_top_edge; o[2] = p.id_left_edge; o[3] = p.id_bot_edge;
    o[4] = p.id_right_edge; o[5] = p.face; o[6] = p.level; o[7] = p.parent_id;
    o[8] = p.child1; o[9] = p.child2; o[10] = p.child3; o[11] = p.child4; o[12] = p.is_leaf ? 1 : 0;
    double* d = dbls + 6 * i;
    d[0] = p.min_xi; d[1] = p.max_xi; d[2] = p.min_eta; d[3] = p.max_eta; d[4] = p.radius; d[5] = p.area;
  }
}

// I x 3 = target_panel, source_panel, interact_type
void ref_get_interactions(void* h, int* out) {
  RefCtx* c = static_cast<RefCtx*>(h);
  for (int i = 0; i < c->rc.fmm_interaction_count; i++) {
    out[3 * i] = c->list_h(i).target_panel;
    out[3 * i + 1] = c->list_h(i).source_panel;
    out[3 * i + 2] = c->list_h(i).interact_type;
  }
}

// xcos/ycos/zcos/area: A x q; interp: q x 4
void ref_get_points(void* h, double* x, double* y, double* z, double* area, double* interp) {
  RefCtx* c = static_cast<RefCtx*>(h);
  copy_out(c->xcos, x);
  copy_out(c->ycos, y);
  copy_out(c->zcos, z);
  copy_out(c->area, area);
  copy_out(c->interp, interp);
}

// Replaces the quadrature weights (A x q) every later call reads, e.g. with
// the exact Clenshaw-Curtis weights of a run that uses them; the reference's
// own weights come from cube_sphere_spec_points (src/initialize_cubed_sphere.cpp:280-288).
void ref_set_area(void* h, const double* area) {
  RefCtx* c = static_cast<RefCtx*>(h);
  copy_in(c->area, area);
}

// The reference's own initial conditions (rh4 / gv / pv / rot), with balance_ic.
void ref_bve_initialize(void* h, const char* ic, int balance, double* vors_out) {
  RefCtx* c = static_cast<RefCtx*>(h);
  RunConfig rc = c->rc;
  rc.initial_condition = ic;
  rc.balance_ic = balance != 0;
  V2H v("vors", rc.active_panel_count, c->q);
  bve_initialize(rc, c->xcos_h, c->ycos_h, c->zcos_h, v, c->area_h);
  copy_out(v, vors_out);
}

// RunConfig::forcing / forcing_type (src/run_config.hpp:35-36): 0 none, 1 "ssw", 2 "ssw2".
void ref_set_forcing(void* h, int forcing) {
  RefCtx* c = static_cast<RefCtx*>(h);
  c->rc.forcing = forcing != 0;
  c->rc.forcing_type = forcing == 2 ? "ssw2" : "ssw";
}

// nsteps calls of bve_back_rk4_step; vors / vel / tracers are in-out (A x q [x T]).
void ref_bve_step(void* h, double* vors, double* vel_x, double* vel_y, double* vel_z, double* tracers,
                  double time, int nsteps) {
  RefCtx* c = static_cast<RefCtx*>(h);
  int A = c->rc.active_panel_count, q = c->q, T = c->rc.tracer_count;
  V2 v("vors", A, q), vx("vel_x", A, q), vy("vel_y", A, q), vz("vel_z", A, q);
  V3 tr("tracers", A, q, T);
  copy_in(v, vors);
  if (T > 0) std::memcpy(tr.data(), tracers, sizeof(double) * A * q * T);
  for (int s = 0; s < nsteps; s++) {
    bve_back_rk4_step(c->rc, c->xcos, c->ycos, c->zcos, c->area, v, c->proxy_source, c->interp, c->panels,
                      c->list, vx, vy, vz, tr, time + s * c->rc.delta_t);
  }
  copy_out(v, vors);
  copy_out(vx, vel_x);
  copy_out(vy, vel_y);
  copy_out(vz, vel_z);
  if (T > 0) std::memcpy(tracers, tr.data(), sizeof(double) * A * q * T);
}

// One pass of bve_vel_interactions over the whole list.  disp_* and source: P x q.
// out_1..3 (P x q) are accumulated into, as the reference does.
void ref_bve_vel_interactions(void* h, const double* disp_x, const double* disp_y, const double* disp_z,
                              const double* source, double* out_1, double* out_2, double* out_3) {
  RefCtx* c = static_cast<RefCtx*>(h);
  int P = c->rc.panel_count, q = c->q;
  V2 dx("dx", P, q), dy("dy", P, q), dz("dz", P, q), s("s", P, q), t1("t1", P, q), t2("t2", P, q),
      t3("t3", P, q);
  copy_in(dx, disp_x);
  copy_in(dy, disp_y);
  copy_in(dz, disp_z);
  copy_in(s, source);
  copy_in(t1, out_1);
  copy_in(t2, out_2);
  copy_in(t3, out_3);
  bve_vel_interactions(c->rc, dx, dy, dz, t1, t2, t3, s, c->list, c->panels, c->interp);
  copy_out(t1, out_1);
  copy_out(t2, out_2);
  copy_out(t3, out_3);
}

// upward_pass with leaf strengths area * pots (A x q); proxy_out: P x q.
void ref_upward_pass(void* h, const double* pots, double* proxy_out) {
  RefCtx* c = static_cast<RefCtx*>(h);
  int A = c->rc.active_panel_count, P = c->rc.panel_count, q = c->q;
  V2 p("pots", A, q), out("proxy", P, q);
  copy_in(p, pots);
  upward_pass(c->rc, c->interp, c->panels, c->area, p, out);
  copy_out(out, proxy_out);
}

// downward_pass_3: targets (P x q, modified in place as in the reference),
// sols (A x q) written.
void ref_downward_pass_3(void* h, double* t1, double* t2, double* t3, double* s1, double* s2, double* s3) {
  RefCtx* c = static_cast<RefCtx*>(h);
  int A = c->rc.active_panel_count, P = c->rc.panel_count, q = c->q;
  V2 a("t1", P, q), b("t2", P, q), d("t3", P, q), x("s1", A, q), y("s2", A, q), z("s3", A, q);
  copy_in(a, t1);
  copy_in(b, t2);
  copy_in(d, t3);
  downward_pass_3(c->rc, c->interp, c->panels, a, b, d, x, y, z);
  copy_out(a, t1);
  copy_out(b, t2);
  copy_out(d, t3);
  copy_out(x, s1);
  copy_out(y, s2);
  copy_out(z, s3);
}

// bve_find_departure_points: vel_k (A x q x 3 each as separate x/y/z arrays), dep out.
void ref_bve_departure(void* h, const double* v0, const double* v1, const double* v2, const double* v3,
                       double dt, double* dep_x, double* dep_y, double* dep_z) {
  // v_k layout: 3 consecutive A x q blocks (x, y, z)
  RefCtx* c = static_cast<RefCtx*>(h);
  int A = c->rc.active_panel_count, q = c->q;
  std::size_t n = (std::size_t)A * q;
  V2 vv[4][3];
  const double* src[4] = {v0, v1, v2, v3};
  for (int k = 0; k < 4; k++)
    for (int d = 0; d < 3; d++) {
      vv[k][d] = V2("v", A, q);
      std::memcpy(vv[k][d].data(), src[k] + d * n, sizeof(double) * n);
    }
  V2 dx("dep x", A, q), dy("dep y", A, q), dz("dep z", A, q);
  int offset = c->rc.panel_count - A;
  // the stepper passes the integer RunConfig::delta_t; the functor takes a double
  Kokkos::parallel_for(A, bve_find_departure_points(c->xcos, c->ycos, c->zcos, vv[0][0], vv[0][1], vv[0][2],
                                                    vv[1][0], vv[1][1], vv[1][2], vv[2][0], vv[2][1], vv[2][2],
                                                    vv[3][0], vv[3][1], vv[3][2], dx, dy, dz, c->panels, dt,
                                                    offset, c->rc.interp_degree));
  copy_out(dx, dep_x);
  copy_out(dy, dep_y);
  copy_out(dz, dep_z);
}

// bve_departure_to_target: remap of vors (and tracers) to departure points.
void ref_bve_remap(void* h, const double* dep_x, const double* dep_y, const double* dep_z, const double* vors,
                   const double* tracers, double* new_vors, double* new_tracers) {
  RefCtx* c = static_cast<RefCtx*>(h);
  int A = c->rc.active_panel_count, q = c->q, T = c->rc.tracer_count;
  V2 dx("dx", A, q), dy("dy", A, q), dz("dz", A, q), v("v", A, q), nv("nv", A, q);
  V3 tr("tr", A, q, T), ntr("ntr", A, q, T);
  copy_in(dx, dep_x);
  copy_in(dy, dep_y);
  copy_in(dz, dep_z);
  copy_in(v, vors);
  if (T > 0) std::memcpy(tr.data(), tracers, sizeof(double) * A * q * T);
  int offset = c->rc.panel_count - A;
  Kokkos::parallel_for(A, bve_departure_to_target(c->zcos, dx, dy, dz, v, nv, tr, ntr, c->panels,
                                                  c->rc.interp_degree, offset, c->rc.omega));
  copy_out(nv, new_vors);
  if (T > 0) std::memcpy(new_tracers, ntr.data(), sizeof(double) * A * q * T);
}

void ref_interp_vals_bli(double* basis, double xi, double eta, double min_xi, double max_xi, double min_eta,
                         double max_eta, int degree) {
  interp_vals_bli(basis, xi, eta, min_xi, max_xi, min_eta, max_eta, degree);
}

int ref_point_locate_panel(void* h, double x, double y, double z) {
  RefCtx* c = static_cast<RefCtx*>(h);
  return point_locate_panel(c->panels, x, y, z);
}

// direct_sum_inv_lap over n points (1-D arrays), one rank.
void ref_direct_sum_inv_lap(int n, const double* x, const double* y, const double* z, const double* area,
                            const double* pots, double* soln) {
  RunConfig rc;
  rc.point_count = n;
  rc.oned_lb = 0;
  rc.oned_ub = n;
  Kokkos::View<double*> vx("x", n), vy("y", n), vz("z", n), va("a", n), vp("p", n), vs("s", n);
  std::memcpy(vx.data(), x, sizeof(double) * n);
  std::memcpy(vy.data(), y, sizeof(double) * n);
  std::memcpy(vz.data(), z, sizeof(double) * n);
  std::memcpy(va.data(), area, sizeof(double) * n);
  std::memcpy(vp.data(), pots, sizeof(double) * n);
  direct_sum_inv_lap(rc, vx, vy, vz, va, vp, vs);
  std::memcpy(soln, vs.data(), sizeof(double) * n);
}

// interp_to_latlon_host (src/interp_funcs.hpp:22-77) of one [leaf][q] field.
void ref_interp_to_latlon(void* h, const double* data, int nlat, const double* lats, int nlon, const double* lons,
                          double* out) {
  RefCtx* c = static_cast<RefCtx*>(h);
  const int A = c->rc.active_panel_count;
  V2H d("data", A, c->q), o("out", nlat, nlon);
  Kokkos::View<double*, Kokkos::HostSpace> la("lats", nlat), lo("lons", nlon);
  std::memcpy(d.data(), data, sizeof(double) * A * c->q);
  std::memcpy(la.data(), lats, sizeof(double) * nlat);
  std::memcpy(lo.data(), lons, sizeof(double) * nlon);
  interp_to_latlon_host(c->rc, d, c->panels_h, o, la, lo);
  std::memcpy(out, o.data(), sizeof(double) * nlat * nlon);
}

// xyz_vel_to_uv_vel (src/general_utils_impl.hpp:195-229) over the grid points.
void ref_xyz_vel_to_uv_vel(void* h, const double* vx, const double* vy, const double* vz, double* u, double* v) {
  RefCtx* c = static_cast<RefCtx*>(h);
  const int A = c->rc.active_panel_count;
  V2 X("vx", A, c->q), Y("vy", A, c->q), Z("vz", A, c->q), U("u", A, c->q), W("v", A, c->q);
  copy_in(X, vx);
  copy_in(Y, vy);
  copy_in(Z, vz);
  Kokkos::parallel_for(A, xyz_vel_to_uv_vel(c->xcos, c->ycos, c->zcos, X, Y, Z, U, W));
  copy_out(U, u);
  copy_out(W, v);
}

// The Poisson FMM driver's solve (executables/poisson_eq_fmm.cpp:128-160):
// upward_pass, poisson_fmm_interactions, downward_pass on the context's list.
void ref_poisson_fmm(void* h, const double* pots, double* proxy_source, double* proxy_target, double* soln) {
  RefCtx* c = static_cast<RefCtx*>(h);
  const int A = c->rc.active_panel_count, P = c->rc.panel_count;
  V2 p("pots", A, c->q), s("soln", A, c->q), src("proxy source", P, c->q), tgt("proxy target", P, c->q);
  copy_in(p, pots);
  upward_pass(c->rc, c->interp, c->panels, c->area, p, src);
  copy_out(src, proxy_source);
  poisson_fmm_interactions(c->rc, tgt, src, c->list, c->panels, c->interp);
  downward_pass(c->rc, c->interp, c->panels, tgt, s);
  copy_out(tgt, proxy_target);
  copy_out(s, soln);
}

// poisson_fmm_interactions alone (target += ...).
void ref_poisson_fmm_interactions(void* h, const double* source, double* target) {
  RefCtx* c = static_cast<RefCtx*>(h);
  const int P = c->rc.panel_count;
  V2 src("proxy source", P, c->q), tgt("proxy target", P, c->q);
  copy_in(src, source);
  copy_in(tgt, target);
  poisson_fmm_interactions(c->rc, tgt, src, c->list, c->panels, c->interp);
  copy_out(tgt, target);
}

int ref_num_threads(void) { return Kokkos::num_threads(); }

}  // extern "C"
