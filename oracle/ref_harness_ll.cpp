// Harness around the reference's own irregular-point FMM functions (the
// "_ll" variants; test infrastructure only), compiled with the reference's
// unmodified src/*.cpp against oracle/shim/ into oracle/_ref/libsbslpm_ref.so
// (recipe: oracle/Makefile).  It runs them on the BVE particle grid with the
// grid's quadtree truncated so that a leaf holds at most leaf_size particles
// (the particles of a tree leaf are those of its descendant grid panels), to
// pin the treecode restatement in oracle/bslpm_oracle.c:
//   dual_tree_traversal_irreg      (src/fmm_funcs.cpp:125-231)
//   upward_pass_ll                 (src/fmm_funcs.cpp:394-405; base_pots_ll,
//                                   child_to_parent_ll src/fmm_funcs_impl.hpp:190-268)
//   swe_vel_interactions_ll        (src/fmm_interactions/swe_vel.cpp:69-100,
//                                   swe_vel_panel_interaction_ll swe_vel_impl.hpp:149-288),
//                                  rotational and divergent parts
//   downward_pass_3_ll             (src/fmm_funcs.cpp:407-419; parent_to_child_3_ll,
//                                   child_panel_interp_3_ll src/fmm_funcs_impl.hpp:270-364)
// The tree table is built as initialize_cube_sphere_irreg_points builds its
// panels (src/initialize_cubed_sphere.cpp:446-592): bounds in radians halved
// from +-pi/4, radius = the largest great-circle distance from the centre to
// a corner, run_config.levels = the deepest level.
#include <Kokkos_Core.hpp>
#include <cmath>
#include <cstring>

#include "run_config.hpp"
#include "initialize_cubed_sphere.hpp"
#include "cubed_sphere_transforms_impl.hpp"
#include "fmm_funcs.hpp"
#include "fmm_interactions/swe_vel.hpp"
#include "ref_ctx.hpp"

using namespace refh;

extern "C" void* ref_create(int levels, int degree, double theta, double kernel_eps, double omega, int delta_t,
                            int tracer_count);
extern "C" void ref_destroy(void* h);

namespace {
struct LLCtx {
  RefCtx* grid;
  RunConfig rc;
  Kokkos::View<CubedSpherePanel*, Kokkos::HostSpace> tree_h;
  Kokkos::View<CubedSpherePanel*> tree;
  Kokkos::View<int**, Kokkos::LayoutRight> lpp;
  Kokkos::View<interact_pair*, Kokkos::HostSpace> list_h;
  Kokkos::View<interact_pair*> list;
  int Lf, npl, qx, Pf;
};
}  // namespace

extern "C" {

void* ref_ll_create(int levels, int degree, int leaf_size, int proxy_degree, double theta, double kernel_eps) {
  LLCtx* c = new LLCtx();
  c->grid = static_cast<RefCtx*>(ref_create(levels, degree, 0.7, kernel_eps, 1.0, 1, 0));
  int q = c->grid->q, m = 0;
  long npl = q;
  while (npl * 4 <= leaf_size && m < levels - 1) {  // split while a panel holds more than leaf_size
    npl *= 4;
    m++;
  }
  c->npl = (int)npl;
  c->Lf = levels - m;
  c->qx = (proxy_degree + 1) * (proxy_degree + 1);
  RunConfig rt;
  rt.levels = c->Lf;
  c->Pf = 2 * ((int)std::pow(4, c->Lf) - 1);
  c->tree_h = Kokkos::View<CubedSpherePanel*, Kokkos::HostSpace>("tree", c->Pf);
  cubed_sphere_panels_init(rt, c->tree_h);
  // radian bounds by halving, as the irregular tree's refinement computes them
  for (int i = 0; i < c->Pf; i++) {
    CubedSpherePanel& p = c->tree_h(i);
    if (p.level == 0) {
      p.min_xi = -M_PI / 4.0, p.max_xi = M_PI / 4.0, p.min_eta = -M_PI / 4.0, p.max_eta = M_PI / 4.0;
    }
    if (p.level < c->Lf - 1) {
      double mid_xi = 0.5 * (p.min_xi + p.max_xi), mid_eta = 0.5 * (p.min_eta + p.max_eta);
      CubedSpherePanel& c1 = c->tree_h(p.child1);
      CubedSpherePanel& c2 = c->tree_h(p.child2);
      CubedSpherePanel& c3 = c->tree_h(p.child3);
      CubedSpherePanel& c4 = c->tree_h(p.child4);
      c1.min_xi = mid_xi, c1.max_xi = p.max_xi, c1.min_eta = mid_eta, c1.max_eta = p.max_eta;
      c2.min_xi = p.min_xi, c2.max_xi = mid_xi, c2.min_eta = mid_eta, c2.max_eta = p.max_eta;
      c3.min_xi = p.min_xi, c3.max_xi = mid_xi, c3.min_eta = p.min_eta, c3.max_eta = mid_eta;
      c4.min_xi = mid_xi, c4.max_xi = p.max_xi, c4.min_eta = p.min_eta, c4.max_eta = mid_eta;
    }
    double pc[3], p1[3], p2[3], p3[3], p4[3];
    double mid_xi = (p.min_xi + p.max_xi) * 0.5, mid_eta = (p.min_eta + p.max_eta) * 0.5;
    xyz_from_xieta(mid_xi, mid_eta, p.face, pc);
    xyz_from_xieta(p.max_xi, p.min_eta, p.face, p1);
    xyz_from_xieta(p.max_xi, p.max_eta, p.face, p2);
    xyz_from_xieta(p.min_xi, p.max_eta, p.face, p3);
    xyz_from_xieta(p.min_xi, p.min_eta, p.face, p4);
    double d1 = std::acos(pc[0] * p1[0] + pc[1] * p1[1] + pc[2] * p1[2]);
    double d2 = std::acos(pc[0] * p2[0] + pc[1] * p2[1] + pc[2] * p2[2]);
    double d3 = std::acos(pc[0] * p3[0] + pc[1] * p3[1] + pc[2] * p3[2]);
    double d4 = std::acos(pc[0] * p4[0] + pc[1] * p4[1] + pc[2] * p4[2]);
    p.radius = std::max(std::max(std::max(d1, d2), d3), d4);
    p.point_count = p.is_leaf ? c->npl : 0;
  }
  const int offf = c->Pf - 6 * (int)std::pow(4, c->Lf - 1);
  c->lpp = Kokkos::View<int**, Kokkos::LayoutRight>("leaf_panel_points", c->Pf, c->npl);
  for (int i = 0; i < c->Pf; i++)
    for (int j = 0; j < c->npl; j++) c->lpp(i, j) = i >= offf ? (i - offf) * c->npl + j : -1;
  RunConfig& rc = c->rc;
  rc.levels = c->Lf - 1;  // the deepest level, as initialize_cube_sphere_irreg_points sets it
  rc.panel_count = c->Pf;
  rc.cubed_sphere_level_start = rt.cubed_sphere_level_start;
  rc.interp_degree = proxy_degree;
  rc.fmm_theta = theta;
  rc.kernel_eps = kernel_eps;
  rc.mpi_p = 1;
  rc.mpi_id = 0;
  c->list_h = Kokkos::View<interact_pair*, Kokkos::HostSpace>("list", 1);
  dual_tree_traversal_irreg(rc, c->tree_h, c->list_h);
  c->tree = c->tree_h;
  c->list = c->list_h;
  return c;
}

void ref_ll_destroy(void* h) {
  LLCtx* c = static_cast<LLCtx*>(h);
  free(c->rc.cubed_sphere_level_start);
  ref_destroy(c->grid);
  delete c;
}

// out[0..4] = tree panels, tree levels, particles per leaf, proxies per panel, list length
void ref_ll_sizes(void* h, int* out) {
  LLCtx* c = static_cast<LLCtx*>(h);
  out[0] = c->Pf;
  out[1] = c->Lf;
  out[2] = c->npl;
  out[3] = c->qx;
  out[4] = c->rc.fmm_interaction_count;
}

// I x 3 = target_panel, source_panel, interact_type
void ref_ll_list(void* h, int* out) {
  LLCtx* c = static_cast<LLCtx*>(h);
  for (int i = 0; i < c->rc.fmm_interaction_count; i++) {
    out[3 * i] = c->list_h(i).target_panel;
    out[3 * i + 1] = c->list_h(i).source_panel;
    out[3 * i + 2] = c->list_h(i).interact_type;
  }
}

// upward_pass_ll of pots (A x q, times the grid's quadrature weights) into proxy (Pf x qx)
void ref_ll_upward(void* h, const double* pots, double* proxy) {
  LLCtx* c = static_cast<LLCtx*>(h);
  RefCtx* g = c->grid;
  V2 p("pots", g->rc.active_panel_count, g->q), s("proxy", c->Pf, c->qx);
  copy_in(p, pots);
  upward_pass_ll(c->rc, g->xcos, g->ycos, g->zcos, c->tree, g->area, p, s, c->lpp);
  copy_out(s, proxy);
}

// downward_pass_3_ll: proxy targets t1..t3 (Pf x qx) down to the particles, added into s1..s3 (A x q)
void ref_ll_downward(void* h, const double* t1, const double* t2, const double* t3, double* s1, double* s2,
                     double* s3) {
  LLCtx* c = static_cast<LLCtx*>(h);
  RefCtx* g = c->grid;
  int A = g->rc.active_panel_count;
  V2 a("t1", c->Pf, c->qx), b("t2", c->Pf, c->qx), d("t3", c->Pf, c->qx), u("s1", A, g->q), v("s2", A, g->q),
      w("s3", A, g->q);
  copy_in(a, t1);
  copy_in(b, t2);
  copy_in(d, t3);
  copy_in(u, s1);
  copy_in(v, s2);
  copy_in(w, s3);
  downward_pass_3_ll(c->rc, g->xcos, g->ycos, g->zcos, c->tree, a, b, d, u, v, w, c->lpp);
  copy_out(u, s1);
  copy_out(v, s2);
  copy_out(w, s3);
}

// The irregular-point FMM velocity of vorticity vors and divergence divs
// (A x q; divs may be NULL: zero divergence): upward_pass_ll of both fields,
// swe_vel_interactions_ll, downward_pass_3_ll.
void ref_ll_velocity(void* h, const double* vors, const double* divs, double* vel_x, double* vel_y, double* vel_z) {
  LLCtx* c = static_cast<LLCtx*>(h);
  RefCtx* g = c->grid;
  int A = g->rc.active_panel_count, q = g->q;
  V2 v("vors", A, q), d("divs", A, q), psv("psv", c->Pf, c->qx), psd("psd", c->Pf, c->qx), t1("t1", c->Pf, c->qx),
      t2("t2", c->Pf, c->qx), t3("t3", c->Pf, c->qx), vx("vx", A, q), vy("vy", A, q), vz("vz", A, q);
  copy_in(v, vors);
  upward_pass_ll(c->rc, g->xcos, g->ycos, g->zcos, c->tree, g->area, v, psv, c->lpp);
  if (divs) {
    copy_in(d, divs);
    upward_pass_ll(c->rc, g->xcos, g->ycos, g->zcos, c->tree, g->area, d, psd, c->lpp);
  }
  swe_vel_interactions_ll(c->rc, g->xcos, g->ycos, g->zcos, t1, t2, t3, vx, vy, vz, psv, psd, v, d, g->area, c->list,
                          c->tree, c->lpp);
  downward_pass_3_ll(c->rc, g->xcos, g->ycos, g->zcos, c->tree, t1, t2, t3, vx, vy, vz, c->lpp);
  copy_out(vx, vel_x);
  copy_out(vy, vel_y);
  copy_out(vz, vel_z);
}

}  // extern "C"
