/* CPU restatement of the reference's BVE hot path (test infrastructure only).
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load
 * this library, and only as the checker or the timed CPU baseline; the product
 * library never calls it.  Function-by-function citations of the reference are
 * in bslpm_oracle.c.  The arithmetic and the accumulation order follow the
 * reference, so with one thread the results agree bit for bit with the
 * reference compiled by oracle/Makefile (checked by tests/test_oracle_golden.py).
 */
#ifndef SBSLPM_BSLPM_ORACLE_H
#define SBSLPM_BSLPM_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

/* Same fields as the reference's CubedSpherePanel
 * (src/initialize_cubed_sphere.hpp:8-29); bounds are in [-1, 1], times pi/4
 * on the sphere. */
typedef struct {
  int id, top, left, bot, right, face, level, parent;
  int child[4];
  int is_leaf;
  double min_xi, max_xi, min_eta, max_eta, radius, area;
} orc_panel;

int orc_panel_count(int levels);
int orc_leaf_count(int levels);
void orc_panels_init(int levels, orc_panel* panels);
/* interp: q x 4 = (xi node, eta node, BLI weight, CC weight).  exact_cc=0
 * reproduces the reference's weights; exact_cc=1 gives exact
 * Clenshaw-Curtis weights (the two agree only at the nodes' positions). */
void orc_interp_init(int degree, int exact_cc, double* interp);
void orc_spec_points(int levels, int degree, const orc_panel* panels, const double* interp, double* x,
                     double* y, double* z, double* area);
/* Returns the interaction count; writes at most cap triples. */
long orc_dual_tree_traversal(int levels, const orc_panel* panels, double theta, int* list, long cap);

void orc_interp_vals_bli(double* basis, double xi, double eta, double min_xi, double max_xi, double min_eta,
                         double max_eta, int degree);
int orc_point_locate_panel(const orc_panel* panels, double x, double y, double z);

void orc_upward_pass(int levels, int degree, const orc_panel* panels, const double* interp, const double* area,
                     const double* pots, double* proxy);
void orc_downward_pass_3(int levels, int degree, const orc_panel* panels, const double* interp, double* t1,
                         double* t2, double* t3, double* s1, double* s2, double* s3);
void orc_bve_vel_interactions(int levels, int degree, const orc_panel* panels, const double* interp, long n_list,
                              const int* list, const double* disp_x, const double* disp_y, const double* disp_z,
                              const double* source, double kernel_eps, double* t1, double* t2, double* t3);
/* Direct (all leaf x all leaf) velocity: the reference FMM in the theta -> 0
 * limit, where every interaction is leaf-leaf.  Targets are undisplaced leaf
 * proxies, sources are displaced leaf proxies. */
void orc_bve_direct_velocity(int levels, int degree, const orc_panel* panels, const double* interp,
                             const double* disp_x, const double* disp_y, const double* disp_z,
                             const double* source, double kernel_eps, double* t1, double* t2, double* t3);
void orc_bve_departure(int levels, int degree, const orc_panel* panels, const double* x, const double* y,
                       const double* z, const double* v0, const double* v1, const double* v2, const double* v3,
                       double dt, double* dep_x, double* dep_y, double* dep_z);
void orc_bve_remap(int levels, int degree, const orc_panel* panels, const double* z, const double* dep_x,
                   const double* dep_y, const double* dep_z, const double* vors, int tracer_count,
                   const double* tracers, double omega, double* new_vors, double* new_tracers);

/* One bve_back_rk4_step.  mode 0 = interaction list (FMM), 1 = direct,
 * 2 = treecode (orc_bltc_velocity with proxy_degree, leaf_size, theta, typed).
 * vors (A x q), vel_* (A x q, out = stage-0 velocity), tracers (A x q x T)
 * are in-out. */
typedef struct {
  int levels, degree, tracer_count, mode;
  double kernel_eps, omega, dt;
  const orc_panel* panels;
  const double* interp;
  const double *x, *y, *z, *area;
  long n_list;
  const int* list;
  int forcing;  /* 0 none, 1 ssw, 2 ssw2 (src/forcing_funcs.cpp:82-96) */
  double time;  /* the step's time (seconds), for the forcing */
  int proxy_degree, leaf_size, typed; /* mode 2 */
  double theta;                       /* mode 2: the treecode's MAC */
} orc_bve_problem;
void orc_bve_step(const orc_bve_problem* pb, double* vors, double* vel_x, double* vel_y, double* vel_z,
                  double* tracers);

/* Treecode with decoupled proxy degree: the reference's irregular-point FMM
 * (base_pots_ll, child_to_parent_ll, dual_tree_traversal_irreg,
 * swe_vel_panel_interaction_ll rotational part, parent_to_child_3_ll,
 * child_panel_interp_3_ll) on the particle grid of (levels, degree), its
 * quadtree truncated so that a leaf holds at most leaf_size particles, degree
 * n proxies.  Particle arrays are N = A x q in [leaf panel][q] order.
 * typed 1: the reference's pp / pc / cp / cc typing of well-separated pairs;
 * 0: every well-separated pair proxy x proxy.  Targets t (grid points),
 * sources s with strengths w; u (3 x N) is overwritten. */
void orc_bltc_shape(int levels, int degree, int leaf_size, int* tree_levels, int* npl);
long orc_bltc_list(int levels, int degree, int leaf_size, int n, double theta, int* list, long cap);
void orc_bltc_upward(int levels, int degree, int leaf_size, int n, const double* sx, const double* sy,
                     const double* sz, const double* w, double* proxy);
/* T (3 x Pf x qx) is interpolated down in place; u (3 x N) accumulated. */
void orc_bltc_downward(int levels, int degree, int leaf_size, int n, double* T, const double* tx, const double* ty,
                       const double* tz, double* u);
void orc_bltc_velocity(int levels, int degree, int leaf_size, int n, double theta, double eps, int typed,
                       const double* tx, const double* ty, const double* tz, const double* sx, const double* sy,
                       const double* sz, const double* w, double* u);
/* The shallow-water form: vorticity sources s (strengths w, rotational part)
 * and divergence sources d (strengths wd, divergent part of
 * swe_vel_panel_interaction_ll, src/fmm_interactions/swe_vel_impl.hpp:256-284). */
void orc_bltc_velocity_swe(int levels, int degree, int leaf_size, int n, double theta, double eps, int typed,
                           const double* tx, const double* ty, const double* tz, const double* sx, const double* sy,
                           const double* sz, const double* w, const double* dx, const double* dy, const double* dz,
                           const double* wd, double* u);

/* Shallow water v2.  swe_vel_interactions_2 (src/fmm_interactions/swe_vel.cpp:39-67,
 * accumulating into t1..t3), swe_tendency_computation_2
 * (src/swe_time_step_2_impl.hpp:41-127, outputs overwritten; the reference's
 * g/a is 9.81 / 6371000), unify_boundary_vals (src/initialize_cubed_sphere.cpp:364-370)
 * over n values with the [leaf][q] -> point map and the copies per point,
 * and one swe_back_rk4_step_2 (src/swe_time_step_2.cpp:785-1035, topography
 * none): vors, divs, height, tracers in-out, vel_* out (the first stage's
 * velocity). */
void orc_swe_vel_interactions(int levels, int degree, const orc_panel* p, const double* interp, long n_list,
                              const int* list, const double* disp_x, const double* disp_y, const double* disp_z,
                              const double* src_vor, const double* src_div, double eps, double* t1, double* t2,
                              double* t3);
void orc_swe_tendencies(int levels, int degree, const orc_panel* p, const double* x, const double* y,
                        const double* z, const double* vx, const double* vy, const double* vz, const double* vors,
                        const double* divs, const double* height, const double* surface, double omega,
                        double g_over_a, double* vor_t, double* div_t, double* h_t);
void orc_swe_unify(int n, const int* map, const int* counts, int points, double* vals);
typedef struct {
  int levels, degree, tracer_count;
  double kernel_eps, omega, dt, g_over_a;
  const orc_panel* panels;
  const double* interp;
  const double *x, *y, *z, *area;
  long n_list;
  const int* list;
  const int *map, *counts; /* the grid's point map (cubed_sphere_2d_to_1d) */
  int point_count;
  const double *base_div, *base_h; /* base tendencies (the vorticity's is not used by the reference) */
} orc_swe_problem;
void orc_swe_step(const orc_swe_problem* pb, double* vors, double* divs, double* height, double* vel_x,
                  double* vel_y, double* vel_z, double* tracers);

/* direct_sum_inv_lap (src/direct_sum_impl.hpp:20-27) over n points. */
void orc_direct_sum_inv_lap(int n, const double* x, const double* y, const double* z, const double* area,
                            const double* pots, double* soln);

/* Poisson FMM: poisson_fmm_interactions (src/fmm_interactions/inverse_poisson.cpp:9-34,
 * target += ...) and downward_pass (src/fmm_funcs.cpp:357-372). */
void orc_poisson_fmm_interactions(int levels, int degree, const orc_panel* p, const double* interp, long n_list,
                                  const int* list, const double* source, double* target);
void orc_downward_pass(int levels, int degree, const orc_panel* p, const double* interp, double* t, double* s);

/* Output path: interp_to_latlon_host (src/interp_funcs.hpp:22-77) of one
 * [leaf][q] field to an nlat x nlon grid in degrees, and xyz_vel_to_uv_vel
 * (src/general_utils_impl.hpp:195-229). */
void orc_interp_to_latlon(int levels, int degree, const orc_panel* p, const double* data, int nlat,
                          const double* lats, int nlon, const double* lons, double* out);
void orc_xyz_vel_to_uv_vel(long n, const double* x, const double* y, const double* z, const double* vx,
                           const double* vy, const double* vz, double* u, double* v);

#ifdef __cplusplus
}
#endif
#endif
