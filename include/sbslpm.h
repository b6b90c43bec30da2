/*
 * sbslpm.h -- C ABI of the B200-native backward semi-Lagrangian (BSL) hot path
 * of spectral-BSLPM: the barotropic vorticity equation (BVE) RK4 step on the
 * cubed sphere, its Biot-Savart velocity (barycentric-Lagrange treecode/FMM or
 * direct sum), the FMM passes, and the departure-point Lagrange remap.
 *
 * Plain pointers and sizes only.  Unless stated otherwise, field pointers are
 * DEVICE pointers (cudaMalloc'd or torch CUDA tensors) in the reference's
 * layout: row-major [panel][q] float64, q = (interp_degree+1)^2, point index
 * i*(degree+1)+j with i the xi node and j the eta node
 * (reference: src/interp_funcs.cpp:64-72).  Leaf-only fields are
 * [leaf_count][q]; proxy fields over the whole tree are [panel_count][q].
 *
 * Every entry point returns an sbslpm_status.  Device code never traps: a
 * point outside its panel (where the reference calls Kokkos::abort,
 * src/interp_funcs_impl.hpp:22-33) or a non-finite input sets a device error
 * word that the host turns into a status after the call.
 *
 * Threading: one host thread per context; calls on one context are ordered
 * on the context's CUDA stream and are not re-entrant.  Separate contexts are
 * independent.
 */
#ifndef SBSLPM_H
#define SBSLPM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  SBSLPM_OK = 0,
  SBSLPM_ERR_CONFIG = 1,       /* invalid configuration / namelist */
  SBSLPM_ERR_CUDA = 2,         /* CUDA runtime error (message: sbslpm_last_error) */
  SBSLPM_ERR_OUT_OF_PANEL = 3, /* BLI point outside its panel (reference aborts) */
  SBSLPM_ERR_NONFINITE = 4,    /* NaN/Inf met in a location step */
  SBSLPM_ERR_ARG = 5,          /* bad argument (null pointer, size) */
  SBSLPM_ERR_NO_DEVICE = 6,    /* no CUDA device / library built without it */
  SBSLPM_ERR_TIMEOUT = 7       /* a bounded device-side wait ran out (the kernel returned) */
} sbslpm_status;

/* Velocity evaluation used by the step. */
enum { SBSLPM_VEL_FMM = 0, SBSLPM_VEL_DIRECT = 1 };
/* Arithmetic of the pair kernels.  FP64: everything in float64.  MIXED: the
 * pair kernels evaluate in float32 on panel-relative coordinates and
 * accumulate per source panel in float32, then in float64; positions,
 * projections, BLI weights, the RK4 update and the remap stay float64. */
enum { SBSLPM_FP64 = 0, SBSLPM_MIXED = 1 };

/* Mirrors the hot-path fields of the reference's RunConfig
 * (src/run_config.hpp:6-44).  dt is a double (the reference's delta_t is an
 * int number of seconds). */
typedef struct {
  int levels;        /* RunConfig::levels: tree depth; leaves at level levels-1 */
  int interp_degree; /* RunConfig::interp_degree, 0..10 */
  double fmm_theta;  /* RunConfig::fmm_theta, MAC parameter */
  double kernel_eps; /* RunConfig::kernel_eps */
  double omega;      /* RunConfig::omega, rotation rate */
  double dt;         /* time step (RunConfig::delta_t as a double) */
  int tracer_count;  /* RunConfig::tracer_count */
  int velocity;      /* SBSLPM_VEL_FMM | SBSLPM_VEL_DIRECT */
  int precision;     /* SBSLPM_FP64 | SBSLPM_MIXED */
  int exact_cc;      /* setup helpers: 1 = exact Clenshaw-Curtis weights */
  /* 0: the reference's spectral FMM, whose proxies are the panels' own
   * interp_degree points (src/fmm_interactions/bve_vel_impl.hpp).  n > 0: a
   * treecode with degree-n Chebyshev proxies (fixed, (n+1)^2 per panel) on the
   * tree truncated so that a leaf holds at most leaf_size particles: near
   * leaf pairs are summed particle by particle, every well-separated pair
   * proxy by proxy (the typed-interaction design of the reference's
   * irregular-point tree, src/fmm_interactions/swe_vel_impl.hpp:149-288). */
  int proxy_degree;
  int leaf_size; /* RunConfig::leaf_size: particles per treecode leaf (proxy_degree > 0) */
  /* Shallow water: the factor of the height Laplacian in the divergence
   * tendency, g/a.  The reference hard-codes 9.81/6371000.0 (Earth, height in
   * units of the radius; src/swe_time_step_2_impl.hpp:103); 1 on the unit
   * sphere with the height field holding g*h. */
  double g_over_a;
  /* BVE forcing (src/forcing_funcs.cpp:82-96; namelist keys forcing=1 and
   * forcing_type): SBSLPM_FORCING_NONE, _SSW (bve_ssw_forcing, wavenumber 1)
   * or _SSW2 (bve_ssw_forcing_2, wavenumber 2) added to the vorticity that
   * sets the source strengths of every velocity evaluation, at the step's
   * time (seconds; the ramps are in days). */
  int forcing;
} sbslpm_config;

enum { SBSLPM_FORCING_NONE = 0, SBSLPM_FORCING_SSW = 1, SBSLPM_FORCING_SSW2 = 2 };

/* Same fields and order as the reference's CubedSpherePanel
 * (src/initialize_cubed_sphere.hpp:8-29); is_leaf is an int here. */
typedef struct {
  int id, id_top_edge, id_left_edge, id_bot_edge, id_right_edge, face, level, parent_id;
  int child1, child2, child3, child4;
  int is_leaf;
  double min_xi, max_xi, min_eta, max_eta, radius, area;
  int point_count;
} sbslpm_panel;

/* The reference's interact_pair (src/fmm_funcs.hpp:10-14). */
typedef struct {
  int target_panel, source_panel, interact_type; /* 0 pp, 1 pc, 2 cp, 3 cc */
} sbslpm_interact_pair;

typedef struct sbslpm_ctx sbslpm_ctx;

/* ---------------- configuration ---------------- */

/* Defaults of the reference's RunConfig / namelist.txt (theta 0.7,
 * kernel_eps 1e-4, Earth omega) with FMM velocity and float64. */
sbslpm_status sbslpm_config_default(sbslpm_config* cfg);
/* Replaces read_run_config (src/io_utils.cpp:11-92): key=value lines read
 * until an unknown key.  Extra keys of this library: dt (double), velocity
 * (fmm|direct), precision (fp64|mixed), exact_cc (0|1). */
sbslpm_status sbslpm_read_run_config(const char* path, sbslpm_config* cfg);
const char* sbslpm_status_string(sbslpm_status s);
/* Last error message of the calling thread (CUDA errors, config errors). */
const char* sbslpm_last_error(void);

/* ---------------- host-side setup (host pointers) ---------------- */

int sbslpm_panel_count(int levels); /* 2(4^levels - 1) */
int sbslpm_leaf_count(int levels);  /* 6 * 4^(levels-1) */
/* Replaces cubed_sphere_panels_init (src/initialize_cubed_sphere.cpp:185-234). */
sbslpm_status sbslpm_cubed_sphere_panels_init(int levels, sbslpm_panel* panels);
/* Replaces interp_init (src/interp_funcs.cpp:24-73); interp is q x 4. */
sbslpm_status sbslpm_interp_init(int degree, int exact_cc, double* interp);
/* Replaces cube_sphere_spec_points (src/initialize_cubed_sphere.cpp:280-288). */
sbslpm_status sbslpm_cube_sphere_spec_points(int levels, int degree, const sbslpm_panel* panels,
                                             const double* interp, double* xcos, double* ycos, double* zcos,
                                             double* area);
/* Replaces dual_tree_traversal (src/fmm_funcs.cpp:17-123).  Writes at most cap
 * pairs to out (may be NULL) and returns the full count in *count. */
sbslpm_status sbslpm_dual_tree_traversal(int levels, const sbslpm_panel* panels, double theta,
                                         sbslpm_interact_pair* out, long cap, long* count);
/* The same traversal on the GPU (generation by generation: classification,
 * prefix sums, emission): the same list in the same order.  Host arrays in
 * and out; device workspace is allocated and freed inside the call. */
sbslpm_status sbslpm_dual_tree_traversal_device(int levels, const sbslpm_panel* panels, double theta,
                                                sbslpm_interact_pair* out, long cap, long* count);
/* The traversal as the treecode uses it (dual_tree_traversal_irreg,
 * src/fmm_funcs.cpp:125-231, has the same pairs and order on a uniform tree):
 * near[e] = 1 for the leaf pairs that failed the MAC (particle x particle),
 * 0 for the well-separated ones.  The _multi form runs one traversal per
 * theta (members) on the GPU in one launch series and writes the members'
 * lists one after the other (counts[m] pairs each, at most cap in all); the
 * treecode contexts and the ensemble build their lists with it. */
sbslpm_status sbslpm_dual_tree_traversal_flagged(int levels, const sbslpm_panel* panels, double theta,
                                                 sbslpm_interact_pair* out, char* near, long cap, long* count);
sbslpm_status sbslpm_dual_tree_traversal_device_multi(int levels, const sbslpm_panel* panels, int members,
                                                      const double* theta, sbslpm_interact_pair* out, char* near,
                                                      long cap, long* counts);
/* Host versions of interp_vals_bli / point_locate_panel
 * (src/interp_funcs_impl.hpp:11-142). */
sbslpm_status sbslpm_interp_vals_bli(double* basis, double xi, double eta, double min_xi, double max_xi,
                                     double min_eta, double max_eta, int degree);
int sbslpm_point_locate_panel(const sbslpm_panel* panels, double x, double y, double z);

/* ---------------- context ---------------- */

/* Builds the panel tree and interaction list for cfg, precomputes the static
 * geometry on the device and allocates the step workspace (all device memory
 * the step needs is owned by the context). */
sbslpm_status sbslpm_create(const sbslpm_config* cfg, sbslpm_ctx** out);
sbslpm_status sbslpm_destroy(sbslpm_ctx* ctx);
/* Orders all later work of ctx on this cudaStream_t (NULL = the legacy
 * default stream).  Until it is called, ctx uses a stream of its own.
 * Treecode contexts also run each stage's tree passes on a second stream of
 * their own, forked from and joined back to this one by events, so every
 * call's work still starts after, and ends before, the work this stream
 * holds around it. */
sbslpm_status sbslpm_set_stream(sbslpm_ctx* ctx, void* cuda_stream);
/* sizes[0..3] = panel_count, leaf_count, q, interaction_count */
sbslpm_status sbslpm_get_sizes(const sbslpm_ctx* ctx, long* sizes);
/* Host copies of the context's panel table (panel_count entries) and
 * interaction list (interaction_count entries, reference order). */
sbslpm_status sbslpm_get_panels(const sbslpm_ctx* ctx, sbslpm_panel* out);
sbslpm_status sbslpm_get_interactions(const sbslpm_ctx* ctx, sbslpm_interact_pair* out);
/* Number of kernels this library has launched in this process (graph
 * replays count every kernel node). */
long sbslpm_kernel_launches(void);

/* ---------------- the step ---------------- */

/* Replaces bve_back_rk4_step (src/bve_time_step.cpp:311-419; declared in
 * src/bve_time_step.hpp:7-13).  Device pointers: xcos, ycos, zcos, area are
 * [leaf][q]; vors is advanced in place; vel_x/y/z receive the stage-0
 * velocity (the reference's vel_x/y/z); tracers [leaf][q][tracer_count] are
 * remapped in place (may be NULL when tracer_count is 0).  time is the
 * step's time in seconds (read by the forcing, unused without it).  Host
 * memory among the arguments is refused with SBSLPM_ERR_ARG (the same holds
 * for the run, SWE and batch steps); sbslpm_bve_step_host takes host arrays. */
sbslpm_status sbslpm_bve_step(sbslpm_ctx* ctx, const double* xcos, const double* ycos, const double* zcos,
                              const double* area, double* vors, double* vel_x, double* vel_y, double* vel_z,
                              double* tracers, double time);
/* The same step on HOST arrays (the layout and meaning of sbslpm_bve_step's
 * arguments; pinned host memory gives the fastest copies, pageable memory
 * works).  The inputs are copied to device buffers the context allocates on
 * first use; the stage-0 velocity is copied back on a second stream while
 * stages 1-3 run, and vors / tracers after the remap.  Returns when every
 * output is in host memory.  The reference's bve_back_rk4_step on Kokkos
 * HostSpace Views (its OpenMP build) maps onto this call. */
sbslpm_status sbslpm_bve_step_host(sbslpm_ctx* ctx, const double* xcos, const double* ycos, const double* zcos,
                                   const double* area, double* vors, double* vel_x, double* vel_y, double* vel_z,
                                   double* tracers, double time);
/* 1 when p is memory the device can address as a device pointer
 * (cudaMalloc'd, managed, or a CUDA tensor's storage), 0 for host memory
 * (pageable or pinned), -1 when the query fails. */
int sbslpm_pointer_on_device(const void* p);
/* nsteps consecutive steps, captured once as a CUDA graph and replayed. */
sbslpm_status sbslpm_bve_run(sbslpm_ctx* ctx, const double* xcos, const double* ycos, const double* zcos,
                             const double* area, double* vors, double* vel_x, double* vel_y, double* vel_z,
                             double* tracers, double time, int nsteps);
/* One velocity evaluation of the step (its first stage, sources on the grid)
 * into vel_x/y/z ([leaf][q]): the Biot-Savart velocity of vors by the
 * context's method -- the velocity part of bve_back_rk4_step
 * (src/bve_time_step.cpp:333-350).  On a sharded context without a
 * communicator only the rank's own slice (sbslpm_shard_range) is written.
 * Refused on a forced context (its velocity includes the step's forcing). */
sbslpm_status sbslpm_bve_velocity(sbslpm_ctx* ctx, const double* xcos, const double* ycos, const double* zcos,
                                  const double* area, const double* vors, double* vel_x, double* vel_y,
                                  double* vel_z);

/* ---------------- one problem over several GPUs (treecode) ----------------
 *
 * Replaces the reference's MPI split of the velocity work
 * (src/fmm_interactions/bve_vel.cpp:15-33: each rank takes a slice of the
 * interaction list; src/bve_time_step.cpp:346-348: MPI_Allreduce of the
 * velocity).  One process per GPU, each with its own context on the same
 * problem.  Rank r of nranks owns the particles of a contiguous slice of the
 * tree leaves (sbslpm_shard_range): it evaluates the near field, the
 * well-separated pairs that land on its slice and its particles' velocities;
 * after every RK stage an NCCL all-gather gives every rank the whole
 * velocity, and the remap runs on every rank.  The result is bit-identical to
 * the one-GPU step.  The adjoint and shallow-water paths refuse a context of
 * more than one rank. */

/* A fresh NCCL unique id (128 bytes) for sbslpm_set_shard; rank 0 makes it and
 * the host sends it to the other ranks (NCCL is loaded at run time:
 * SBSLPM_ERR_NO_DEVICE when libnccl.so.2 cannot be loaded). */
sbslpm_status sbslpm_shard_unique_id(unsigned char* id);
/* Makes the context rank `rank` of `nranks` (nranks must divide the tree's
 * leaf count; 1 restores the whole problem).  With nccl_id (128 bytes, the
 * same on every rank) it joins the ranks' communicator -- every rank calls it
 * together; a rank missing for timeout_s seconds (<= 0: 300) ends it with
 * SBSLPM_ERR_TIMEOUT and leaves the context as it was.  Without nccl_id a
 * context of more than one rank only
 * evaluates its own slice (sbslpm_bve_velocity) and refuses whole steps.
 * Launch shapes are timed again on the next call. */
sbslpm_status sbslpm_set_shard(sbslpm_ctx* ctx, int rank, int nranks, const unsigned char* nccl_id,
                               double timeout_s);
/* The rank's particles: indices [first, first + count) of a [leaf][q] field. */
sbslpm_status sbslpm_shard_range(const sbslpm_ctx* ctx, long* first, long* count);
/* Ends the context's communicator (also done by sbslpm_destroy); every rank
 * calls it together. */
sbslpm_status sbslpm_shard_release(sbslpm_ctx* ctx);

/* ---------------- pieces of the step (device pointers) ---------------- */

/* Replaces upward_pass (src/fmm_funcs.cpp:341-355): leaf strengths
 * area*pots ([leaf][q]) anterpolated up the tree into proxy_source
 * ([panel][q], overwritten). */
sbslpm_status sbslpm_upward_pass(sbslpm_ctx* ctx, const double* area, const double* pots, double* proxy_source);
/* Replaces bve_vel_interactions (src/fmm_interactions/bve_vel.cpp:9-37):
 * proxy-target velocities of every pair in the interaction list with sources
 * at proj(proxy + disp); disp_* and source are [panel][q]; target_1..3
 * ([panel][q]) are accumulated into, as in the reference. */
sbslpm_status sbslpm_bve_vel_interactions(sbslpm_ctx* ctx, const double* disp_x, const double* disp_y,
                                          const double* disp_z, const double* source, double* target_1,
                                          double* target_2, double* target_3);
/* Replaces downward_pass_3 (src/fmm_funcs.cpp:374-392): targets ([panel][q],
 * updated in place as in the reference) interpolated down the tree; sols_*
 * ([leaf][q]) receive the leaf values. */
sbslpm_status sbslpm_downward_pass_3(sbslpm_ctx* ctx, double* target_1, double* target_2, double* target_3,
                                     double* sols_1, double* sols_2, double* sols_3);
/* Replaces the bve_find_departure_points functor (src/bve_time_step.cpp:172-309):
 * v0..v3 are [3][leaf][q] (x, y, z blocks); dep_* are [leaf][q]. */
sbslpm_status sbslpm_bve_departure(sbslpm_ctx* ctx, const double* xcos, const double* ycos, const double* zcos,
                                   const double* v0, const double* v1, const double* v2, const double* v3,
                                   double dt, double* dep_x, double* dep_y, double* dep_z);
/* Replaces the bve_departure_to_target functor (src/bve_time_step.cpp:15-67):
 * new_vors = BLI(vors)(dep) + 2 omega (dep_z - zcos); tracers likewise. */
sbslpm_status sbslpm_bve_remap(sbslpm_ctx* ctx, const double* zcos, const double* dep_x, const double* dep_y,
                               const double* dep_z, const double* vors, const double* tracers, double* new_vors,
                               double* new_tracers);

/* ---------------- shallow water, SWE v2 (device pointers) ---------------- */

/* The shallow-water entry points need interp_degree >= 2 (the one-sided
 * finite-difference stencils of src/deriv_funcs_impl.hpp:94-185 read three
 * nodes) and the spectral FMM (proxy_degree 0) or the direct velocity.
 * Fields are [leaf][q]; vel_* hold the velocity, base_* the base tendencies
 * the driver computes once (sbslpm_swe_init).  The reference's
 * one_d_no_of_points / two_d_to_1d arguments are not taken: the context keeps
 * the same map (sbslpm_cubed_sphere_2d_to_1d), built once from its grid. */

/* Replaces swe_back_rk4_step_2 (src/swe_time_step_2.cpp:785-1035, declared in
 * src/swe_time_step_2.hpp:7-14): four velocity evaluations of the vorticity
 * (displaced sources) and divergence (fixed sources) fields, finite-difference
 * tendencies, forward-Euler arrival values, backward RK4 departure points and
 * the remap of vorticity and tracers.  vors, divs, height and tracers are
 * advanced in place; vel_x/y/z receive the first-stage velocity (unified
 * across panel edges as the reference leaves it).  time is unused. */
sbslpm_status sbslpm_swe_step(sbslpm_ctx* ctx, const double* xcos, const double* ycos, const double* zcos,
                              const double* area, double* vors, double* divs, double* height, double* vel_x,
                              double* vel_y, double* vel_z, double* tracers, const double* base_vor_tend,
                              const double* base_div_tend, const double* base_h_tend, double time);
/* nsteps steps of the reference driver's loop (executables/swe_time_evo.cpp:413-418):
 * each step followed by unify_boundary_vals of vors, divs and height;
 * captured once as a CUDA graph and replayed. */
sbslpm_status sbslpm_swe_run(sbslpm_ctx* ctx, const double* xcos, const double* ycos, const double* zcos,
                             const double* area, double* vors, double* divs, double* height, double* vel_x,
                             double* vel_y, double* vel_z, double* tracers, const double* base_vor_tend,
                             const double* base_div_tend, const double* base_h_tend, double time, int nsteps);
/* The driver's set-up before its time loop (executables/swe_time_evo.cpp:352-410):
 * velocity of the undisplaced vorticity and divergence (unified), and the
 * base tendencies computed from it (unified).  vel_* and base_* are written. */
sbslpm_status sbslpm_swe_init(sbslpm_ctx* ctx, const double* xcos, const double* ycos, const double* zcos,
                              const double* area, const double* vors, const double* divs, const double* height,
                              double* vel_x, double* vel_y, double* vel_z, double* base_vor_tend,
                              double* base_div_tend, double* base_h_tend);
/* Replaces swe_tendency_computation_2 (src/swe_time_step_2_impl.hpp:10-128)
 * over every leaf panel: vorticity, divergence and height tendencies from the
 * velocity, vorticity, divergence, height and surface (the height with
 * topography) fields. */
sbslpm_status sbslpm_swe_tendencies(sbslpm_ctx* ctx, const double* xcos, const double* ycos, const double* zcos,
                                    const double* vel_x, const double* vel_y, const double* vel_z,
                                    const double* vors, const double* divs, const double* height,
                                    const double* surface, double* vor_tend, double* div_tend, double* h_tend);
/* Replaces unify_boundary_vals (src/initialize_cubed_sphere.cpp:364-370):
 * every copy of a grid point shared by several panels gets the mean of the
 * copies (summed in [leaf][q] order). */
sbslpm_status sbslpm_unify_boundary_vals(sbslpm_ctx* ctx, double* vals);
/* The shallow-water velocity on the treecode (contexts with proxy_degree > 0
 * and leaves of at most 256 particles; the SWE step uses it then): vorticity
 * sources at the grid points displaced by (dx, dy, dz) (re-projected), with
 * strengths w_vor, and divergence sources at the grid points with strengths
 * w_div (A x q each), near leaf pairs particle x particle, every
 * well-separated pair proxy x proxy -- the design of the reference's
 * irregular-point FMM (swe_vel_panel_interaction_ll,
 * src/fmm_interactions/swe_vel_impl.hpp:149-288).  u_* (A x q) receive the
 * velocity at the grid points. */
sbslpm_status sbslpm_swe_tree_velocity(sbslpm_ctx* ctx, const double* dx, const double* dy, const double* dz,
                                       const double* w_vor, const double* w_div, double* u_x, double* u_y,
                                       double* u_z);
/* Replaces swe_vel_interactions_2 (src/fmm_interactions/swe_vel.cpp:39-67):
 * proxy-target velocities of vorticity sources at proj(proxy + disp) and
 * divergence sources at the fixed proxies; [panel][q] inputs; target_1..3
 * are accumulated into, as in the reference. */
sbslpm_status sbslpm_swe_vel_interactions(sbslpm_ctx* ctx, const double* disp_x, const double* disp_y,
                                          const double* disp_z, const double* source_vor, const double* source_div,
                                          double* target_1, double* target_2, double* target_3);
/* Host.  Replaces cubed_sphere_2d_to_1d (src/initialize_cubed_sphere.cpp:290-326)
 * with a hashed search (the reference compares every point with every
 * distinct point found so far): two_d_to_1d [leaf][q] receives the index of
 * each grid point's distinct position (numbered in order of first appearance,
 * coordinates equal within 1e-15), counts [unique] how many grid points share
 * it.  counts must hold leaf_count*interp_degree^2 + 2 entries; *unique
 * receives the number found. */
sbslpm_status sbslpm_cubed_sphere_2d_to_1d(long n_leaves, int degree, const double* xcos, const double* ycos,
                                           const double* zcos, int* two_d_to_1d, int* counts, long* unique);

/* ---------------- adjoint (device pointers) ---------------- */

/* No counterpart in the reference (it has no derivatives).  One reverse step
 * of bve_back_rk4_step: given the step's input vorticity vors (the per-step
 * checkpoint) and the adjoint of its output vorticity vors_bar_next, writes
 * the adjoint of the input vorticity, vors_bar = (d vors_next / d vors)^T
 * vors_bar_next, through the four velocity evaluations (source positions and
 * strengths), the departure search and the remap.  The forward step is
 * recomputed from the checkpoint inside the call.  Runs on every velocity
 * method: the direct sum and the treecode (proxy_degree > 0) in float64 or
 * mixed precision (mixed: the forward recomputed in mixed precision and the
 * transposed pair sums in float32 on coordinates packed relative to their
 * leaves' or panels' centres, the rest float64), and the reference's
 * spectral FMM in float64 (displaced proxies on every panel; the non-leaf
 * displacement interpolation reversed).  Needs no tracers or forcing.
 * Locating points in panels is piecewise constant and is not
 * differentiated. */
sbslpm_status sbslpm_bve_adjoint_step(sbslpm_ctx* ctx, const double* xcos, const double* ycos, const double* zcos,
                                      const double* area, const double* vors, const double* vors_bar_next,
                                      double* vors_bar);
/* Vector-Jacobian product of sbslpm_direct_sum_bve (float64) with respect to
 * the sources: given ubar at the targets, strength_bar_j = sum_i ubar_i .
 * du_i/dq_j and s*_bar = the same with respect to the source positions
 * (written, not accumulated).  stream: cudaStream_t or NULL. */
sbslpm_status sbslpm_direct_sum_bve_vjp(long n_targets, const double* tx, const double* ty, const double* tz,
                                        const double* ubar_x, const double* ubar_y, const double* ubar_z,
                                        long n_sources, const double* sx, const double* sy, const double* sz,
                                        const double* strength, double eps, double* strength_bar, double* sx_bar,
                                        double* sy_bar, double* sz_bar, void* stream);

/* ---------------- batched ensemble (device pointers) ---------------- */

/* No counterpart in the reference (its drivers run one problem per process).
 * An ensemble of `members` BVE problems on one particle grid (base->levels,
 * base->interp_degree, kernel_eps, omega, dt, precision, leaf_size shared),
 * each with its own vorticity, MAC parameter theta[m] and treecode proxy
 * degree proxy_degree[m] (5..10), so the members' trees and interaction lists
 * differ.  A step is one launch per phase over all members (the
 * well-separated proxy interactions once per proxy degree in use); member m's
 * result is the one a single context with (theta[m], proxy_degree[m]) gives
 * on the same input.  The near-field launch shape is chosen by timing the
 * candidates on the first step. */
typedef struct sbslpm_batch sbslpm_batch;
sbslpm_status sbslpm_batch_create(const sbslpm_config* base, int members, const double* theta,
                                  const int* proxy_degree, sbslpm_batch** out);
sbslpm_status sbslpm_batch_destroy(sbslpm_batch* batch);
sbslpm_status sbslpm_batch_set_stream(sbslpm_batch* batch, void* cuda_stream);
/* sizes[0..3] = members, leaf_count, q, particles per member */
sbslpm_status sbslpm_batch_get_sizes(const sbslpm_batch* batch, long* sizes);
/* One bve_back_rk4_step of every member.  xcos..area: [leaf][q] (shared);
 * vors: [members][leaf][q], advanced in place; vel: [members][3][leaf][q]
 * receives the stage-0 velocities. */
sbslpm_status sbslpm_batch_step(sbslpm_batch* batch, const double* xcos, const double* ycos, const double* zcos,
                                const double* area, double* vors, double* vel, double time);
/* nsteps steps, captured once as a CUDA graph and replayed. */
sbslpm_status sbslpm_batch_run(sbslpm_batch* batch, const double* xcos, const double* ycos, const double* zcos,
                               const double* area, double* vors, double* vel, double time, int nsteps);
/* The autotuner's choice: shape[0..3] = threads per block, targets per thread,
 * source-list splits, candidates timed; *ms_per_launch of the chosen shape. */
sbslpm_status sbslpm_batch_tuning(const sbslpm_batch* batch, int* shape, double* ms_per_launch);
/* Fixes the near-field launch shape instead of the autotuner's choice:
 * threads per block 64 | 128 | 256, targets per thread 1 | 2 | 4 (threads x
 * targets >= particles per treecode leaf), source-list splits 1..4.  The
 * split count sets the order in which a target's near-field partial sums are
 * added (a single context uses 2). */
sbslpm_status sbslpm_batch_set_tuning(sbslpm_batch* batch, int threads, int targets_per_thread, int splits);
/* Pair evaluations of one velocity evaluation over all members: near field
 * (particle x particle) and well-separated (proxy x proxy). */
sbslpm_status sbslpm_batch_pairs(const sbslpm_batch* batch, double* near_pairs, double* far_pairs);
/* Well-separated (cluster-cluster) interactions of a mixed-precision batch:
 * mode -1 = chosen per proxy-degree group by the autotuner of the first
 * step (the default), 0 = CUDA-core float32 pairs per member (bit-exact with
 * single contexts on the whole-panel well-separated kernel,
 * sbslpm_set_cc_tuning(ctx, 0, 0), with sbslpm_batch_set_stage0_shared(batch,
 * 0)), 1 = tensor-core GEMM over the members sharing a proxy
 * degree in 3xTF32, 2 = the same GEMM in one TF32 pass, 3 = CUDA-core
 * float32 pairs whose distances and reciprocals are shared by groups of 4
 * theta-consecutive members of a degree group (the proxies never move, so a
 * cluster pair's geometry is the same for every member).  Float64 batches
 * accept mode 0 only.  sbslpm_batch_cc_info reports the mode, the union of
 * the members' well-separated pairs over the degree groups (cluster pairs),
 * and the MMA flops one velocity evaluation issues.  sbslpm_batch_cc_groups
 * reports per group (at most n): proxy degree, members, the mode in use and
 * the autotuner's timings of one launch in modes 0, 1 and 3 (0 before the
 * first step). */
sbslpm_status sbslpm_batch_set_cc_mode(sbslpm_batch* batch, int mode);
/* Mixed-precision batches: the near field of each step's first stage, where
 * every member's particles sit on the shared grid, evaluated once per leaf
 * pair for theta-sorted groups of 8 members and applied to their strengths
 * (shared = 1, the default), or by every member's own near kernel (0: the
 * arithmetic of single contexts, bit-exact with them).  The two differ only
 * in the order of float32 additions.  SBSLPM_ERR_CONFIG for float64 batches.
 * Replaces nothing in the reference (one problem per process there). */
sbslpm_status sbslpm_batch_set_stage0_shared(sbslpm_batch* batch, int shared);
/* Mixed-precision batches: the near-field pair form of the members' own near
 * kernel, as sbslpm_set_near_form (set-up chooses the expanded form when every
 * member's near list allows it).  A member is bit-exact with a single context
 * only when both use the same form. */
sbslpm_status sbslpm_batch_set_near_form(sbslpm_batch* batch, int expanded);
sbslpm_status sbslpm_batch_near_form(const sbslpm_batch* batch, int* expanded);
sbslpm_status sbslpm_batch_cc_info(const sbslpm_batch* batch, int* mode, double* union_pairs, double* mma_flops);
/* Wall time (seconds) of sbslpm_batch_create's list build: every member's
 * tree traversal on the GPU in one launch series, with the lists' CSR
 * assembly on the host. */
sbslpm_status sbslpm_batch_setup_times(const sbslpm_batch* batch, double* lists_s);
/* Test of the tensor-core kernel's failure path (no counterpart in the
 * reference).  on = 1: every CTA of the tensor-core well-separated kernel
 * (modes 1 and 2) withholds one producer thread's arrival on its first
 * chunk's barrier and bounds its waits to 2 ms, so the MMA warp's wait runs
 * out before any MMA is issued: the CTA frees its tensor memory and returns,
 * and the step reports SBSLPM_ERR_TIMEOUT (its results are not valid).
 * on = 0 restores the normal one-second bound. */
sbslpm_status sbslpm_batch_set_wait_test(sbslpm_batch* batch, int on);
sbslpm_status sbslpm_batch_cc_groups(const sbslpm_batch* batch, int n, int* degree, int* members, int* mode,
                                     double* ms_cuda_cores, double* ms_tensor_cores, double* ms_shared);

/* ---------------- Poisson (inverse Laplacian) FMM ---------------- */

/* The solve of executables/poisson_eq_fmm.cpp:128-160 on a spectral-FMM
 * context (proxy_degree 0, velocity SBSLPM_VEL_FMM): upward_pass, then
 * poisson_fmm_interactions (src/fmm_interactions/inverse_poisson.cpp:9-34,
 * kernel -1/(4 pi) log(1 - x.y), pairs with x.y >= 1 - 1e-15 skipped), then
 * downward_pass (src/fmm_funcs.cpp:357-372); soln[leaf][q] is written.
 * sbslpm_poisson_fmm_interactions adds into target[panel][q] from
 * source[panel][q] like the reference; sbslpm_downward_pass updates
 * proxy_target[panel][q] in place and writes soln[leaf][q].  Device pointers. */
sbslpm_status sbslpm_poisson_fmm(sbslpm_ctx* ctx, const double* area, const double* pots, double* soln);
sbslpm_status sbslpm_poisson_fmm_interactions(sbslpm_ctx* ctx, const double* source, double* target);
sbslpm_status sbslpm_downward_pass(sbslpm_ctx* ctx, double* proxy_target, double* soln);

/* ---------------- output path (the drivers' per-step output) ---------------- */

/* Replaces interp_to_latlon_host (src/interp_funcs.hpp:22-77, host, OpenMP):
 * a [leaf][q] field interpolated to the nlat x nlon grid of latitudes lats
 * and longitudes lons (degrees), out[nlat][nlon]; all device pointers, on the
 * context's stream. */
sbslpm_status sbslpm_interp_to_latlon(sbslpm_ctx* ctx, const double* data, int nlat, const double* lats, int nlon,
                                      const double* lons, double* out);
/* Replaces xyz_vel_to_uv_vel (src/general_utils_impl.hpp:195-229): zonal and
 * meridional velocity of the [leaf][q] grid (device pointers). */
sbslpm_status sbslpm_xyz_vel_to_uv_vel(sbslpm_ctx* ctx, const double* x, const double* y, const double* z,
                                       const double* vel_x, const double* vel_y, const double* vel_z, double* vel_u,
                                       double* vel_v);
/* The drivers' output grid (executables/bve_time_evo.cpp:93-95, 206-211):
 * spacing 2^floor(log2(sqrt(4 pi / point_count) 180 / pi)) degrees,
 * nlat = 180 / spacing + 1 latitudes from -90, nlon = 360 / spacing
 * longitudes from 0; lats / lons (host, may be NULL) receive the values. */
sbslpm_status sbslpm_output_grid(long point_count, double* spacing, int* nlat, int* nlon, double* lats,
                                 double* lons);

/* netCDF classic (64-bit offset) writer for the drivers' output files; the
 * calls mirror the netCDF library's nc_create, nc_def_dim, nc_def_var,
 * nc_put_att_text / _int / _double, nc_enddef, nc_put_vara_double / _int and
 * nc_close as executables/bve_time_evo.cpp:125-358 uses them.  Types: 4 =
 * int, 6 = double.  varid -1 names the global attributes.  start / count
 * NULL = the whole variable.  Host memory. */
typedef struct sbslpm_nc sbslpm_nc;
sbslpm_status sbslpm_nc_create(const char* path, sbslpm_nc** out);
sbslpm_status sbslpm_nc_def_dim(sbslpm_nc* nc, const char* name, long len, int* dimid);
sbslpm_status sbslpm_nc_def_var(sbslpm_nc* nc, const char* name, int type, int ndims, const int* dimids, int* varid);
sbslpm_status sbslpm_nc_put_att_text(sbslpm_nc* nc, int varid, const char* name, const char* text);
sbslpm_status sbslpm_nc_put_att_int(sbslpm_nc* nc, int varid, const char* name, long n, const int* vals);
sbslpm_status sbslpm_nc_put_att_double(sbslpm_nc* nc, int varid, const char* name, long n, const double* vals);
sbslpm_status sbslpm_nc_enddef(sbslpm_nc* nc);
sbslpm_status sbslpm_nc_put_vara_double(sbslpm_nc* nc, int varid, const long* start, const long* count,
                                        const double* data);
sbslpm_status sbslpm_nc_put_vara_int(sbslpm_nc* nc, int varid, const long* start, const long* count, const int* data);
sbslpm_status sbslpm_nc_close(sbslpm_nc* nc);

/* ---------------- direct sums (device pointers, no context) ---------------- */

/* Biot-Savart direct sum on the sphere (the reference's BVE kernel,
 * src/fmm_interactions/bve_vel_impl.hpp:113-118, over all pairs):
 *   u_i = -1/(4 pi) sum_j (x_i x y_j) s_j / (1 - x_i.y_j + eps)
 * evaluated as x_i x sum_j s_j (y_j - x_i) / (|y_j - x_i|^2/2 + eps).
 * Pairs with y_j == x_i contribute nothing.  precision: SBSLPM_FP64 or
 * SBSLPM_MIXED.  stream: cudaStream_t or NULL. */
sbslpm_status sbslpm_direct_sum_bve(long n_targets, const double* tx, const double* ty, const double* tz,
                                    long n_sources, const double* sx, const double* sy, const double* sz,
                                    const double* strength, double eps, int precision, double* u_x, double* u_y,
                                    double* u_z, void* stream);
/* Replaces direct_sum_inv_lap (src/direct_sum.cpp:8-15, inv_lap
 * src/direct_sum_impl.hpp:20-27): soln_i += sum_{j != i}
 * -1/(4 pi) log(1 - x_i.x_j) area_j pots_j (soln accumulated into). */
sbslpm_status sbslpm_direct_sum_inv_lap(long n, const double* x, const double* y, const double* z,
                                        const double* area, const double* pots, double* soln, void* stream);

/* No counterpart in the reference.  The same Biot-Savart direct sum as
 * sbslpm_direct_sum_bve, for callers that cannot let a library allocate
 * device memory: a host model that fixes its device footprint at start-up, or
 * that routes every device allocation through its own allocator, cannot
 * accept the cudaMallocAsync/cudaFreeAsync of scratch that
 * sbslpm_direct_sum_bve makes on every call.  This entry point allocates
 * nothing: its scratch is one fixed 16 MiB array compiled into the library,
 * which each GPU that loads the library holds until the process exits.
 * Limit: n_targets <= 699,050 (3 * n_targets doubles of scratch); larger
 * calls return SBSLPM_ERR_ARG with a message and do nothing.  Results equal
 * sbslpm_direct_sum_bve's up to summation order: from about 100,000 targets
 * the scratch holds fewer source groups than that entry point would use.
 * The first call on each device looks the array's device address up
 * (cudaGetSymbolAddress, with that device current) and keeps it, so make
 * that first call before any stream capture, and do not reset the device
 * (cudaDeviceReset) while the library is in use.  Every call on a device shares the one array and each call
 * overwrites the parts it uses, so calls whose kernels overlap on the GPU
 * (different streams or host threads) race: serialise them.  Synchronises
 * the stream before returning. */
sbslpm_status sbslpm_direct_sum_bve_noalloc(long n_targets, const double* tx, const double* ty, const double* tz,
                                            long n_sources, const double* sx, const double* sy, const double* sz,
                                            const double* strength, double eps, int precision, double* u_x,
                                            double* u_y, double* u_z, void* stream);

/* ---------------- measurement ---------------- */

/* Average device time of one launch of the interaction kernel alone (the
 * dominant kernel of the step), over reps launches on the current sources of
 * the context (those of the last stage run), timed with CUDA events on the
 * context's stream.  *pairs receives the pair evaluations per launch. */
sbslpm_status sbslpm_time_interactions(sbslpm_ctx* ctx, int reps, double* ms_per_launch, double* pairs);
/* Treecode contexts (proxy_degree > 0): the near-field launch shape.  The
 * first step of a context times every shape (threads per block 64 | 128 |
 * 256 x targets per thread covering a treecode leaf, 1..4 source-list
 * splits) and keeps the fastest; sbslpm_set_near_tuning fixes one instead
 * (the split count sets the order in which a target's near-field partial
 * sums are added).  shape[0..3] = threads, targets per thread, splits,
 * candidates timed. */
sbslpm_status sbslpm_set_near_tuning(sbslpm_ctx* ctx, int threads, int targets_per_thread, int splits);
sbslpm_status sbslpm_near_tuning(const sbslpm_ctx* ctx, int* shape, double* ms_per_launch);
/* Mixed-precision treecode contexts with 256-particle leaves: the first RK
 * stage's near field can run two-sided.  At that stage the sources are the
 * grid particles themselves, so a leaf pair's distances and reciprocals
 * serve both directions: one CTA per unordered near leaf pair (diagonal and
 * unmirrored pairs one-sided) writes float32 sums per list entry, added per
 * leaf in list order.  The first-step timing keeps it for stage 0 when it
 * beats the chosen shape; sbslpm_set_near_mutual turns it on or off (it
 * changes the order of float32 additions only).  *ms_per_launch: its timed
 * launch (with the per-leaf sums). */
sbslpm_status sbslpm_set_near_mutual(sbslpm_ctx* ctx, int on);
/* Mixed-precision treecode contexts: the arithmetic of the near-field pair
 * kernel.  0 = difference form: d = (source - target) in packed float32,
 * |d|^2 + eps, g d accumulated (10 float32 operations per pair).  1 =
 * expanded form: |d|^2 + eps = (|s|^2 + eps) + |b|^2 + 2 b.s with the
 * source's offset s from its leaf centre and b = the target's offset to that
 * centre, and sum g d = sum r (w s) + b sum r w (8 operations per pair).  The
 * expanded form rounds the denominator relative to (|b| + |s|)^2 rather than
 * to |d|; set-up chooses it when eps is at least 3 * 2^-14 times the largest
 * (|c_S - c_T| + 2 r_T + 2 r_S)^2 / 2 over the near leaf pairs (rounding at
 * most 2^-10 of eps), else the difference form.  This call overrides the
 * choice (1 needs kernel_eps > 0). */
sbslpm_status sbslpm_set_near_form(sbslpm_ctx* ctx, int expanded);
sbslpm_status sbslpm_near_form(const sbslpm_ctx* ctx, int* expanded);
sbslpm_status sbslpm_near_mutual(const sbslpm_ctx* ctx, int* on, double* ms_per_launch);
/* Treecode contexts with 36..121 proxies (proxy_degree 5..10): the launch
 * shape of the well-separated (cluster-cluster) interactions, either one
 * block of four warps per target panel (slots 0, chunk length 0, the kernel
 * of the batched CUDA-core path) or blocks of 1 | 2 | 3 | 4 | 6 | 8 chunk
 * slots of q threads each (rounded up to whole warps: at most 512 threads,
 * at most a fifth of them idle), a chunk being 1..4 consecutive list entries
 * of one target panel.  The first step times every shape with the near field
 * and keeps the fastest; sbslpm_set_cc_tuning fixes one instead (the chunk
 * length sets the order in which a target's sums are added, the slot count
 * does not; SBSLPM_ERR_CONFIG for other proxy counts).  shape[0..3] = slots,
 * chunk length, threads per block, candidates timed.  Both replace nothing
 * in the reference (its interactions run one list entry per Kokkos
 * iteration, src/fmm_interactions/bve_vel.cpp:35-150). */
sbslpm_status sbslpm_set_cc_tuning(sbslpm_ctx* ctx, int slots, int chunk_len);
sbslpm_status sbslpm_cc_tuning(const sbslpm_ctx* ctx, int* shape, double* ms_per_launch);
/* Mixed-precision treecode contexts (36..121 proxies) also have a barrier-free
 * form of the chunked kernel: each slot reads its source proxies straight
 * from a pair-transposed copy through the L1 cache instead of staging them in
 * shared memory, with targets_per_thread (1 | 2) target proxies per thread.
 * A third form keeps the staged form's slots but brings each slot's source
 * panels into shared memory with bulk copies (the TMA engine's
 * cp.async.bulk), double-buffered through mbarriers so that the next panel
 * arrives while the current one is evaluated and no barrier spans the block;
 * its waits are bounded (a copy that never lands gives SBSLPM_ERR_TIMEOUT).
 * A fourth form runs one warp per chunk: the lanes hold the target panel's
 * proxies, ceil(q / 32) per lane, so every staged source pair feeds that many
 * targets, and each warp stages its own source panels with cp.async into two
 * buffers of its own (the next entry's panel in flight during the current
 * one), synchronising with __syncwarp only; `warps` (1, 2, 4 or 8) warps per
 * block.  All four forms give bit-identical results for the same chunk
 * length.  The first-step timing includes all of them;
 * sbslpm_set_cc_tuning_direct, sbslpm_set_cc_tuning_bulk and
 * sbslpm_set_cc_tuning_warp fix one (the chunk length sets the order of the
 * float64 additions, as above); sbslpm_cc_form reports 0 for the staged
 * form, 1 | 2 (targets per thread) for the barrier-free one, 3 for the
 * bulk-copy one, 4 for the warp-per-chunk one. */
sbslpm_status sbslpm_set_cc_tuning_direct(sbslpm_ctx* ctx, int slots, int chunk_len, int targets_per_thread);
sbslpm_status sbslpm_set_cc_tuning_bulk(sbslpm_ctx* ctx, int slots, int chunk_len);
sbslpm_status sbslpm_set_cc_tuning_warp(sbslpm_ctx* ctx, int warps, int chunk_len);
sbslpm_status sbslpm_cc_form(const sbslpm_ctx* ctx, int* targets_per_thread);
/* CUDA-core fused multiply-add throughput of this GPU, measured with
 * independent FMA chains on every SM for about ms milliseconds: kind 0 =
 * float32, 1 = float64.  Returns FLOP/s (2 per FMA) in *flops. */
sbslpm_status sbslpm_measure_fma_peak(int kind, double ms, double* flops);

#ifdef __cplusplus
}
#endif
#endif /* SBSLPM_H */
