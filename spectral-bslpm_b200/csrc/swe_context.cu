// Shallow-water (SWE v2) step orchestration and its C ABI: swe_back_rk4_step_2
// (src/swe_time_step_2.cpp:785-1035) on the context's stream, the driver's
// set-up and time loop (executables/swe_time_evo.cpp:352-418), and the
// piecewise entry points (tendencies, edge unification, interactions).
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "context_internal.hpp"
#include "geometry.cuh"

using namespace sbslpm;

namespace sbslpm {
namespace {

// Entries per chunk of the mixed treecode's well-separated list for the SWE
// (the chunk lists of 1..4 entries are built with the treecode's lists).
constexpr int kSweCcLen = 2;

// Static tables and workspace of the SWE step, built on the first SWE call.
sbslpm_status swe_setup(sbslpm_ctx* c) {
  if (c->swe_ready) return SBSLPM_OK;
  if (c->d < 2)
    return set_last_error("the shallow-water step needs interp_degree >= 2 (three-node stencils)"), SBSLPM_ERR_CONFIG;
  if (c->tree && c->npl > 256)
    return set_last_error("the shallow-water treecode takes leaves of at most 256 particles"), SBSLPM_ERR_CONFIG;
  const long ln = (long)c->A * c->q;
  std::vector<double> interp, g(3 * ln), area(ln);
  build_interp(c->d, false, interp);
  build_points(c->L, c->d, c->panels, interp.data(), g.data(), g.data() + ln, g.data() + 2 * ln, area.data());
  const double *x = g.data(), *y = g.data() + ln, *z = g.data() + 2 * ln;

  c->two_d_to_1d.assign(ln, 0);
  const long U = unique_points(c->A, c->q, x, y, z, c->two_d_to_1d.data(), c->unique_counts);
  std::vector<int> ustart(U + 1, 0), umem(ln);
  for (long o = 0; o < ln; o++) ustart[c->two_d_to_1d[o] + 1]++;
  for (long u = 0; u < U; u++) ustart[u + 1] += ustart[u];
  std::vector<int> fill(ustart.begin(), ustart.end() - 1);
  for (long o = 0; o < ln; o++) umem[fill[c->two_d_to_1d[o]]++] = (int)o;

  std::vector<double> fd, ntan, pow15, filt, ptan;
  std::vector<int> pface;
  build_swe_tables(c->d, c->panels, c->off, c->A, x, y, z, fd, ntan, pow15, filt, ptan, pface);
  SB_TRY(upload(&c->s_fd, fd));
  SB_TRY(upload(&c->s_ntan, ntan));
  SB_TRY(upload(&c->s_pow15, pow15));
  SB_TRY(upload(&c->s_filt, filt));
  SB_TRY(upload(&c->s_ptan, ptan));
  SB_TRY(upload(&c->s_pface, pface));
  SB_TRY(upload(&c->s_ustart, ustart));
  SB_TRY(upload(&c->s_umem, umem));
  if (c->tree) {  // the divergence field on the treecode: particle sources and proxies
    const size_t fpn = (size_t)c->Pf * c->qx;
    SB_TRY(dalloc(&c->psrc2, (size_t)ln));
    SB_TRY(dalloc(&c->fsrc2, fpn));
    std::vector<double4> init(fpn);
    std::vector<double> fpx(3 * fpn);
    SB_CUDA(cudaMemcpy(fpx.data(), c->fpx, sizeof(double) * 3 * fpn, cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < fpn; i++) init[i] = make_double4(fpx[i], fpx[fpn + i], fpx[2 * fpn + i], 0.0);
    SB_CUDA(cudaMemcpy(c->fsrc2, init.data(), sizeof(double4) * fpn, cudaMemcpyHostToDevice));
    if (c->cfg.precision == SBSLPM_MIXED) {
      SB_TRY(dalloc(&c->psrcf2, (size_t)ln));
      SB_TRY(dalloc(&c->fsrcf2, fpn));
      if (c->n_cc > 0 && c->cc_chunks[kSweCcLen - 1] && swe_tree_cc_supported(c->qx))
        SB_TRY(dalloc(&c->swe_cc_partial, (size_t)c->n_cc * 6 * c->qx));
    }
  } else {
    const size_t pn = (size_t)c->P * c->q;
    if (!c->src) SB_TRY(dalloc(&c->src, pn));
    SB_TRY(dalloc(&c->src2, pn));
    if (c->cfg.precision == SBSLPM_MIXED) {
      if (!c->srcf) SB_TRY(dalloc(&c->srcf, pn));
      SB_TRY(dalloc(&c->srcf2, pn));
    }
    if (!c->tgt) SB_TRY(dalloc(&c->tgt, 3 * pn));
  }
  SB_TRY(dalloc(&c->tend, 9 * (size_t)ln));
  SB_TRY(dalloc(&c->avor, (size_t)ln));

  SweGeom& s = c->sgeom;
  s.g_over_a = c->cfg.g_over_a;
  s.unique = U;
  s.fd = c->s_fd;
  s.ntan = c->s_ntan;
  s.pow15 = c->s_pow15;
  s.filt = c->s_filt;
  s.ptan = c->s_ptan;
  s.pface = c->s_pface;
  s.ustart = c->s_ustart;
  s.umem = c->s_umem;
  s.srcf2 = c->tree ? c->fsrcf2 : c->srcf2;
  if (!c->tree) c->geom.srcf = c->srcf;
  c->swe_ready = true;
  return SBSLPM_OK;
}

// The treecode velocity of both fields (bltc_swe.cu): leaf sources and their
// anterpolation, then, on the auxiliary stream, the upward pass of each
// field, the SWE proxy kernel over the well-separated list and the downward
// pass, beside the near field of both fields; the leaf interpolation adds
// the two.  Piecewise mode with explicit displacements and strengths.
void swe_tree_velocity(sbslpm_ctx* c, int stage, double dtd, double dts, const double* vprev, const double* tprev,
                       const double* x, const double* y, const double* z, const double* area, const double* vors,
                       const double* divs, const double* dispx, const double* dispy, const double* dispz,
                       const double* wv, const double* wd, double* v) {
  cudaStream_t st = c->stream();
  const bool mixed = c->cfg.precision == SBSLPM_MIXED;
  const StepGeom& fg = c->fgeom;
  launch_bltc_swe_sources(c->tgeom, fg, c->ftab, stage, dtd, dts, vprev, tprev, x, y, z, vors, divs, area, dispx,
                          dispy, dispz, wv, wd, c->psrc, c->psrcf, c->psrc2, c->psrcf2, c->fsrc, c->fsrc2, mixed,
                          c->centre + 4 * (size_t)c->off, c->q, st);
  cudaStream_t tree_st = c->aux_stream ? c->aux_stream : st;
  if (c->aux_stream) {
    cudaEventRecord(c->ev_fork, st);
    cudaStreamWaitEvent(tree_st, c->ev_fork, 0);
  }
  launch_upward_fused(fg, 2, 0, 0.0, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, c->fsrc, mixed, tree_st);
  StepGeom fg2 = fg;  // the divergence proxies pack into their own buffer
  fg2.srcf = c->fsrcf2;
  launch_upward_fused(fg2, 2, 0, 0.0, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, c->fsrc2, mixed,
                      tree_st);
  if (c->swe_cc_partial)
    launch_swe_tree_cc(fg, c->fsrcf2, c->cc_chunks[kSweCcLen - 1], c->cc_nchunks[kSweCcLen - 1],
                       c->cc_cstart[kSweCcLen - 1], c->swe_cc_partial, c->ftgt, tree_st);
  else
    launch_swe_interactions(fg, c->sgeom, c->cfg.precision, c->fsrc, c->fsrc2, c->ftgt, tree_st);
  launch_downward_fused(fg, c->ftgt, nullptr, tree_st);
  if (c->aux_stream) cudaEventRecord(c->ev_join, tree_st);
  constexpr int kSplits = 4;
  launch_bltc_swe_near(c->tgeom, fg, c->cfg.precision, x, y, z, c->psrc, c->psrc2, c->psrcf, c->psrcf2, c->near,
                       kSplits, c->centre + 4 * (size_t)c->off, c->q, st);
  if (c->aux_stream) cudaStreamWaitEvent(st, c->ev_join, 0);
  launch_bltc_to_particles(c->tgeom, fg, c->ftgt, c->near, kSplits, v, st);
}

// One velocity evaluation of both source fields (stage 0 undisplaced;
// stage s displaced by dtd*vprev with the tendencies tprev applied over dts).
void swe_velocity_eval(sbslpm_ctx* c, int stage, double dtd, double dts, const double* vprev, const double* tprev,
                       const double* x, const double* y, const double* z, const double* area, const double* vors,
                       const double* divs, double* v) {
  cudaStream_t st = c->stream();
  const StepGeom& g = c->geom;
  const bool mixed = c->cfg.precision == SBSLPM_MIXED;
  if (c->tree) {
    swe_tree_velocity(c, stage, dtd, dts, vprev, tprev, x, y, z, area, vors, divs, nullptr, nullptr, nullptr, nullptr,
                      nullptr, v);
    return;
  }
  if (c->cfg.velocity == SBSLPM_VEL_DIRECT) {
    launch_swe_leaf_sources(g, c->sgeom, stage, dtd, dts, vprev, tprev, vors, divs, area, c->src, c->src2, mixed, st);
    launch_swe_direct(g, c->sgeom, c->cfg.precision, c->src, c->src2, v, c->partial, c->groups, st);
    return;
  }
  launch_swe_upward(g, c->sgeom, stage, dtd, dts, vprev, tprev, x, y, z, vors, divs, area, c->src, c->src2, mixed,
                    st);
  launch_swe_interactions(g, c->sgeom, c->cfg.precision, c->src, c->src2, c->tgt, st);
  if (c->L == 1) {
    cudaMemcpyAsync(v, c->tgt, sizeof(double) * 3 * c->P * c->q, cudaMemcpyDeviceToDevice, st);
    return;
  }
  launch_downward_fused(g, c->tgt, v, st);
}

// The work of one swe_back_rk4_step_2, enqueued on the stream.  Stage k
// (reference k1..k4 = s 0..3) evaluates the velocity, then (s < 3) the
// tendencies with modify_tendencies and unify_boundary_vals; the fourth
// stage's tendencies reach no result and are skipped.  The reference unifies
// the first-stage velocity after every stage (src/swe_time_step_2.cpp:843-845,
// 894-896, 940-942, 991-993); only the departure search and the returned
// velocity read it after the second stage, so the later three unifications
// run together before them.
void swe_enqueue_step(sbslpm_ctx* c, const double* x, const double* y, const double* z, const double* area,
                      double* vors, double* divs, double* height, double* vel_x, double* vel_y, double* vel_z,
                      double* tracers, const double* bv, const double* bd, const double* bh) {
  NvtxRange step_range("sbslpm swe step");
  (void)bv;  // modify_tendencies leaves the vorticity tendency alone (src/swe_time_step_2.cpp:778-782)
  cudaStream_t st = c->stream();
  const size_t ln = (size_t)c->A * c->q;
  const double dt = c->cfg.dt;
  const StepGeom& g = c->geom;
  const SweGeom& s = c->sgeom;
  double* v[4];
  for (int k = 0; k < 4; k++) v[k] = c->vbuf + (size_t)k * 3 * ln;
  double* T[3] = {c->tend, c->tend + 3 * ln, c->tend + 6 * ln};
  const double dtd[4] = {0.0, 0.5 * dt, 0.5 * dt, dt};
  const double dts[4] = {0.0, 0.5 * dt, 0.5 * dt, 0.5 * dt};
  for (int k = 0; k < 4; k++) {
    swe_velocity_eval(c, k, dtd[k], dts[k], k ? v[k - 1] : nullptr, k ? T[k - 1] : nullptr, x, y, z, area, vors,
                      divs, v[k]);
    if (k == 0) launch_unify(s, v[0], v[0] + ln, v[0] + 2 * ln, 1, st);
    if (k < 3) {
      launch_swe_tendency(g, s, x, y, z, v[k], vors, divs, height, nullptr, dts[k], k ? T[k - 1] : nullptr, bd, bh,
                          T[k], st);
      launch_unify(s, T[k], T[k] + ln, T[k] + 2 * ln, 1, st);
    }
  }
  launch_unify(s, v[0], v[0] + ln, v[0] + 2 * ln, 3, st);
  launch_swe_arrival(g, T[0], dt, vors, divs, height, c->avor, st);
  // departure points as the BVE step (swe_find_departure_points_2 is the same
  // functor), remap of the arrival vorticity without the planetary term
  StepGeom g0 = g;
  g0.omega = 0.0;
  const int nt = c->cfg.tracer_count;
  launch_depart_remap(g0, &c->tab, x, y, z, v[0], v[1], v[2], v[3], dt, c->dep, c->avor, tracers, nt, c->newvor,
                      c->newtr, 3, st);
  cudaMemcpyAsync(vors, c->newvor, sizeof(double) * ln, cudaMemcpyDeviceToDevice, st);
  if (nt > 0) cudaMemcpyAsync(tracers, c->newtr, sizeof(double) * ln * nt, cudaMemcpyDeviceToDevice, st);
  cudaMemcpyAsync(vel_x, v[0], sizeof(double) * ln, cudaMemcpyDeviceToDevice, st);
  cudaMemcpyAsync(vel_y, v[0] + ln, sizeof(double) * ln, cudaMemcpyDeviceToDevice, st);
  cudaMemcpyAsync(vel_z, v[0] + 2 * ln, sizeof(double) * ln, cudaMemcpyDeviceToDevice, st);
}

bool bad(const void* p) { return p == nullptr; }

}  // namespace
}  // namespace sbslpm

extern "C" {

sbslpm_status sbslpm_swe_step(sbslpm_ctx* c, const double* x, const double* y, const double* z, const double* area,
                              double* vors, double* divs, double* height, double* vel_x, double* vel_y,
                              double* vel_z, double* tracers, const double* bv, const double* bd, const double* bh,
                              double) {
  if (!c || bad(x) || bad(y) || bad(z) || bad(area) || bad(vors) || bad(divs) || bad(height) || bad(vel_x) ||
      bad(vel_y) || bad(vel_z) || bad(bv) || bad(bd) || bad(bh) || (c->cfg.tracer_count > 0 && bad(tracers)))
    return SBSLPM_ERR_ARG;
  if (any_on_host({x, y, z, area, vors, divs, height, vel_x, vel_y, vel_z, tracers, bv, bd, bh}))
    return set_last_error("device-pointer step given host memory"), SBSLPM_ERR_ARG;
  SB_TRY(shard_allows(c, false, "the shallow-water path"));
  SB_TRY(swe_setup(c));
  swe_enqueue_step(c, x, y, z, area, vors, divs, height, vel_x, vel_y, vel_z, tracers, bv, bd, bh);
  return finish(c);
}

sbslpm_status sbslpm_swe_run(sbslpm_ctx* c, const double* x, const double* y, const double* z, const double* area,
                             double* vors, double* divs, double* height, double* vel_x, double* vel_y, double* vel_z,
                             double* tracers, const double* bv, const double* bd, const double* bh, double,
                             int nsteps) {
  if (!c || bad(x) || bad(y) || bad(z) || bad(area) || bad(vors) || bad(divs) || bad(height) || bad(vel_x) ||
      bad(vel_y) || bad(vel_z) || bad(bv) || bad(bd) || bad(bh) || (c->cfg.tracer_count > 0 && bad(tracers)) ||
      nsteps < 0)
    return SBSLPM_ERR_ARG;
  if (any_on_host({x, y, z, area, vors, divs, height, vel_x, vel_y, vel_z, tracers, bv, bd, bh}))
    return set_last_error("device-pointer step given host memory"), SBSLPM_ERR_ARG;
  SB_TRY(shard_allows(c, false, "the shallow-water path"));
  SB_TRY(swe_setup(c));
  GraphKey key{{x, y, z, area, vors, divs, height, vel_x, vel_y, vel_z, tracers, bv, bd, bh}};
  if (!c->swe_graph || !(key == c->swe_graph_key)) {
    SB_TRY(capture_graph(c, &c->swe_graph, [&] {
      swe_enqueue_step(c, x, y, z, area, vors, divs, height, vel_x, vel_y, vel_z, tracers, bv, bd, bh);
      launch_unify(c->sgeom, vors, divs, height, 1, c->stream());
    }));
    c->swe_graph_key = key;
    c->swe_launches_per_step = c->launches_per_step;
  }
  cudaStream_t st = c->stream();
  for (int s = 0; s < nsteps; s++) {
    SB_CUDA(cudaGraphLaunch(c->swe_graph, st));
    launch_counter() += c->swe_launches_per_step;
  }
  return finish(c);
}

sbslpm_status sbslpm_swe_init(sbslpm_ctx* c, const double* x, const double* y, const double* z, const double* area,
                              const double* vors, const double* divs, const double* height, double* vel_x,
                              double* vel_y, double* vel_z, double* bv, double* bd, double* bh) {
  if (!c || bad(x) || bad(y) || bad(z) || bad(area) || bad(vors) || bad(divs) || bad(height) || bad(vel_x) ||
      bad(vel_y) || bad(vel_z) || bad(bv) || bad(bd) || bad(bh))
    return SBSLPM_ERR_ARG;
  SB_TRY(shard_allows(c, false, "the shallow-water path"));
  SB_TRY(swe_setup(c));
  cudaStream_t st = c->stream();
  const size_t ln = (size_t)c->A * c->q;
  double* v0 = c->vbuf;
  double* t0 = c->tend;
  swe_velocity_eval(c, 0, 0.0, 0.0, nullptr, nullptr, x, y, z, area, vors, divs, v0);
  launch_unify(c->sgeom, v0, v0 + ln, v0 + 2 * ln, 1, st);
  launch_swe_tendency(c->geom, c->sgeom, x, y, z, v0, vors, divs, height, nullptr, 0.0, nullptr, nullptr, nullptr, t0,
                      st);
  launch_unify(c->sgeom, t0, t0 + ln, t0 + 2 * ln, 1, st);
  double* outs[6] = {vel_x, vel_y, vel_z, bv, bd, bh};
  const double* ins[6] = {v0, v0 + ln, v0 + 2 * ln, t0, t0 + ln, t0 + 2 * ln};
  for (int k = 0; k < 6; k++) SB_CUDA(cudaMemcpyAsync(outs[k], ins[k], sizeof(double) * ln, cudaMemcpyDeviceToDevice, st));
  return finish(c);
}

sbslpm_status sbslpm_swe_tendencies(sbslpm_ctx* c, const double* x, const double* y, const double* z,
                                    const double* vel_x, const double* vel_y, const double* vel_z, const double* vors,
                                    const double* divs, const double* height, const double* surface, double* vt,
                                    double* dtn, double* ht) {
  if (!c || bad(x) || bad(y) || bad(z) || bad(vel_x) || bad(vel_y) || bad(vel_z) || bad(vors) || bad(divs) ||
      bad(height) || bad(surface) || bad(vt) || bad(dtn) || bad(ht))
    return SBSLPM_ERR_ARG;
  SB_TRY(swe_setup(c));
  cudaStream_t st = c->stream();
  const size_t ln = (size_t)c->A * c->q;
  double* v0 = c->vbuf;
  const double* vin[3] = {vel_x, vel_y, vel_z};
  for (int k = 0; k < 3; k++) SB_CUDA(cudaMemcpyAsync(v0 + k * ln, vin[k], sizeof(double) * ln, cudaMemcpyDeviceToDevice, st));
  launch_swe_tendency(c->geom, c->sgeom, x, y, z, v0, vors, divs, height, surface, 0.0, nullptr, nullptr, nullptr,
                      c->tend, st);
  double* outs[3] = {vt, dtn, ht};
  for (int k = 0; k < 3; k++)
    SB_CUDA(cudaMemcpyAsync(outs[k], c->tend + k * ln, sizeof(double) * ln, cudaMemcpyDeviceToDevice, st));
  return finish(c);
}

sbslpm_status sbslpm_unify_boundary_vals(sbslpm_ctx* c, double* vals) {
  if (!c || bad(vals)) return SBSLPM_ERR_ARG;
  SB_TRY(swe_setup(c));
  launch_unify(c->sgeom, vals, nullptr, nullptr, 1, c->stream());
  return finish(c);
}

sbslpm_status sbslpm_swe_vel_interactions(sbslpm_ctx* c, const double* dx, const double* dy, const double* dz,
                                          const double* sv, const double* sd, double* t1, double* t2, double* t3) {
  if (!c || bad(dx) || bad(dy) || bad(dz) || bad(sv) || bad(sd) || bad(t1) || bad(t2) || bad(t3))
    return SBSLPM_ERR_ARG;
  if (c->cfg.velocity != SBSLPM_VEL_FMM)
    return set_last_error("the interaction list exists only with FMM velocity"), SBSLPM_ERR_CONFIG;
  if (c->tree)
    return set_last_error("a treecode context has no spectral interaction list (sbslpm_swe_tree_velocity)"),
           SBSLPM_ERR_CONFIG;
  SB_TRY(shard_allows(c, false, "the shallow-water path"));
  SB_TRY(swe_setup(c));
  cudaStream_t st = c->stream();
  launch_swe_sources_from_disp(c->geom, c->sgeom, dx, dy, dz, sv, sd, c->src, c->src2,
                               c->cfg.precision == SBSLPM_MIXED, st);
  launch_swe_interactions(c->geom, c->sgeom, c->cfg.precision, c->src, c->src2, c->tgt, st);
  launch_add3(c->tgt, (long)c->P * c->q, t1, t2, t3, st);
  return finish(c);
}

sbslpm_status sbslpm_swe_tree_velocity(sbslpm_ctx* c, const double* dx, const double* dy, const double* dz,
                                       const double* w_vor, const double* w_div, double* u_x, double* u_y,
                                       double* u_z) {
  if (!c || bad(dx) || bad(dy) || bad(dz) || bad(w_vor) || bad(w_div) || bad(u_x) || bad(u_y) || bad(u_z))
    return SBSLPM_ERR_ARG;
  if (any_on_host({dx, dy, dz, w_vor, w_div, u_x, u_y, u_z}))
    return set_last_error("device pointers expected"), SBSLPM_ERR_ARG;
  if (!c->tree) return set_last_error("the context has no treecode (proxy_degree 0)"), SBSLPM_ERR_CONFIG;
  SB_TRY(shard_allows(c, false, "the shallow-water path"));
  SB_TRY(swe_setup(c));
  cudaStream_t st = c->stream();
  const size_t ln = (size_t)c->A * c->q;
  double* v = c->vbuf;
  swe_tree_velocity(c, 0, 0.0, 0.0, nullptr, nullptr, c->gx, c->gx + ln, c->gx + 2 * ln, nullptr, nullptr, nullptr,
                    dx, dy, dz, w_vor, w_div, v);
  double* outs[3] = {u_x, u_y, u_z};
  for (int k = 0; k < 3; k++) SB_CUDA(cudaMemcpyAsync(outs[k], v + k * ln, sizeof(double) * ln, cudaMemcpyDeviceToDevice, st));
  return finish(c);
}

sbslpm_status sbslpm_cubed_sphere_2d_to_1d(long n_leaves, int degree, const double* x, const double* y,
                                           const double* z, int* two_d_to_1d, int* counts, long* unique) {
  if (n_leaves <= 0 || degree < 0 || degree > kMaxDegree || !x || !y || !z || !two_d_to_1d || !counts || !unique)
    return SBSLPM_ERR_ARG;
  const int q = (degree + 1) * (degree + 1);
  std::vector<int> cnt;
  *unique = unique_points(n_leaves, q, x, y, z, two_d_to_1d, cnt);
  const long cap = n_leaves * (long)degree * degree + 2;
  if (*unique > cap) return set_last_error("more distinct points than leaf_count*degree^2 + 2"), SBSLPM_ERR_ARG;
  std::memcpy(counts, cnt.data(), sizeof(int) * cnt.size());
  return SBSLPM_OK;
}

}  // extern "C"
