// C ABI of the adjoint: one reverse step of bve_back_rk4_step
// (src/bve_time_step.cpp:311-419) and the stand-alone vector-Jacobian product
// of the Biot-Savart direct sum.
//
// The reverse step recomputes the forward step from its input vorticity (the
// per-step checkpoint): stage velocities v0..v3 and stage sources, then runs
// the departure/remap adjoint and the four velocity evaluations' adjoints in
// reverse stage order (stage s's sources depend on v_{s-1}).
#include <cuda_runtime.h>

#include <string>

#include <vector>

#include "adjoint.cuh"
#include "adjoint_tree.cuh"
#include "context_internal.hpp"

using namespace sbslpm;

namespace {

sbslpm_status adjoint_setup(sbslpm_ctx* c) {
  if (c->adj_vbar) return SBSLPM_OK;
  const size_t pn = (size_t)c->P * c->q, ln = (size_t)c->A * c->q;
  c->adj_groups = adjoint_groups((long)ln, (long)ln);
  if (!c->tree) SB_TRY(dalloc(&c->adj_src, 4 * pn));
  SB_TRY(dalloc(&c->adj_vbar, 4 * 3 * ln));
  SB_TRY(dalloc(&c->adj_q, ln));
  SB_TRY(dalloc(&c->adj_y, 3 * ln));
  SB_TRY(dalloc(&c->adj_part, (size_t)c->adj_groups * 4 * ln));
  SB_TRY(dalloc(&c->adj_w, ln));
  SB_TRY(dalloc(&c->adj_vel, 3 * ln));
  if (c->tree) {
    // transposed near and well-separated lists of the treecode
    TreeTables t;
    SB_TRY(build_tree_tables(c->L, c->d, c->panels, c->cfg.leaf_size, c->cfg.proxy_degree, t));
    TreeLists l;
    build_tree_lists(t, c->cfg.fmm_theta, l);
    auto transpose = [](const std::vector<int>& start, const std::vector<int>& src, int nsrc, int base,
                        std::vector<int>& tstart, std::vector<int>& ttgt) {
      const int nt = (int)start.size() - 1;
      tstart.assign(nsrc + 1, 0);
      for (int e = 0; e < start[nt]; e++) tstart[src[e] - base + 1]++;
      for (int i = 0; i < nsrc; i++) tstart[i + 1] += tstart[i];
      ttgt.assign(start[nt], 0);
      std::vector<int> fill(tstart.begin(), tstart.end() - 1);
      for (int tg = 0; tg < nt; tg++)
        for (int e = start[tg]; e < start[tg + 1]; e++) ttgt[fill[src[e] - base]++] = tg;
    };
    std::vector<int> nts, ntt, cts, ctt;
    transpose(l.ns, l.nsrc, t.Af, 0, nts, ntt);
    transpose(l.cs, l.csrc, t.Pf, 0, cts, ctt);
    SB_TRY(upload(&c->adj_near_ts, nts));
    SB_TRY(upload(&c->adj_near_tt, ntt));
    SB_TRY(upload(&c->adj_cc_ts, cts));
    SB_TRY(upload(&c->adj_cc_tt, ctt));
    SB_TRY(dalloc(&c->adj_tbar, (size_t)3 * t.Pf * t.qx));
    SB_TRY(dalloc(&c->adj_qbl, (size_t)t.Pf * t.qx));
  } else if (c->cfg.velocity == SBSLPM_VEL_FMM) {
    // the spectral interaction list transposed: target panels by source panel, in list order
    std::vector<int> ts(c->P + 1, 0), tt(c->list.size());
    for (const auto& e : c->list) ts[e.source_panel + 1]++;
    for (int p = 0; p < c->P; p++) ts[p + 1] += ts[p];
    std::vector<int> fill(ts.begin(), ts.end() - 1);
    for (const auto& e : c->list) tt[fill[e.source_panel]++] = e.target_panel;
    SB_TRY(upload(&c->adj_cc_ts, ts));
    SB_TRY(upload(&c->adj_cc_tt, tt));
    SB_TRY(dalloc(&c->adj_tbar, 3 * pn));
    SB_TRY(dalloc(&c->adj_qbl, pn));
    SB_TRY(dalloc(&c->adj_ynl, (size_t)3 * c->off * c->q));
  }
  return SBSLPM_OK;
}

bool bad(const void* p) { return p == nullptr; }

}  // namespace

extern "C" {

sbslpm_status sbslpm_bve_adjoint_step(sbslpm_ctx* c, const double* x, const double* y, const double* z,
                                      const double* area, const double* vors, const double* vors_bar_next,
                                      double* vors_bar) {
  if (!c || bad(x) || bad(y) || bad(z) || bad(area) || bad(vors) || bad(vors_bar_next) || bad(vors_bar))
    return SBSLPM_ERR_ARG;
  if (c->cfg.tracer_count != 0 || c->cfg.forcing != SBSLPM_FORCING_NONE)
    return set_last_error("the adjoint step needs a context without tracers or forcing"), SBSLPM_ERR_CONFIG;
  SB_TRY(shard_allows(c, false, "the adjoint step"));
  NvtxRange range("sbslpm bve adjoint step");
  SB_TRY(adjoint_setup(c));
  SB_TRY(near_autotune(c, x, y, z, area, vors));
  cudaStream_t st = c->stream();
  const size_t ln = (size_t)c->A * c->q, pn = (size_t)c->P * c->q, off = (size_t)c->off * c->q;
  const double dt = c->cfg.dt;
  // forward recompute from the checkpoint: stage velocities into vbuf
  SB_CUDA(cudaMemcpyAsync(c->adj_w, vors, sizeof(double) * ln, cudaMemcpyDeviceToDevice, st));
  enqueue_step(c, x, y, z, area, c->adj_w, c->adj_vel, c->adj_vel + ln, c->adj_vel + 2 * ln, nullptr);
  const double* v[4];
  for (int k = 0; k < 4; k++) v[k] = c->vbuf + (size_t)k * 3 * ln;
  const double h[4] = {0.0, 0.5 * dt, 0.5 * dt, dt};
  const bool spectral = !c->tree && c->cfg.velocity == SBSLPM_VEL_FMM;
  if (spectral)  // every panel's stage sources: displaced proxies and anterpolated strengths
    for (int s = 0; s < 4; s++)
      launch_upward_fused(c->geom, 0, s, h[s], s ? v[s - 1] : nullptr, x, y, z, vors, area, c->adj_src + s * pn,
                          false, st);
  else if (!c->tree)
    for (int s = 0; s < 4; s++)
      launch_leaf_sources(c->geom, s, h[s], s ? v[s - 1] : nullptr, x, y, z, vors, area, c->adj_src + s * pn, st);
  // reverse: departure search and remap, then the stages from the last
  double* vb[4];
  for (int k = 0; k < 4; k++) vb[k] = c->adj_vbar + (size_t)k * 3 * ln;
  SB_CUDA(cudaMemsetAsync(vors_bar, 0, sizeof(double) * ln, st));
  SB_CUDA(cudaMemsetAsync(c->adj_vbar, 0, sizeof(double) * 4 * 3 * ln, st));
  launch_depart_remap_adjoint(c->geom, c->tab, x, y, z, v[0], v[1], v[2], v[3], dt, vors, vors_bar_next, vors_bar,
                              vb[0], vb[1], vb[2], vb[3], st);
  const TreeAdjointLists tl{c->adj_near_ts, c->adj_near_tt, c->adj_cc_ts, c->adj_cc_tt};
  for (int s = 3; s >= 0; s--) {
    if (c->tree) {
      // this stage's particle sources, then the treecode's adjoint
      launch_bltc_sources(c->tgeom, c->fgeom, c->ftab, s, h[s], s ? v[s - 1] : nullptr, x, y, z, vors, area, c->psrc,
                          nullptr, c->fsrc, false, st);
      launch_tree_velocity_adjoint(c->tgeom, c->fgeom, c->ftab, tl, x, y, z, vb[s], c->psrc, c->adj_tbar, c->adj_qbl,
                                   c->adj_q, c->adj_y, c->cfg.precision == SBSLPM_MIXED, st);
    } else if (spectral) {
      launch_spectral_velocity_adjoint(c->geom, c->adj_cc_ts, c->adj_cc_tt, vb[s], c->adj_src + s * pn,
                                       c->adj_tbar, c->adj_qbl, c->adj_y, c->adj_ynl,
                                       c->cfg.precision == SBSLPM_MIXED, st);
      if (s > 0) launch_nonleaf_positions_adjoint(c->geom, h[s], v[s - 1], c->adj_ynl, vb[s - 1], st);
    } else if (c->cfg.precision == SBSLPM_MIXED) {
      launch_bs_vjp_leaves32(c->geom, x, y, z, vb[s], vb[s] + ln, vb[s] + 2 * ln, c->adj_src + s * pn + off,
                             c->adj_part, c->adj_groups, c->adj_q, c->adj_y, st);
    } else {
      launch_bs_vjp((long)ln, x, y, z, vb[s], vb[s] + ln, vb[s] + 2 * ln, (long)ln, c->adj_src + s * pn + off,
                    c->cfg.kernel_eps, c->adj_part, c->adj_groups, c->adj_q, c->adj_y, st);
    }
    launch_src_adjoint((long)ln, s, h[s], c->cfg.omega, s ? v[s - 1] : nullptr, x, y, z, area,
                       spectral ? c->adj_qbl + off : c->adj_q, c->adj_y, vors_bar, s ? vb[s - 1] : nullptr, st);
  }
  return finish(c);
}

sbslpm_status sbslpm_direct_sum_bve_vjp(long nt, const double* tx, const double* ty, const double* tz,
                                        const double* ubar_x, const double* ubar_y, const double* ubar_z, long ns,
                                        const double* sx, const double* sy, const double* sz, const double* strength,
                                        double eps, double* strength_bar, double* sx_bar, double* sy_bar,
                                        double* sz_bar, void* stream) {
  if (nt <= 0 || ns <= 0 || bad(tx) || bad(ty) || bad(tz) || bad(ubar_x) || bad(ubar_y) || bad(ubar_z) ||
      bad(sx) || bad(sy) || bad(sz) || bad(strength) || bad(strength_bar) || bad(sx_bar) || bad(sy_bar) ||
      bad(sz_bar) || !(eps >= 0))
    return SBSLPM_ERR_ARG;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int groups = adjoint_groups(nt, ns);
  double4* src = nullptr;
  double *part = nullptr, *ybar = nullptr;
  SB_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&src), sizeof(double4) * ns, st));
  SB_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&part), sizeof(double) * groups * 4 * ns, st));
  SB_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&ybar), sizeof(double) * 3 * ns, st));
  launch_pack_sources(ns, sx, sy, sz, strength, src, st);
  launch_bs_vjp(nt, tx, ty, tz, ubar_x, ubar_y, ubar_z, ns, src, eps, part, groups, strength_bar, ybar, st);
  SB_CUDA(cudaMemcpyAsync(sx_bar, ybar, sizeof(double) * ns, cudaMemcpyDeviceToDevice, st));
  SB_CUDA(cudaMemcpyAsync(sy_bar, ybar + ns, sizeof(double) * ns, cudaMemcpyDeviceToDevice, st));
  SB_CUDA(cudaMemcpyAsync(sz_bar, ybar + 2 * ns, sizeof(double) * ns, cudaMemcpyDeviceToDevice, st));
  cudaFreeAsync(src, st);
  cudaFreeAsync(part, st);
  cudaFreeAsync(ybar, st);
  SB_CUDA(cudaGetLastError());
  SB_CUDA(cudaStreamSynchronize(st));
  return SBSLPM_OK;
}

}  // extern "C"
