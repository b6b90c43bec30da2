// C ABI of the BVE hot path: context set-up (tree, interaction list and the
// static geometry precomputed on the host and uploaded once), the RK4 step
// orchestration on one CUDA stream, CUDA-graph replay of whole steps, and the
// piecewise entry points that mirror the reference's FMM functions.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "context_internal.hpp"
#include "geometry.cuh"

using namespace sbslpm;

namespace sbslpm {
namespace {
thread_local std::string g_last_error;
}
void set_last_error(const std::string& msg) { g_last_error = msg; }
}  // namespace sbslpm

namespace {

sbslpm_status validate(const sbslpm_config& c) {
  if (c.levels < 1 || c.levels > 12) return set_last_error("levels must be in 1..12"), SBSLPM_ERR_CONFIG;
  if (c.interp_degree < 0 || c.interp_degree > kMaxDegree)
    return set_last_error("interp_degree must be in 0..10"), SBSLPM_ERR_CONFIG;
  if (c.tracer_count < 0) return set_last_error("tracer_count must be >= 0"), SBSLPM_ERR_CONFIG;
  if (c.velocity != SBSLPM_VEL_FMM && c.velocity != SBSLPM_VEL_DIRECT)
    return set_last_error("velocity must be SBSLPM_VEL_FMM or SBSLPM_VEL_DIRECT"), SBSLPM_ERR_CONFIG;
  if (c.precision != SBSLPM_FP64 && c.precision != SBSLPM_MIXED)
    return set_last_error("precision must be SBSLPM_FP64 or SBSLPM_MIXED"), SBSLPM_ERR_CONFIG;
  if (c.proxy_degree < 0 || c.proxy_degree > kMaxDegree)
    return set_last_error("proxy_degree must be in 0..10"), SBSLPM_ERR_CONFIG;
  if (c.proxy_degree > 0 && c.velocity == SBSLPM_VEL_FMM) {
    const int qp = (c.interp_degree + 1) * (c.interp_degree + 1);
    if (c.leaf_size < qp || c.leaf_size > 512 * 1024)
      return set_last_error("leaf_size must hold at least one panel's points"), SBSLPM_ERR_CONFIG;
    long npl = qp;
    while (npl * 4 <= c.leaf_size) npl *= 4;
    if (npl > 512) return set_last_error("treecode leaves hold at most 512 particles"), SBSLPM_ERR_CONFIG;
  }
  if (!(c.kernel_eps >= 0) || !std::isfinite(c.dt) || !std::isfinite(c.omega) || !std::isfinite(c.g_over_a))
    return set_last_error("kernel_eps, dt and omega must be finite (kernel_eps >= 0)"), SBSLPM_ERR_CONFIG;
  if (c.forcing != SBSLPM_FORCING_NONE && c.forcing != SBSLPM_FORCING_SSW && c.forcing != SBSLPM_FORCING_SSW2)
    return set_last_error("forcing must be SBSLPM_FORCING_NONE, _SSW or _SSW2"), SBSLPM_ERR_CONFIG;
  return SBSLPM_OK;
}

// Host precomputation of everything that does not change during a run.

// The entry table of the mixed-precision kernels for q <= 32: per entry of a
// CSR list (start by target, src) the source panel and the offset of its
// centre from the target's centre, (float)((c_S - c_T) kPackScale), as float
// bits; the same double arithmetic and rounding as the direct-sum kernels
// apply per source leaf on the device.
std::vector<int4> entry_table(const std::vector<int>& start, const std::vector<int>& src,
                              const std::vector<double>& centre) {
  std::vector<int4> out(src.size());
  for (size_t t = 0; t + 1 < start.size(); t++)
    for (int e = start[t]; e < start[t + 1]; e++) {
      const size_t sp = (size_t)src[e];
      float b[3];
      for (int k = 0; k < 3; k++) b[k] = (float)((centre[4 * sp + k] - centre[4 * t + k]) * kPackScale);
      int bits[3];
      std::memcpy(bits, b, sizeof b);
      out[e] = make_int4(src[e], bits[0], bits[1], bits[2]);
    }
  return out;
}

sbslpm_status precompute(sbslpm_ctx* c) {
  const int q = c->q, P = c->P, off = c->off, d = c->d;
  std::vector<double> interp;
  build_interp(d, false, interp);

  bli_table(d, c->tab);
  // panel centres for the mixed-precision relative coordinates (the treecode's
  // shallow-water near field packs its particles by grid leaf as well)
  std::vector<double> centre((size_t)4 * P, 0.0);
  for (int p = 0; p < P; p++) {
    const sbslpm_panel& pp = c->panels[p];
    double xyz[3];
    xyz_from_xieta(kPi / 4.0 * 0.5 * (pp.min_xi + pp.max_xi), kPi / 4.0 * 0.5 * (pp.min_eta + pp.max_eta), pp.face,
                   xyz);
    for (int k = 0; k < 3; k++) centre[4 * (size_t)p + k] = xyz[k];
  }
  SB_TRY(upload(&c->centre, centre));
  if (c->tree) return SBSLPM_OK;  // the treecode has its own set-up

  // proxy positions, exactly as the reference's interaction kernel places them
  std::vector<double> px((size_t)3 * P * q);
  const size_t pn = (size_t)P * q;
  for (int p = 0; p < P; p++)
    for (int j = 0; j < q; j++) {
      double xyz[3];
      proxy_point(c->panels[p], interp.data(), j, xyz);
      px[(size_t)p * q + j] = xyz[0];
      px[pn + (size_t)p * q + j] = xyz[1];
      px[2 * pn + (size_t)p * q + j] = xyz[2];
    }
  SB_TRY(upload(&c->px, px));

  if (c->cfg.velocity != SBSLPM_VEL_FMM) return SBSLPM_OK;

  // displacement interpolation at non-leaf proxies (bve_disp_interp,
  // src/bve_time_step.cpp:131-159): located leaf row and BLI basis
  std::vector<int> il_row((size_t)off * q);
  std::vector<double> il_basis((size_t)off * q * q);
  unsigned err = 0;
  for (int i = 0; i < off; i++) {
    const sbslpm_panel& p = c->panels[i];
    double xo = kPi / 4 * 0.5 * (p.max_xi + p.min_xi), xs = kPi / 4 * 0.5 * (p.max_xi - p.min_xi);
    double eo = kPi / 4 * 0.5 * (p.max_eta + p.min_eta), es = kPi / 4 * 0.5 * (p.max_eta - p.min_eta);
    for (int j = 0; j < q; j++) {
      double xi = interp[4 * j] * xs + xo, eta = interp[4 * j + 1] * es + eo, xyz[3], lxi, leta;
      xyz_from_xieta(xi, eta, p.face, xyz);
      Bounds b;
      int leaf = locate_leaf(xyz[0], xyz[1], xyz[2], c->L, lxi, leta, b, err);
      il_row[(size_t)i * q + j] = leaf - off;
      double basis[(kMaxDegree + 1) * (kMaxDegree + 1)];
      host_bli(basis, xi, eta, kPi / 4.0 * b.min_xi, kPi / 4.0 * b.max_xi, kPi / 4.0 * b.min_eta,
               kPi / 4.0 * b.max_eta, d, err);
      for (int m = 0; m < q; m++) il_basis[(size_t)m * off * q + (size_t)i * q + j] = basis[m];
    }
  }
  if (err) {
    set_last_error("a non-leaf proxy point fell outside its located leaf (the reference aborts here too)");
    return SBSLPM_ERR_OUT_OF_PANEL;
  }
  SB_TRY(upload(&c->il_row, il_row));
  SB_TRY(upload(&c->il_basis, il_basis));

  // child-in-parent BLI bases (child_to_parent / parent_to_child_3,
  // src/fmm_funcs_impl.hpp:47-70, 138-171), the same for every parent of the
  // uniform quadtree
  if (c->L > 1) {
    std::vector<double> c1d;
    child_basis_1d(c->panels, c->tab, d, c1d, err);
    SB_TRY(upload(&c->child_mat, c1d));
  }

  // interaction list grouped by target panel, list order kept within a target
  std::vector<int> start(P + 1, 0), srcs(c->list.size());
  for (const auto& e : c->list) start[e.target_panel + 1]++;
  for (int p = 0; p < P; p++) start[p + 1] += start[p];
  std::vector<int> fill(start.begin(), start.end() - 1);
  for (const auto& e : c->list) srcs[fill[e.target_panel]++] = e.source_panel;
  SB_TRY(upload(&c->tgt_start, start));
  SB_TRY(upload(&c->src_panel, srcs));
  if (c->cfg.precision == SBSLPM_MIXED && q <= 32) SB_TRY(upload(&c->entry32, entry_table(start, srcs, centre)));
  return SBSLPM_OK;
}

// Treecode set-up: the quadtree truncated so that a leaf holds npl <=
// leaf_size particles, degree-n proxies on every tree panel, the canonical
// leaf-box basis of the particle grid, and the near / well-separated lists.
sbslpm_status precompute_tree(sbslpm_ctx* c) {
  const int qp = c->q;
  TreeTables t;
  SB_TRY(build_tree_tables(c->L, c->d, c->panels, c->cfg.leaf_size, c->cfg.proxy_degree, t));
  c->tree = true;
  c->n = t.n;
  c->qx = t.qx;
  c->npl = t.npl;
  c->Lf = t.Lf;
  c->Pf = t.Pf;
  c->Af = t.Af;
  c->fpanels = t.fpanels;
  c->ftab = t.ftab;
  const size_t pn = (size_t)t.Pf * t.qx;
  const std::vector<double>& fpx = t.fpx;
  SB_TRY(upload(&c->fpx, t.fpx));
  SB_TRY(upload(&c->fcentre, t.centre));
  SB_TRY(upload(&c->fbounds, t.bounds));
  SB_TRY(upload(&c->fface, t.face));
  if (!t.c1d.empty()) SB_TRY(upload(&c->fchild, t.c1d));
  SB_TRY(upload(&c->flx, t.lx));
  SB_TRY(upload(&c->fly, t.ly));

  // the traversal of the tree on the GPU (the same list, in the same order, as on the host)
  std::vector<TreeLists> lv;
  SB_TRY(device_tree_lists(t, std::vector<double>{c->cfg.fmm_theta}, lv, nullptr));
  TreeLists& l = lv[0];
  c->n_near = l.ns.back();
  c->n_cc = l.cs.back();
  c->list = l.list;
  c->h_ns = l.ns;
  c->h_cs = l.cs;
  c->h_csrc = l.csrc;
  c->h_fcentre = t.centre;
  c->near_expanded = c->cfg.precision == SBSLPM_MIXED && near_expanded_ok(t, l, c->cfg.kernel_eps);
  SB_TRY(upload(&c->near_start, l.ns));
  SB_TRY(upload(&c->near_src, l.nsrc));
  SB_TRY(install_cc_lists(c, l.cs, l.csrc));
  if (c->cfg.precision == SBSLPM_MIXED && t.npl == kMutualLeaf && c->n_near > 0) {
    std::vector<int4> units;
    build_mutual_units(l.ns, l.nsrc, units);
    c->n_mutual = (int)units.size();
    SB_TRY(upload(&c->mutual_units, units));
    SB_TRY(dalloc(&c->near_slot, (size_t)c->n_near * 3 * kMutualLeaf));
  }
  if (c->n_cc > 0 && cc_chunk_supported(t.qx)) {
    SB_TRY(dalloc(&c->cc_partial, (size_t)c->n_cc * 3 * t.qx));
  } else {
    c->cc_tuned = true;  // k_interact_wide / k_interact32 over whole target panels
  }

  // workspace; proxy positions are fixed, strengths are written every stage
  const size_t N = (size_t)c->A * qp;
  {
    std::vector<double> interp_p, g(3 * N), area(N);
    build_interp(c->d, false, interp_p);
    build_points(c->L, c->d, c->panels, interp_p.data(), g.data(), g.data() + N, g.data() + 2 * N, area.data());
    SB_TRY(upload(&c->gx, g));
  }
  SB_TRY(dalloc(&c->fsrc, pn));
  std::vector<double4> init(pn);
  for (size_t i = 0; i < pn; i++) init[i] = make_double4(fpx[i], fpx[pn + i], fpx[2 * pn + i], 0.0);
  SB_CUDA(cudaMemcpy(c->fsrc, init.data(), sizeof(double4) * pn, cudaMemcpyHostToDevice));
  SB_TRY(dalloc(&c->ftgt, 3 * pn));
  SB_TRY(dalloc(&c->psrc, N));
  SB_TRY(dalloc(&c->near, (size_t)4 * 3 * N));
  if (c->cfg.precision == SBSLPM_MIXED) {
    SB_TRY(dalloc(&c->fsrcf, pn));
    SB_TRY(dalloc(&c->psrcf, N));
    if (c->cc_partial) SB_TRY(dalloc(&c->fsrcp, (size_t)t.Pf * 2 * ((t.qx + 1) / 2)));
  }
  return SBSLPM_OK;
}

sbslpm_status allocate_workspace(sbslpm_ctx* c) {
  const size_t pn = (size_t)c->P * c->q, ln = (size_t)c->A * c->q;
  if (!c->tree) {
    SB_TRY(dalloc(&c->src, pn));
    if (c->cfg.precision == SBSLPM_MIXED) SB_TRY(dalloc(&c->srcf, pn));
    SB_TRY(dalloc(&c->tgt, 3 * pn));
  }
  SB_TRY(dalloc(&c->vbuf, 4 * 3 * ln));
  SB_TRY(dalloc(&c->dep, 3 * ln));
  SB_TRY(dalloc(&c->newvor, ln));
  if (c->cfg.tracer_count > 0) SB_TRY(dalloc(&c->newtr, ln * c->cfg.tracer_count));
  if (c->cfg.velocity == SBSLPM_VEL_DIRECT) {
    long g = (148L * 64) / c->A;
    c->groups = (int)(g < 1 ? 1 : (g > 64 ? 64 : g));
    SB_TRY(dalloc(&c->partial, (size_t)c->groups * 3 * ln));
  }
  SB_TRY(dalloc(&c->err, 1));
  SB_CUDA(cudaMemset(c->err, 0, sizeof(unsigned)));
  SB_CUDA(cudaMallocHost(reinterpret_cast<void**>(&c->h_err), sizeof(unsigned)));
  return SBSLPM_OK;
}

void fill_geom(sbslpm_ctx* c) {
  StepGeom& g = c->geom;
  g.levels = c->L;
  g.degree = c->d;
  g.q = c->q;
  g.panels = c->P;
  g.leaves = c->A;
  g.offset = c->off;
  g.eps = c->cfg.kernel_eps;
  g.omega = c->cfg.omega;
  g.px = c->px;
  g.tgt_start = c->tgt_start;
  g.src_panel = c->src_panel;
  g.il_row = c->il_row;
  g.il_basis = c->il_basis;
  g.child_1d = c->child_mat;
  g.pd_centre = c->centre;
  g.srcf = c->srcf;
  g.entry = c->entry32;
  g.err = c->err;
  if (c->tree) {
    StepGeom& f = c->fgeom;
    f.levels = c->Lf;
    f.degree = c->n;
    f.q = c->qx;
    f.panels = c->Pf;
    f.leaves = c->Af;
    f.offset = c->Pf - c->Af;
    f.eps = c->cfg.kernel_eps;
    f.omega = c->cfg.omega;
    f.px = c->fpx;
    f.tgt_start = c->cc_start;
    f.src_panel = c->cc_src;
    f.child_1d = c->fchild;
    f.pd_centre = c->fcentre;
    f.srcf = c->fsrcf;
    f.entry = c->fentry32;
    f.err = c->err;
    TreeGeom& t = c->tgeom;
    t.n = c->n;
    t.npl = c->npl;
    t.N = (long)c->A * c->q;
    t.eps = c->cfg.kernel_eps;
    t.omega = c->cfg.omega;
    t.lx = c->flx;
    t.ly = c->fly;
    t.fbounds = c->fbounds;
    t.fface = c->fface;
    t.near_start = c->near_start;
    t.near_src = c->near_src;
  }
}

}  // namespace

namespace sbslpm {

// Uploads a well-separated CSR of the treecode (by target tree panel) and what
// is derived from it: the entry table (mixed precision, q <= 32) and the lists
// of chunks of 1..4 entries; the arrays of an earlier list are released.
sbslpm_status install_cc_lists(sbslpm_ctx* c, const std::vector<int>& cs, const std::vector<int>& csrc) {
  auto drop = [](auto*& p) {
    if (p) cudaFree(p);
    p = nullptr;
  };
  drop(c->cc_start);
  drop(c->cc_src);
  drop(c->fentry32);
  for (int k = 0; k < 4; k++) {
    drop(c->cc_chunks[k]);
    drop(c->cc_cstart[k]);
    c->cc_nchunks[k] = 0;
  }
  SB_TRY(upload(&c->cc_start, cs));
  SB_TRY(upload(&c->cc_src, csrc));
  if (c->cfg.precision == SBSLPM_MIXED && c->qx <= 32)
    SB_TRY(upload(&c->fentry32, entry_table(cs, csrc, c->h_fcentre)));
  if (c->n_cc > 0 && cc_chunk_supported(c->qx)) {
    for (int k = 0; k < 4; k++) {
      std::vector<int4> chunks;
      std::vector<int> cstart;
      build_cc_chunks(cs, k + 1, chunks, cstart);
      c->cc_nchunks[k] = (int)chunks.size();
      SB_TRY(upload(&c->cc_chunks[k], chunks));
      SB_TRY(upload(&c->cc_cstart[k], cstart));
    }
  }
  c->fgeom.tgt_start = c->cc_start;
  c->fgeom.src_panel = c->cc_src;
  c->fgeom.entry = c->fentry32;
  return SBSLPM_OK;
}

void launch_tree_cc(sbslpm_ctx* c, cudaStream_t st) {
  if (c->cc_partial && c->cc_slots > 0) {
    const int k = c->cc_len - 1;
    if (c->cc_tpt > 0) launch_cc_pair_sources(c->fsrcf, c->qx, c->Pf, c->fsrcp, st);
    launch_cc_chunks(c->fgeom, c->cfg.precision, c->cc_slots, c->cc_chunks[k], c->cc_nchunks[k], c->cc_cstart[k],
                     c->fsrc, c->cc_partial, c->ftgt, st, c->cc_tpt, c->fsrcp);
  } else {
    launch_interactions_only(c->fgeom, c->cfg.precision, c->fsrc, c->ftgt, st);
  }
}

// One velocity evaluation (one RK4 stage) into v (contiguous [3][leaves*q]).
void velocity_eval(sbslpm_ctx* c, int stage, double dt_s, const double* vprev, const double* x, const double* y,
                   const double* z, const double* area, const double* vors, double* v) {
  cudaStream_t st = c->stream();
  const StepGeom& g = c->geom;
  if (c->cfg.velocity == SBSLPM_VEL_DIRECT) {
    launch_leaf_sources(g, stage, dt_s, vprev, x, y, z, vors, area, c->src, st);
    launch_direct_leaves(g, c->cfg.precision, c->src, v, c->partial, c->groups, st);
    return;
  }
  const bool mixed = c->cfg.precision == SBSLPM_MIXED;
  if (c->tree) {
    const StepGeom& fg = c->fgeom;
    launch_bltc_sources(c->tgeom, fg, c->ftab, stage, dt_s, vprev, x, y, z, vors, area, c->psrc, c->psrcf, c->fsrc,
                        mixed, st);
    // the tree passes (proxy sources up, well-separated pairs, proxy targets
    // down) depend only on the leaf proxies, the near field only on the
    // particle sources: the tree runs on the auxiliary stream beside it
    cudaStream_t tree_st = c->aux_stream ? c->aux_stream : st;
    if (c->aux_stream) {
      cudaEventRecord(c->ev_fork, st);
      cudaStreamWaitEvent(tree_st, c->ev_fork, 0);
    }
    launch_upward_fused(fg, 2, 0, 0.0, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, c->fsrc, mixed, tree_st);
    launch_tree_cc(c, tree_st);
    launch_downward_fused(fg, c->ftgt, nullptr, tree_st);
    if (c->aux_stream) cudaEventRecord(c->ev_join, tree_st);
    int splits = c->near_splits;
    if (stage == 0 && c->near_mutual) {  // sources on the grid: each leaf pair once for both directions
      launch_bltc_near_mutual(c->tgeom, fg, c->mutual_units, c->n_mutual, c->psrcf, c->near_slot, x, y, z, c->near,
                              st);
      splits = 1;
    } else {
      launch_bltc_near_batch(c->self, 1, owned_leaves(c), c->npl, c->cfg.kernel_eps, c->cfg.precision, x, y, z, c->psrc,
                             c->psrcf, c->near, c->near_splits, c->near_nt, c->near_tpt, c->near_expanded, st);
    }
    if (c->aux_stream) cudaStreamWaitEvent(st, c->ev_join, 0);
    launch_bltc_to_particles(c->tgeom, fg, c->ftgt, c->near, splits, v, st);
    return;
  }
  launch_upward_fused(g, 0, stage, dt_s, vprev, x, y, z, vors, area, c->src, mixed, st);
  launch_interactions_only(g, c->cfg.precision, c->src, c->tgt, st);
  if (c->L == 1) {
    cudaMemcpyAsync(v, c->tgt, sizeof(double) * 3 * c->P * c->q, cudaMemcpyDeviceToDevice, st);
    return;
  }
  launch_downward_fused(g, c->tgt, v, st);
}

// The work of one bve_back_rk4_step (src/bve_time_step.cpp:311-419), enqueued on the stream.
// vel_x == nullptr: the stage-0 velocity stays in vbuf (its first 3 x
// leaves*q values); stage0, when given, is recorded once it is complete.
void enqueue_step(sbslpm_ctx* c, const double* x, const double* y, const double* z, const double* area, double* vors,
                  double* vel_x, double* vel_y, double* vel_z, double* tracers, cudaEvent_t stage0) {
  cudaStream_t st = c->stream();
  const size_t ln = (size_t)c->A * c->q;
  const double dt = c->cfg.dt;
  double* v[4];
  for (int k = 0; k < 4; k++) v[k] = c->vbuf + (size_t)k * 3 * ln;
  const double stage_dt[4] = {0.0, 0.5 * dt, 0.5 * dt, dt};
  // bve_forcing at the step's time, the same for all four stages (src/bve_time_step.cpp:323-395)
  NvtxRange step_range("sbslpm bve step");
  if (c->force) launch_ssw_forcing(c->A, c->q, c->cfg.forcing, c->cfg.omega, c->d_time, x, y, z, c->force, st);
  static const char* const stage_name[4] = {"sbslpm stage 0 velocity", "sbslpm stage 1 velocity",
                                            "sbslpm stage 2 velocity", "sbslpm stage 3 velocity"};
  for (int s = 0; s < 4; s++) {
    {
      NvtxRange r(stage_name[s]);
      velocity_eval(c, s, stage_dt[s], s ? v[s - 1] : nullptr, x, y, z, area, vors, v[s]);
    }
    if (c->nccl_comm) {
      NvtxRange r("sbslpm stage velocity all-gather");
      shard_exchange(c, v[s]);  // every rank's slice into every rank's copy (sharded contexts)
    }
    if (s == 0 && stage0) cudaEventRecord(stage0, st);
  }
  if (c->force) launch_time_advance(c->d_time, dt, st);
  const int T = c->cfg.tracer_count;
  NvtxRange remap_range("sbslpm departure + remap");
  launch_depart_remap(c->geom, &c->tab, x, y, z, v[0], v[1], v[2], v[3], dt, c->dep, vors, tracers, T, c->newvor,
                      c->newtr, 3, st);
  cudaMemcpyAsync(vors, c->newvor, sizeof(double) * ln, cudaMemcpyDeviceToDevice, st);
  if (T > 0) cudaMemcpyAsync(tracers, c->newtr, sizeof(double) * ln * T, cudaMemcpyDeviceToDevice, st);
  if (vel_x) {
    cudaMemcpyAsync(vel_x, v[0], sizeof(double) * ln, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(vel_y, v[0] + ln, sizeof(double) * ln, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(vel_z, v[0] + 2 * ln, sizeof(double) * ln, cudaMemcpyDeviceToDevice, st);
  }
}

// Waits for the stream, then turns launch errors and the device error word
// into a status.
sbslpm_status finish(sbslpm_ctx* c) {
  cudaStream_t st = c->stream();
  SB_CUDA(cudaGetLastError());
  SB_CUDA(cudaMemcpyAsync(c->h_err, c->err, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
  SB_CUDA(cudaStreamSynchronize(st));
  unsigned e = *c->h_err;
  if (c->shard_status != SBSLPM_OK) {
    const sbslpm_status s = c->shard_status;
    c->shard_status = SBSLPM_OK;
    return set_last_error(c->shard_error), s;
  }
  if (e) {
    SB_CUDA(cudaMemsetAsync(c->err, 0, sizeof(unsigned), st));
    SB_CUDA(cudaStreamSynchronize(st));
    if (e & kErrTimeout)
      return set_last_error("a well-separated kernel's bounded copy wait ran out"), SBSLPM_ERR_TIMEOUT;
    if (e & kErrNonFinite) return set_last_error("non-finite point in a location step"), SBSLPM_ERR_NONFINITE;
    return set_last_error("interpolation point outside its panel"), SBSLPM_ERR_OUT_OF_PANEL;
  }
  return SBSLPM_OK;
}

// Captures body() once on the context's own stream (the legacy default stream
// cannot be captured), after the current stream's earlier work, into *graph.
// Kernels enqueued by body() are not counted as launched; the count per
// replay is returned through c->launches_per_step.
void drop_step_graphs(sbslpm_ctx* c) {
  if (c->graph) cudaGraphExecDestroy(c->graph);
  if (c->host_graph) cudaGraphExecDestroy(c->host_graph);
  c->graph = nullptr;
  c->host_graph = nullptr;
}

sbslpm_status capture_graph(sbslpm_ctx* c, cudaGraphExec_t* graph, const std::function<void()>& body) {
  if (*graph) {
    cudaGraphExecDestroy(*graph);
    *graph = nullptr;
  }
  cudaStream_t st = c->stream(), cap = c->own_stream;
  if (st != cap) {
    cudaEvent_t ev;
    SB_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    SB_CUDA(cudaEventRecord(ev, st));
    SB_CUDA(cudaStreamWaitEvent(cap, ev, 0));
    cudaEventDestroy(ev);
  }
  const bool saved_set = c->user_stream_set;
  c->user_stream_set = false;  // enqueue on the capturing stream
  const long before = launch_counter();
  cudaGraph_t g;
  SB_CUDA(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
  body();
  cudaError_t ce = cudaStreamEndCapture(cap, &g);
  c->user_stream_set = saved_set;
  c->launches_per_step = launch_counter() - before;
  launch_counter() = before;
  SB_CUDA(ce);
  // kernels captured from the higher-priority auxiliary stream keep that
  // priority on replay (otherwise a graph runs every node at its launch
  // stream's priority and the tree passes queue behind the near field)
  SB_CUDA(cudaGraphInstantiateWithFlags(graph, g, cudaGraphInstantiateFlagUseNodePriority));
  cudaGraphDestroy(g);
  return SBSLPM_OK;
}

// Times every well-separated launch shape (the whole-panel kernel, and blocks
// of 1..8 chunk slots over chunks of 1..4 list entries) on the current proxy
// sources and keeps the fastest.
sbslpm_status cc_autotune(sbslpm_ctx* c) {
  cudaStream_t st = c->stream();
  cudaEvent_t e0, e1;
  SB_CUDA(cudaEventCreate(&e0));
  SB_CUDA(cudaEventCreate(&e1));
  double best = 1e30;
  int cand = 0;
  const int keep_slots = c->cc_slots, keep_len = c->cc_len, keep_tpt = c->cc_tpt;
  int best_slots = keep_slots, best_len = keep_len, best_tpt = keep_tpt;
  // kernel form: 0 staged in shared memory, 1 | 2 barrier-free, 3 bulk copies, 4 warp per chunk (mixed precision)
  const int max_tpt = c->cfg.precision == SBSLPM_MIXED && c->fsrcp ? kCcWarpForm : 0;
  for (int tpt = 0; tpt <= max_tpt; tpt++)
  for (int sl = tpt > 0 ? 1 : 0; sl <= 8; sl++) {  // chunk slots (warps) per block; 0: one block per target panel
    const bool direct = tpt == 1 || tpt == 2;
    const bool shape_ok = tpt == kCcWarpForm ? cc_warp_shape_ok(c->qx, sl)
                          : direct          ? cc_direct_shape_ok(c->qx, sl, tpt)
                                            : cc_chunk_shape_ok(c->qx, sl);
    if (sl > 0 && !shape_ok) continue;
    for (int len = sl > 0 ? 1 : 0; len <= (sl > 0 ? 4 : 0); len++) {
      c->cc_slots = sl;
      c->cc_len = len;
      c->cc_tpt = tpt;
      launch_tree_cc(c, st);
      SB_CUDA(cudaEventRecord(e0, st));
      for (int r = 0; r < 5; r++) launch_tree_cc(c, st);
      SB_CUDA(cudaEventRecord(e1, st));
      SB_CUDA(cudaEventSynchronize(e1));
      float ms = 0;
      SB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      cand++;
      if (ms / 5 < best) {
        best = ms / 5;
        best_slots = sl;
        best_len = len;
        best_tpt = tpt;
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  c->cc_slots = best_slots;
  c->cc_len = best_len;
  c->cc_tpt = best_tpt;
  c->cc_candidates = cand;
  c->cc_tuned_ms = best;
  c->cc_tuned = true;
  return SBSLPM_OK;
}

// Times every near-field launch shape (threads x targets per thread covering a
// treecode leaf, 1..4 source-list splits) on the stage-0 sources and keeps the
// fastest.  Runs once per context, before the first step, outside any capture.
sbslpm_status near_autotune(sbslpm_ctx* c, const double* x, const double* y, const double* z, const double* area,
                            const double* vors) {
  if (!c->tree || (c->near_tuned && c->cc_tuned)) return SBSLPM_OK;
  NvtxRange r("sbslpm launch-shape timing");
  cudaStream_t st = c->stream();
  const int prec = c->cfg.precision;
  launch_bltc_sources(c->tgeom, c->fgeom, c->ftab, 0, 0.0, nullptr, x, y, z, vors, area, c->psrc, c->psrcf, c->fsrc,
                      prec == SBSLPM_MIXED, st);
  if (!c->cc_tuned) {
    launch_upward_fused(c->fgeom, 2, 0, 0.0, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, c->fsrc,
                        prec == SBSLPM_MIXED, st);
    SB_TRY(cc_autotune(c));
  }
  if (c->near_tuned) return finish(c);
  const int shapes[][2] = {{64, 4}, {128, 2}, {256, 1}, {256, 2}, {64, 2}, {64, 1}, {128, 1}};
  cudaEvent_t e0, e1;
  SB_CUDA(cudaEventCreate(&e0));
  SB_CUDA(cudaEventCreate(&e1));
  double best = 1e30;
  int cand = 0;
  for (const auto& sh : shapes) {
    if (sh[0] * sh[1] < c->npl || sh[0] * sh[1] >= 4 * c->npl) continue;
    for (int sp = 1; sp <= 4; sp++) {
      auto run = [&] {
        launch_bltc_near_batch(c->self, 1, owned_leaves(c), c->npl, c->cfg.kernel_eps, prec, x, y, z, c->psrc,
                               c->psrcf, c->near, sp, sh[0], sh[1], c->near_expanded, st);
      };
      run();
      SB_CUDA(cudaEventRecord(e0, st));
      for (int r = 0; r < 5; r++) run();
      SB_CUDA(cudaEventRecord(e1, st));
      SB_CUDA(cudaEventSynchronize(e1));
      float ms = 0;
      SB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      cand++;
      if (ms / 5 < best) {
        best = ms / 5;
        c->near_nt = sh[0];
        c->near_tpt = sh[1];
        c->near_splits = sp;
      }
    }
  }
  // the first stage's two-sided kernel, where it applies: kept for stage 0
  // if it beats the chosen shape on these (stage-0) sources
  c->near_mutual = false;
  if (c->n_mutual > 0 && c->shard_n == 1) {  // a unit writes both of its leaves: unsharded contexts only
    auto run = [&] {
      launch_bltc_near_mutual(c->tgeom, c->fgeom, c->mutual_units, c->n_mutual, c->psrcf, c->near_slot, x, y, z,
                              c->near, st);
    };
    run();
    SB_CUDA(cudaEventRecord(e0, st));
    for (int r = 0; r < 5; r++) run();
    SB_CUDA(cudaEventRecord(e1, st));
    SB_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    SB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    c->near_mutual_ms = ms / 5;
    c->near_mutual = c->near_mutual_ms < best;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  c->near_candidates = cand;
  c->near_tuned_ms = best;
  c->near_tuned = true;
  return finish(c);
}

}  // namespace sbslpm

namespace {

bool bad(const void* p) { return p == nullptr; }

}  // namespace

// ---------------------------------------------------------------------------

extern "C" {

sbslpm_status sbslpm_config_default(sbslpm_config* cfg) {
  if (!cfg) return SBSLPM_ERR_ARG;
  *cfg = sbslpm_config{};
  cfg->levels = 5;
  cfg->interp_degree = 3;
  cfg->fmm_theta = 0.7;
  cfg->kernel_eps = 1e-4;
  cfg->omega = 0.00007272205216643039;  // RunConfig::omega default, src/run_config.hpp:31
  cfg->dt = 1.0;
  cfg->tracer_count = 0;
  cfg->velocity = SBSLPM_VEL_FMM;
  cfg->precision = SBSLPM_FP64;
  cfg->exact_cc = 0;
  cfg->g_over_a = 9.81 / 6371000.0;  // src/swe_time_step_2_impl.hpp:103
  return SBSLPM_OK;
}

sbslpm_status sbslpm_read_run_config(const char* path, sbslpm_config* cfg) {
  if (!path || !cfg) return SBSLPM_ERR_ARG;
  std::string msg;
  if (!read_namelist(path, cfg, msg)) {
    set_last_error(msg);
    return SBSLPM_ERR_CONFIG;
  }
  return SBSLPM_OK;  // combinations are validated by sbslpm_create
}

const char* sbslpm_status_string(sbslpm_status s) {
  switch (s) {
    case SBSLPM_OK: return "ok";
    case SBSLPM_ERR_CONFIG: return "invalid configuration";
    case SBSLPM_ERR_CUDA: return "CUDA error";
    case SBSLPM_ERR_OUT_OF_PANEL: return "interpolation point outside its panel";
    case SBSLPM_ERR_NONFINITE: return "non-finite value";
    case SBSLPM_ERR_ARG: return "invalid argument";
    case SBSLPM_ERR_NO_DEVICE: return "no CUDA device";
    case SBSLPM_ERR_TIMEOUT: return "device wait timed out";
  }
  return "unknown status";
}

const char* sbslpm_last_error(void) { return g_last_error.c_str(); }

int sbslpm_panel_count(int levels) { return 2 * ((1 << (2 * levels)) - 1); }
int sbslpm_leaf_count(int levels) { return 6 * (1 << (2 * (levels - 1))); }

sbslpm_status sbslpm_cubed_sphere_panels_init(int levels, sbslpm_panel* out) {
  if (!out || levels < 1 || levels > 12) return SBSLPM_ERR_ARG;
  std::vector<sbslpm_panel> p;
  build_panels(levels, p);
  std::memcpy(out, p.data(), sizeof(sbslpm_panel) * p.size());
  return SBSLPM_OK;
}

sbslpm_status sbslpm_interp_init(int degree, int exact_cc, double* interp) {
  if (!interp || degree < 0 || degree > kMaxDegree) return SBSLPM_ERR_ARG;
  std::vector<double> v;
  build_interp(degree, exact_cc != 0, v);
  std::memcpy(interp, v.data(), sizeof(double) * v.size());
  return SBSLPM_OK;
}

sbslpm_status sbslpm_cube_sphere_spec_points(int levels, int degree, const sbslpm_panel* panels, const double* interp,
                                             double* x, double* y, double* z, double* area) {
  if (!panels || !interp || !x || !y || !z || !area) return SBSLPM_ERR_ARG;
  std::vector<sbslpm_panel> p(panels, panels + sbslpm_panel_count(levels));
  build_points(levels, degree, p, interp, x, y, z, area);
  return SBSLPM_OK;
}

sbslpm_status sbslpm_dual_tree_traversal(int levels, const sbslpm_panel* panels, double theta,
                                         sbslpm_interact_pair* out, long cap, long* count) {
  if (!panels || !count) return SBSLPM_ERR_ARG;
  std::vector<sbslpm_panel> p(panels, panels + sbslpm_panel_count(levels));
  std::vector<sbslpm_interact_pair> list;
  build_interactions(levels, p, theta, list);
  *count = (long)list.size();
  if (out) std::memcpy(out, list.data(), sizeof(sbslpm_interact_pair) * std::min<size_t>(cap, list.size()));
  return SBSLPM_OK;
}

sbslpm_status sbslpm_dual_tree_traversal_flagged(int levels, const sbslpm_panel* panels, double theta,
                                                 sbslpm_interact_pair* out, char* near, long cap, long* count) {
  if (!panels || !count || levels < 1 || levels > 12) return SBSLPM_ERR_ARG;
  std::vector<sbslpm_panel> p(panels, panels + sbslpm_panel_count(levels));
  std::vector<sbslpm_interact_pair> list;
  std::vector<char> flags;
  build_interactions_flagged(levels, p, theta, list, flags);
  *count = (long)list.size();
  const size_t n = std::min<size_t>(cap > 0 ? (size_t)cap : 0, list.size());
  if (out && n) std::memcpy(out, list.data(), sizeof(sbslpm_interact_pair) * n);
  if (near && n) std::memcpy(near, flags.data(), n);
  return SBSLPM_OK;
}

sbslpm_status sbslpm_interp_vals_bli(double* basis, double xi, double eta, double min_xi, double max_xi,
                                     double min_eta, double max_eta, int degree) {
  if (!basis || degree < 0 || degree > kMaxDegree) return SBSLPM_ERR_ARG;
  unsigned err = 0;
  host_bli(basis, xi, eta, min_xi, max_xi, min_eta, max_eta, degree, err);
  return err ? SBSLPM_ERR_OUT_OF_PANEL : SBSLPM_OK;
}

int sbslpm_point_locate_panel(const sbslpm_panel* panels, double x, double y, double z) {
  if (!panels) return -1;
  // depth of the uniform tree from the panel table (leaves are the last level)
  int levels = 1;
  while (!panels[level_start(levels - 1)].is_leaf) levels++;
  double xi, eta;
  Bounds b;
  unsigned err = 0;
  int leaf = locate_leaf(x, y, z, levels, xi, eta, b, err);
  return err ? -1 : leaf;
}

sbslpm_status sbslpm_create(const sbslpm_config* cfg, sbslpm_ctx** out) {
  if (!cfg || !out) return SBSLPM_ERR_ARG;
  *out = nullptr;
  SB_TRY(validate(*cfg));
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    set_last_error("no CUDA device available");
    return SBSLPM_ERR_NO_DEVICE;
  }
  sbslpm_ctx* c = new sbslpm_ctx();
  c->cfg = *cfg;
  cudaGetDevice(&c->device);
  c->L = cfg->levels;
  c->d = cfg->interp_degree;
  c->q = (c->d + 1) * (c->d + 1);
  c->P = sbslpm_panel_count(c->L);
  c->A = sbslpm_leaf_count(c->L);
  c->off = c->P - c->A;
  build_panels(c->L, c->panels);
  c->tree = cfg->velocity == SBSLPM_VEL_FMM && cfg->proxy_degree > 0;
  if (cfg->velocity == SBSLPM_VEL_FMM && !c->tree) build_interactions(c->L, c->panels, cfg->fmm_theta, c->list);
  sbslpm_status s = SBSLPM_OK;
  if (cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess) s = SBSLPM_ERR_CUDA;
  if (s == SBSLPM_OK) s = precompute(c);
  if (s == SBSLPM_OK && c->tree) s = precompute_tree(c);
  if (s == SBSLPM_OK && c->tree) {
    int least = 0, greatest = 0;
    if (cudaDeviceGetStreamPriorityRange(&least, &greatest) != cudaSuccess ||
        cudaStreamCreateWithPriority(&c->aux_stream, cudaStreamNonBlocking, greatest) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming) != cudaSuccess)
      s = SBSLPM_ERR_CUDA;
  }
  if (s == SBSLPM_OK) s = allocate_workspace(c);
  if (s == SBSLPM_OK && cfg->forcing != SBSLPM_FORCING_NONE) {
    s = dalloc(&c->force, (size_t)c->A * c->q);
    if (s == SBSLPM_OK) s = dalloc(&c->d_time, 1);
    if (s == SBSLPM_OK && cudaMemset(c->force, 0, sizeof(double) * c->A * c->q) != cudaSuccess) s = SBSLPM_ERR_CUDA;
  }
  c->I = (long)c->list.size();
  if (s != SBSLPM_OK) {
    sbslpm_destroy(c);
    return s;
  }
  fill_geom(c);
  c->geom.force = c->force;
  c->fgeom.force = c->force;
  if (c->tree) {
    BatchMember m{};
    m.fg = c->fgeom;
    m.tg = c->tgeom;
    m.tab = c->ftab;
    m.fsrc = c->fsrc;
    m.ftgt = c->ftgt;
    std::vector<BatchMember> one(1, m);
    s = upload(&c->self, one);
    if (s != SBSLPM_OK) {
      sbslpm_destroy(c);
      return s;
    }
  }
  *out = c;
  return SBSLPM_OK;
}

sbslpm_status sbslpm_destroy(sbslpm_ctx* c) {
  if (!c) return SBSLPM_OK;
  if (c->nccl_comm) {
    cudaStreamSynchronize(c->stream());
    shard_release(c);
  }
  drop_step_graphs(c);
  if (c->swe_graph) cudaGraphExecDestroy(c->swe_graph);
  void* bufs[] = {c->px, c->il_basis, c->child_mat, c->centre, c->tgt_start, c->src_panel, c->il_row, c->src,
                  c->srcf, c->tgt, c->vbuf, c->partial, c->newvor, c->newtr, c->dep, c->err, c->fpx, c->fchild,
                  c->fcentre, c->flx, c->fly, c->fbounds, c->fface, c->near_start, c->near_src, c->cc_start,
                  c->cc_src, c->fsrc, c->psrc, c->fsrcf, c->psrcf, c->ftgt, c->gx, c->near, c->s_fd,
                  c->s_ntan, c->s_pow15, c->s_filt, c->s_ptan, c->s_pface, c->s_ustart, c->s_umem, c->src2,
                  c->srcf2, c->tend, c->avor, c->adj_src, c->adj_vbar, c->adj_q, c->adj_y, c->adj_part,
                  c->adj_w, c->adj_vel, c->adj_near_ts, c->adj_near_tt, c->adj_cc_ts, c->adj_cc_tt, c->adj_tbar,
                  c->adj_qbl, c->self, c->force, c->d_time, c->cc_partial, c->entry32, c->fentry32, c->fsrcp,
                  c->mutual_units, c->near_slot, c->fsrc2, c->psrc2, c->fsrcf2, c->psrcf2, c->adj_ynl,
                  c->swe_cc_partial};
  for (void* b : bufs)
    if (b) cudaFree(b);
  for (int k = 0; k < 4; k++) {
    if (c->cc_chunks[k]) cudaFree(c->cc_chunks[k]);
    if (c->cc_cstart[k]) cudaFree(c->cc_cstart[k]);
  }
  if (c->h_err) cudaFreeHost(c->h_err);
  if (c->own_stream) cudaStreamDestroy(c->own_stream);
  if (c->hio) cudaFree(c->hio);
  if (c->aux_stream) cudaStreamDestroy(c->aux_stream);
  if (c->ev_fork) cudaEventDestroy(c->ev_fork);
  if (c->ev_join) cudaEventDestroy(c->ev_join);
  if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
  if (c->ev_stage0) cudaEventDestroy(c->ev_stage0);
  if (c->ev_copied) cudaEventDestroy(c->ev_copied);
  delete c;
  return SBSLPM_OK;
}

sbslpm_status sbslpm_set_stream(sbslpm_ctx* c, void* stream) {
  if (!c) return SBSLPM_ERR_ARG;
  c->user_stream = static_cast<cudaStream_t>(stream);
  c->user_stream_set = true;
  return SBSLPM_OK;
}

sbslpm_status sbslpm_get_sizes(const sbslpm_ctx* c, long* sizes) {
  if (!c || !sizes) return SBSLPM_ERR_ARG;
  sizes[0] = c->P;
  sizes[1] = c->A;
  sizes[2] = c->q;
  sizes[3] = c->I;
  return SBSLPM_OK;
}

sbslpm_status sbslpm_get_panels(const sbslpm_ctx* c, sbslpm_panel* out) {
  if (!c || !out) return SBSLPM_ERR_ARG;
  std::memcpy(out, c->panels.data(), sizeof(sbslpm_panel) * c->panels.size());
  return SBSLPM_OK;
}

sbslpm_status sbslpm_get_interactions(const sbslpm_ctx* c, sbslpm_interact_pair* out) {
  if (!c || !out) return SBSLPM_ERR_ARG;
  if (!c->list.empty()) std::memcpy(out, c->list.data(), sizeof(sbslpm_interact_pair) * c->list.size());
  return SBSLPM_OK;
}

long sbslpm_kernel_launches(void) { return launch_counter(); }

sbslpm_status sbslpm_bve_step(sbslpm_ctx* c, const double* x, const double* y, const double* z, const double* area,
                              double* vors, double* vel_x, double* vel_y, double* vel_z, double* tracers, double time) {
  if (!c || bad(x) || bad(y) || bad(z) || bad(area) || bad(vors) || bad(vel_x) || bad(vel_y) || bad(vel_z) ||
      (c->cfg.tracer_count > 0 && bad(tracers)) || !std::isfinite(time))
    return SBSLPM_ERR_ARG;
  if (any_on_host({x, y, z, area, vors, vel_x, vel_y, vel_z, tracers}))
    return set_last_error("device-pointer step given host memory (sbslpm_bve_step_host takes host arrays)"), SBSLPM_ERR_ARG;
  SB_TRY(shard_allows(c, true, "a step"));
  SB_TRY(near_autotune(c, x, y, z, area, vors));
  if (c->force) SB_CUDA(cudaMemcpyAsync(c->d_time, &time, sizeof(double), cudaMemcpyHostToDevice, c->stream()));
  enqueue_step(c, x, y, z, area, vors, vel_x, vel_y, vel_z, tracers);
  return finish(c);
}

sbslpm_status sbslpm_bve_step_host(sbslpm_ctx* c, const double* x, const double* y, const double* z,
                                   const double* area, double* vors, double* vel_x, double* vel_y, double* vel_z,
                                   double* tracers, double time) {
  if (!c || bad(x) || bad(y) || bad(z) || bad(area) || bad(vors) || bad(vel_x) || bad(vel_y) || bad(vel_z) ||
      (c->cfg.tracer_count > 0 && bad(tracers)) || !std::isfinite(time))
    return SBSLPM_ERR_ARG;
  SB_TRY(shard_allows(c, true, "a step"));
  const int T = c->cfg.tracer_count;
  const size_t ln = (size_t)c->A * c->q, bytes = sizeof(double) * ln;
  if (!c->hio) {
    SB_TRY(dalloc(&c->hio, (size_t)(5 + T) * ln));
    SB_CUDA(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
    SB_CUDA(cudaEventCreateWithFlags(&c->ev_stage0, cudaEventDisableTiming));
    SB_CUDA(cudaEventCreateWithFlags(&c->ev_copied, cudaEventDisableTiming));
  }
  double* d[5];
  for (int k = 0; k < 5; k++) d[k] = c->hio + (size_t)k * ln;
  double* dtr = T > 0 ? c->hio + 5 * ln : nullptr;
  const double* in[5] = {x, y, z, area, vors};
  double* vel[3] = {vel_x, vel_y, vel_z};
  // copies in, the step, and the copies out; the stage-0 velocity (vbuf's
  // first 3 x leaves*q) leaves on the copy stream while stages 1-3 run
  auto step = [&](bool tune) -> sbslpm_status {
    cudaStream_t st = c->stream();
    for (int k = 0; k < 5; k++) SB_CUDA(cudaMemcpyAsync(d[k], in[k], bytes, cudaMemcpyHostToDevice, st));
    if (T > 0) SB_CUDA(cudaMemcpyAsync(dtr, tracers, bytes * T, cudaMemcpyHostToDevice, st));
    if (tune) SB_TRY(near_autotune(c, d[0], d[1], d[2], d[3], d[4]));
    if (c->force) SB_CUDA(cudaMemcpyAsync(c->d_time, &time, sizeof(double), cudaMemcpyHostToDevice, st));
    enqueue_step(c, d[0], d[1], d[2], d[3], d[4], nullptr, nullptr, nullptr, dtr, c->ev_stage0);
    SB_CUDA(cudaStreamWaitEvent(c->copy_stream, c->ev_stage0, 0));
    for (int k = 0; k < 3; k++)
      SB_CUDA(cudaMemcpyAsync(vel[k], c->vbuf + (size_t)k * ln, bytes, cudaMemcpyDeviceToHost, c->copy_stream));
    SB_CUDA(cudaEventRecord(c->ev_copied, c->copy_stream));
    SB_CUDA(cudaMemcpyAsync(vors, d[4], bytes, cudaMemcpyDeviceToHost, st));
    if (T > 0) SB_CUDA(cudaMemcpyAsync(tracers, dtr, bytes * T, cudaMemcpyDeviceToHost, st));
    SB_CUDA(cudaStreamWaitEvent(st, c->ev_copied, 0));
    return SBSLPM_OK;
  };
  // Page-locked arrays (every one of them) and no forcing or communicator:
  // the step and its copies replay as one CUDA graph, captured after the
  // first eager step with these arrays (which also times the launch shapes).
  auto pinned = [](const void* p) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    return a.type == cudaMemoryTypeHost;
  };
  bool replay = !c->force && !c->nccl_comm;
  for (const void* p : {(const void*)x, (const void*)y, (const void*)z, (const void*)area, (const void*)vors,
                        (const void*)vel_x, (const void*)vel_y, (const void*)vel_z})
    replay = replay && pinned(p);
  if (T > 0) replay = replay && pinned(tracers);
  GraphKey key{{x, y, z, area, vors, vel_x, vel_y, vel_z, tracers}};
  if (replay && c->host_graph && key == c->host_graph_key) {
    SB_CUDA(cudaGraphLaunch(c->host_graph, c->stream()));
    launch_counter() += c->host_launches_per_step;
    return finish(c);
  }
  SB_TRY(step(true));
  const sbslpm_status s = finish(c);
  if (s != SBSLPM_OK || !replay) return s;
  SB_TRY(capture_graph(c, &c->host_graph, [&] { step(false); }));
  c->host_graph_key = key;
  c->host_launches_per_step = c->launches_per_step;
  return SBSLPM_OK;
}

int sbslpm_pointer_on_device(const void* p) {
  if (!p) return -1;
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return -1;
  }
  return (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) ? 1 : 0;
}

sbslpm_status sbslpm_bve_run(sbslpm_ctx* c, const double* x, const double* y, const double* z, const double* area,
                             double* vors, double* vel_x, double* vel_y, double* vel_z, double* tracers, double time,
                             int nsteps) {
  if (!c || bad(x) || bad(y) || bad(z) || bad(area) || bad(vors) || bad(vel_x) || bad(vel_y) || bad(vel_z) ||
      (c->cfg.tracer_count > 0 && bad(tracers)) || nsteps < 0 || !std::isfinite(time))
    return SBSLPM_ERR_ARG;
  if (any_on_host({x, y, z, area, vors, vel_x, vel_y, vel_z, tracers}))
    return set_last_error("device-pointer step given host memory (sbslpm_bve_step_host takes host arrays)"), SBSLPM_ERR_ARG;
  SB_TRY(shard_allows(c, true, "a step"));
  SB_TRY(near_autotune(c, x, y, z, area, vors));
  GraphKey key{{x, y, z, area, vors, vel_x, vel_y, vel_z, tracers}};
  cudaStream_t st = c->stream();
  // step n of the replays runs at time + n dt (each step advances the device time)
  if (c->force) SB_CUDA(cudaMemcpyAsync(c->d_time, &time, sizeof(double), cudaMemcpyHostToDevice, st));
  if (c->nccl_comm) {  // a sharded run enqueues its steps (and their all-gathers) one by one, uncaptured
    for (int s = 0; s < nsteps && c->shard_status == SBSLPM_OK; s++)
      enqueue_step(c, x, y, z, area, vors, vel_x, vel_y, vel_z, tracers);
    return finish(c);
  }
  if (!c->graph || !(key == c->graph_key)) {
    SB_TRY(capture_graph(c, &c->graph, [&] { enqueue_step(c, x, y, z, area, vors, vel_x, vel_y, vel_z, tracers); }));
    c->graph_key = key;
  }
  NvtxRange r("sbslpm bve run (graph replays)");
  for (int s = 0; s < nsteps; s++) {
    SB_CUDA(cudaGraphLaunch(c->graph, st));
    launch_counter() += c->launches_per_step;
  }
  return finish(c);
}

sbslpm_status sbslpm_bve_velocity(sbslpm_ctx* c, const double* x, const double* y, const double* z,
                                  const double* area, const double* vors, double* vel_x, double* vel_y,
                                  double* vel_z) {
  if (!c || bad(x) || bad(y) || bad(z) || bad(area) || bad(vors) || bad(vel_x) || bad(vel_y) || bad(vel_z))
    return SBSLPM_ERR_ARG;
  if (any_on_host({x, y, z, area, vors, vel_x, vel_y, vel_z}))
    return set_last_error("device pointers expected"), SBSLPM_ERR_ARG;
  SB_TRY(on_device(c->device, "the context"));
  if (c->force)
    return set_last_error("a forced context's velocity includes the step's forcing: use the step"), SBSLPM_ERR_CONFIG;
  SB_TRY(near_autotune(c, x, y, z, area, vors));
  cudaStream_t st = c->stream();
  velocity_eval(c, 0, 0.0, nullptr, x, y, z, area, vors, c->vbuf);
  shard_exchange(c, c->vbuf);
  long first = 0, count = (long)c->A * c->q;
  if (!c->nccl_comm) sbslpm_shard_range(c, &first, &count);  // a rank without exchange: its own slice
  const size_t ln = (size_t)c->A * c->q;
  double* out[3] = {vel_x, vel_y, vel_z};
  for (int k = 0; k < 3; k++)
    SB_CUDA(cudaMemcpyAsync(out[k] + first, c->vbuf + k * ln + first, sizeof(double) * count, cudaMemcpyDeviceToDevice,
                            st));
  return finish(c);
}

sbslpm_status sbslpm_upward_pass(sbslpm_ctx* c, const double* area, const double* pots, double* proxy_source) {
  if (!c || bad(area) || bad(pots) || bad(proxy_source)) return SBSLPM_ERR_ARG;
  if (c->tree || c->cfg.velocity != SBSLPM_VEL_FMM)
    return set_last_error("the reference's spectral FMM passes need proxy_degree 0 and FMM velocity"), SBSLPM_ERR_CONFIG;
  cudaStream_t st = c->stream();
  SB_CUDA(cudaMemsetAsync(c->src, 0, sizeof(double4) * c->P * c->q, st));
  launch_upward_fused(c->geom, 1, 0, 0.0, nullptr, nullptr, nullptr, nullptr, pots, area, c->src, false, st);
  launch_copy_strength(c->geom, c->src, proxy_source, st);
  return finish(c);
}

extern "C++" {
namespace sbslpm {
// t_c[i] += tgt[c][i] for the three components (accumulating API of bve_vel_interactions).
__global__ void k_add3(const double* __restrict__ t, long n, double* a, double* b, double* cc) {
  long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  a[i] += t[i];
  b[i] += t[n + i];
  cc[i] += t[2 * n + i];
}
void launch_add3(const double* t, long n, double* a, double* b, double* cc, cudaStream_t st) {
  k_add3<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(t, n, a, b, cc);
  launch_counter()++;
}
}  // namespace sbslpm
}  // extern "C++"

sbslpm_status sbslpm_bve_vel_interactions(sbslpm_ctx* c, const double* dx, const double* dy, const double* dz,
                                          const double* source, double* t1, double* t2, double* t3) {
  if (!c || bad(dx) || bad(dy) || bad(dz) || bad(source) || bad(t1) || bad(t2) || bad(t3)) return SBSLPM_ERR_ARG;
  if (c->cfg.velocity != SBSLPM_VEL_FMM || c->tree)
    return set_last_error("the reference's interaction list needs proxy_degree 0 and FMM velocity"), SBSLPM_ERR_CONFIG;
  cudaStream_t st = c->stream();
  launch_sources_from_disp(c->geom, dx, dy, dz, source, c->src, st);
  launch_interactions(c->geom, c->cfg.precision, c->src, c->tgt, false, st);
  launch_add3(c->tgt, (long)c->P * c->q, t1, t2, t3, st);
  return finish(c);
}

sbslpm_status sbslpm_downward_pass_3(sbslpm_ctx* c, double* t1, double* t2, double* t3, double* s1, double* s2,
                                     double* s3) {
  if (!c || bad(t1) || bad(t2) || bad(t3) || bad(s1) || bad(s2) || bad(s3)) return SBSLPM_ERR_ARG;
  if (c->tree || c->cfg.velocity != SBSLPM_VEL_FMM)
    return set_last_error("the reference's spectral FMM passes need proxy_degree 0 and FMM velocity"), SBSLPM_ERR_CONFIG;
  cudaStream_t st = c->stream();
  size_t pn = (size_t)c->P * c->q, ln = (size_t)c->A * c->q, off = (size_t)c->off * c->q;
  double* tin[3] = {t1, t2, t3};
  double* sout[3] = {s1, s2, s3};
  for (int k = 0; k < 3; k++)
    SB_CUDA(cudaMemcpyAsync(c->tgt + k * pn, tin[k], sizeof(double) * pn, cudaMemcpyDeviceToDevice, st));
  launch_downward_fused(c->geom, c->tgt, nullptr, st);
  for (int k = 0; k < 3; k++) {
    SB_CUDA(cudaMemcpyAsync(tin[k], c->tgt + k * pn, sizeof(double) * pn, cudaMemcpyDeviceToDevice, st));
    SB_CUDA(cudaMemcpyAsync(sout[k], c->tgt + k * pn + off, sizeof(double) * ln, cudaMemcpyDeviceToDevice, st));
  }
  return finish(c);
}

sbslpm_status sbslpm_bve_departure(sbslpm_ctx* c, const double* x, const double* y, const double* z, const double* v0,
                                   const double* v1, const double* v2, const double* v3, double dt, double* dep_x,
                                   double* dep_y, double* dep_z) {
  if (!c || bad(x) || bad(y) || bad(z) || bad(v0) || bad(v1) || bad(v2) || bad(v3) || bad(dep_x) || bad(dep_y) ||
      bad(dep_z))
    return SBSLPM_ERR_ARG;
  cudaStream_t st = c->stream();
  size_t ln = (size_t)c->A * c->q;
  launch_depart_remap(c->geom, &c->tab, x, y, z, v0, v1, v2, v3, dt, c->dep, nullptr, nullptr, 0, nullptr, nullptr, 1,
                      st);
  double* outs[3] = {dep_x, dep_y, dep_z};
  for (int k = 0; k < 3; k++)
    SB_CUDA(cudaMemcpyAsync(outs[k], c->dep + k * ln, sizeof(double) * ln, cudaMemcpyDeviceToDevice, st));
  return finish(c);
}

sbslpm_status sbslpm_bve_remap(sbslpm_ctx* c, const double* z, const double* dep_x, const double* dep_y,
                               const double* dep_z, const double* vors, const double* tracers, double* new_vors,
                               double* new_tracers) {
  if (!c || bad(z) || bad(dep_x) || bad(dep_y) || bad(dep_z) || bad(vors) || bad(new_vors) ||
      (c->cfg.tracer_count > 0 && (bad(tracers) || bad(new_tracers))))
    return SBSLPM_ERR_ARG;
  cudaStream_t st = c->stream();
  size_t ln = (size_t)c->A * c->q;
  const double* ins[3] = {dep_x, dep_y, dep_z};
  for (int k = 0; k < 3; k++)
    SB_CUDA(cudaMemcpyAsync(c->dep + k * ln, ins[k], sizeof(double) * ln, cudaMemcpyDeviceToDevice, st));
  launch_depart_remap(c->geom, &c->tab, nullptr, nullptr, z, nullptr, nullptr, nullptr, nullptr, 0.0, c->dep, vors,
                      tracers, c->cfg.tracer_count, new_vors, new_tracers, 2, st);
  return finish(c);
}

sbslpm_status sbslpm_direct_sum_bve(long nt, const double* tx, const double* ty, const double* tz, long ns,
                                    const double* sx, const double* sy, const double* sz, const double* s, double eps,
                                    int precision, double* ux, double* uy, double* uz, void* stream) {
  if (nt < 0 || ns < 0 || (nt > 0 && (bad(tx) || bad(ty) || bad(tz) || bad(ux) || bad(uy) || bad(uz))) ||
      (ns > 0 && (bad(sx) || bad(sy) || bad(sz) || bad(s))) || (precision != SBSLPM_FP64 && precision != SBSLPM_MIXED))
    return set_last_error("sbslpm_direct_sum_bve: negative size, null array or unknown precision"), SBSLPM_ERR_ARG;
  if (any_on_host({tx, ty, tz, sx, sy, sz, s, ux, uy, uz}))
    return set_last_error("sbslpm_direct_sum_bve: an array is host memory (device pointers expected)"), SBSLPM_ERR_ARG;
  if (nt == 0) return SBSLPM_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (ns == 0) {
    SB_CUDA(cudaMemsetAsync(ux, 0, sizeof(double) * nt, st));
    SB_CUDA(cudaMemsetAsync(uy, 0, sizeof(double) * nt, st));
    SB_CUDA(cudaMemsetAsync(uz, 0, sizeof(double) * nt, st));
    SB_CUDA(cudaStreamSynchronize(st));
    return SBSLPM_OK;
  }
  int groups = direct_groups(nt, ns);
  double* partial = nullptr;
  SB_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&partial), sizeof(double) * 3 * nt * groups, st));
  launch_direct_bve(nt, tx, ty, tz, ns, sx, sy, sz, s, eps, precision, partial, groups, ux, uy, uz, st);
  SB_CUDA(cudaGetLastError());
  SB_CUDA(cudaFreeAsync(partial, st));
  SB_CUDA(cudaStreamSynchronize(st));
  return SBSLPM_OK;
}

sbslpm_status sbslpm_direct_sum_inv_lap(long n, const double* x, const double* y, const double* z, const double* area,
                                        const double* pots, double* soln, void* stream) {
  if (n < 0 || (n > 0 && (bad(x) || bad(y) || bad(z) || bad(area) || bad(pots) || bad(soln))))
    return set_last_error("sbslpm_direct_sum_inv_lap: negative size or null array"), SBSLPM_ERR_ARG;
  if (any_on_host({x, y, z, area, pots, soln}))
    return set_last_error("sbslpm_direct_sum_inv_lap: an array is host memory (device pointers expected)"),
           SBSLPM_ERR_ARG;
  if (n == 0) return SBSLPM_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  launch_inv_lap(n, x, y, z, area, pots, soln, st);
  SB_CUDA(cudaGetLastError());
  SB_CUDA(cudaStreamSynchronize(st));
  return SBSLPM_OK;
}

sbslpm_status sbslpm_time_interactions(sbslpm_ctx* c, int reps, double* ms_per_launch, double* pairs) {
  if (!c || reps < 1 || !ms_per_launch) return SBSLPM_ERR_ARG;
  if (c->cfg.velocity != SBSLPM_VEL_FMM) return set_last_error("context has no interaction list"), SBSLPM_ERR_CONFIG;
  cudaStream_t st = c->stream();
  if (c->tree) {  // the dominant kernel is the near-field particle kernel
    cudaEvent_t a, b;
    SB_CUDA(cudaEventCreate(&a));
    SB_CUDA(cudaEventCreate(&b));
    SB_CUDA(cudaEventRecord(a, st));
    for (int r = 0; r < reps; r++)
      launch_bltc_near_batch(c->self, 1, owned_leaves(c), c->npl, c->cfg.kernel_eps, c->cfg.precision, c->gx,
                             c->gx + c->tgeom.N, c->gx + 2 * c->tgeom.N, c->psrc, c->psrcf, c->near, c->near_splits,
                             c->near_nt, c->near_tpt, c->near_expanded, st);
    SB_CUDA(cudaEventRecord(b, st));
    SB_CUDA(cudaEventSynchronize(b));
    float tms = 0;
    SB_CUDA(cudaEventElapsedTime(&tms, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    *ms_per_launch = tms / reps;
    const long owned_near = c->tgeom.owned > 0 ? c->h_ns[c->tgeom.leaf0 + c->tgeom.owned] - c->h_ns[c->tgeom.leaf0]
                                                : c->n_near;
    if (pairs) *pairs = (double)owned_near * c->npl * c->npl;
    return finish(c);
  }
  if (c->cfg.precision == SBSLPM_MIXED) launch_pack_mixed(c->geom, c->src, st);
  cudaEvent_t e0, e1;
  SB_CUDA(cudaEventCreate(&e0));
  SB_CUDA(cudaEventCreate(&e1));
  SB_CUDA(cudaEventRecord(e0, st));
  for (int r = 0; r < reps; r++) launch_interactions_only(c->geom, c->cfg.precision, c->src, c->tgt, st);
  SB_CUDA(cudaEventRecord(e1, st));
  SB_CUDA(cudaEventSynchronize(e1));
  float ms = 0;
  SB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *ms_per_launch = ms / reps;
  if (pairs) *pairs = (double)c->I * c->q * c->q;
  return finish(c);
}

sbslpm_status sbslpm_set_near_tuning(sbslpm_ctx* c, int threads, int targets_per_thread, int splits) {
  if (!c || !c->tree) return SBSLPM_ERR_ARG;
  const bool ok = ((threads == 64 && (targets_per_thread == 1 || targets_per_thread == 2 || targets_per_thread == 4)) ||
                   (threads == 128 && (targets_per_thread == 1 || targets_per_thread == 2)) ||
                   (threads == 256 && (targets_per_thread == 1 || targets_per_thread == 2))) &&
                  threads * targets_per_thread >= c->npl && splits >= 1 && splits <= 4;
  if (!ok) return set_last_error("unsupported near-field launch shape"), SBSLPM_ERR_ARG;
  c->near_nt = threads;
  c->near_tpt = targets_per_thread;
  c->near_splits = splits;
  c->near_candidates = 0;
  c->near_tuned_ms = 0;
  c->near_tuned = true;
  drop_step_graphs(c);
  return SBSLPM_OK;
}

sbslpm_status sbslpm_set_cc_tuning(sbslpm_ctx* c, int slots, int chunk_len) {
  if (!c || !c->tree) return SBSLPM_ERR_ARG;
  if (!c->cc_partial) return set_last_error("the treecode's proxy count has no chunked well-separated kernel"), SBSLPM_ERR_CONFIG;
  const bool whole = slots == 0 && chunk_len == 0;
  if (!whole && (!cc_chunk_shape_ok(c->qx, slots) || chunk_len < 1 || chunk_len > 4))
    return set_last_error("unsupported well-separated launch shape"), SBSLPM_ERR_ARG;
  c->cc_slots = slots;
  c->cc_len = chunk_len;
  c->cc_tpt = 0;
  c->cc_candidates = 0;
  c->cc_tuned_ms = 0;
  c->cc_tuned = true;
  drop_step_graphs(c);
  return SBSLPM_OK;
}

sbslpm_status sbslpm_set_cc_tuning_direct(sbslpm_ctx* c, int slots, int chunk_len, int targets_per_thread) {
  if (!c || !c->tree) return SBSLPM_ERR_ARG;
  if (!c->cc_partial || !c->fsrcp)
    return set_last_error("the barrier-free well-separated kernel needs mixed precision and 36..121 proxies"),
           SBSLPM_ERR_CONFIG;
  if (!cc_direct_shape_ok(c->qx, slots, targets_per_thread) || chunk_len < 1 || chunk_len > 4)
    return set_last_error("unsupported well-separated launch shape"), SBSLPM_ERR_ARG;
  SB_TRY(sbslpm_set_cc_tuning(c, 0, 0));
  c->cc_slots = slots;
  c->cc_len = chunk_len;
  c->cc_tpt = targets_per_thread;
  return SBSLPM_OK;
}

sbslpm_status sbslpm_cc_tuning(const sbslpm_ctx* c, int* shape, double* ms_per_launch) {
  if (!c || !c->tree || !shape || !ms_per_launch) return SBSLPM_ERR_ARG;
  shape[0] = c->cc_partial && c->cc_slots > 0 ? c->cc_slots : 0;
  shape[1] = c->cc_partial && c->cc_slots > 0 ? c->cc_len : 0;
  shape[2] = c->cc_partial && c->cc_slots > 0 ? cc_chunk_threads(c->qx, c->cc_slots, c->cc_tpt) : 128;
  shape[3] = c->cc_candidates;
  *ms_per_launch = c->cc_tuned_ms;
  return SBSLPM_OK;
}

sbslpm_status sbslpm_set_cc_tuning_bulk(sbslpm_ctx* c, int slots, int chunk_len) {
  if (!c || !c->tree) return SBSLPM_ERR_ARG;
  if (!c->cc_partial || !c->fsrcp)
    return set_last_error("the bulk-copy well-separated kernel needs mixed precision and 36..121 proxies"),
           SBSLPM_ERR_CONFIG;
  if (!cc_chunk_shape_ok(c->qx, slots) || chunk_len < 1 || chunk_len > 4)
    return set_last_error("unsupported well-separated launch shape"), SBSLPM_ERR_ARG;
  SB_TRY(sbslpm_set_cc_tuning(c, 0, 0));
  c->cc_slots = slots;
  c->cc_len = chunk_len;
  c->cc_tpt = kCcBulkForm;
  return SBSLPM_OK;
}

sbslpm_status sbslpm_set_cc_tuning_warp(sbslpm_ctx* c, int warps, int chunk_len) {
  if (!c || !c->tree) return SBSLPM_ERR_ARG;
  if (!c->cc_partial || !c->fsrcp)
    return set_last_error("the warp-per-chunk well-separated kernel needs mixed precision and 36..121 proxies"),
           SBSLPM_ERR_CONFIG;
  if (!cc_warp_shape_ok(c->qx, warps) || chunk_len < 1 || chunk_len > 4)
    return set_last_error("unsupported well-separated launch shape"), SBSLPM_ERR_ARG;
  SB_TRY(sbslpm_set_cc_tuning(c, 0, 0));
  c->cc_slots = warps;
  c->cc_len = chunk_len;
  c->cc_tpt = kCcWarpForm;
  return SBSLPM_OK;
}

sbslpm_status sbslpm_cc_form(const sbslpm_ctx* c, int* targets_per_thread) {
  if (!c || !c->tree || !targets_per_thread) return SBSLPM_ERR_ARG;
  *targets_per_thread = c->cc_partial && c->cc_slots > 0 ? c->cc_tpt : 0;
  return SBSLPM_OK;
}

sbslpm_status sbslpm_set_near_mutual(sbslpm_ctx* c, int on) {
  if (!c || !c->tree) return SBSLPM_ERR_ARG;
  if (on && c->n_mutual == 0)
    return set_last_error("the two-sided near-field kernel needs mixed precision and 256-particle leaves"),
           SBSLPM_ERR_CONFIG;
  if (on && c->shard_n > 1)
    return set_last_error("the two-sided near-field kernel writes both leaves of a pair: one rank only"),
           SBSLPM_ERR_CONFIG;
  c->near_mutual = on != 0;
  drop_step_graphs(c);
  return SBSLPM_OK;
}

sbslpm_status sbslpm_set_near_form(sbslpm_ctx* c, int expanded) {
  if (!c || !c->tree || (expanded != 0 && expanded != 1)) return SBSLPM_ERR_ARG;
  if (expanded && (c->cfg.precision != SBSLPM_MIXED || !(c->cfg.kernel_eps > 0)))
    return set_last_error("the expanded near-field form needs mixed precision and kernel_eps > 0"),
           SBSLPM_ERR_CONFIG;
  c->near_expanded = expanded != 0;
  drop_step_graphs(c);
  return SBSLPM_OK;
}

sbslpm_status sbslpm_near_form(const sbslpm_ctx* c, int* expanded) {
  if (!c || !c->tree || !expanded) return SBSLPM_ERR_ARG;
  *expanded = c->near_expanded ? 1 : 0;
  return SBSLPM_OK;
}

sbslpm_status sbslpm_near_mutual(const sbslpm_ctx* c, int* on, double* ms_per_launch) {
  if (!c || !c->tree || !on || !ms_per_launch) return SBSLPM_ERR_ARG;
  *on = c->near_mutual ? 1 : 0;
  *ms_per_launch = c->near_mutual_ms;
  return SBSLPM_OK;
}

sbslpm_status sbslpm_near_tuning(const sbslpm_ctx* c, int* shape, double* ms_per_launch) {
  if (!c || !c->tree || !shape || !ms_per_launch) return SBSLPM_ERR_ARG;
  shape[0] = c->near_nt;
  shape[1] = c->near_tpt;
  shape[2] = c->near_splits;
  shape[3] = c->near_candidates;
  *ms_per_launch = c->near_tuned_ms;
  return SBSLPM_OK;
}

sbslpm_status sbslpm_measure_fma_peak(int kind, double ms_target, double* flops) {
  if ((kind != 0 && kind != 1) || !flops || !(ms_target > 0)) return SBSLPM_ERR_ARG;
  int dev = 0, sms = 0;
  SB_CUDA(cudaGetDevice(&dev));
  SB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int blocks = sms * 8;  // 8 x 256 threads per SM
  float* o32 = nullptr;
  double* o64 = nullptr;
  SB_CUDA(cudaMalloc(&o32, sizeof(float)));
  SB_CUDA(cudaMalloc(&o64, sizeof(double)));
  cudaEvent_t e0, e1;
  SB_CUDA(cudaEventCreate(&e0));
  SB_CUDA(cudaEventCreate(&e1));
  int iters = 1 << 12;
  float ms = 0;
  for (int attempt = 0; attempt < 12; attempt++) {  // grow iters until the launch lasts ms_target
    launch_fma_probe(kind, blocks, iters, o32, o64, nullptr);
    SB_CUDA(cudaEventRecord(e0, nullptr));
    launch_fma_probe(kind, blocks, iters, o32, o64, nullptr);
    SB_CUDA(cudaEventRecord(e1, nullptr));
    SB_CUDA(cudaEventSynchronize(e1));
    SB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    if (ms >= ms_target) break;
    iters *= 2;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(o32);
  cudaFree(o64);
  *flops = 2.0 * 8.0 * (double)iters * blocks * 256 / (ms * 1e-3);
  return SBSLPM_OK;
}

}  // extern "C"
