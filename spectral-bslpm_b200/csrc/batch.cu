// Batched ensemble of BVE problems on one particle grid: M members, each with
// its own vorticity, MAC parameter theta and treecode proxy degree (uneven
// trees and lists).  One velocity evaluation is one launch per phase over all
// members (the well-separated proxy interactions once per proxy degree), the
// departure search and remap one launch over all members' particles, and a
// whole step one CUDA graph.  The near-field tile shape and source-list split
// are chosen by a timing autotuner on the first step.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "cc_tcgen05.cuh"
#include "context_internal.hpp"
#include "geometry.cuh"

using namespace sbslpm;

struct sbslpm_batch {
  sbslpm_config cfg{};
  int device = 0;  // the device current at creation: buffers and streams live there
  int M = 0, L = 0, d = 0, q = 0, P = 0, A = 0, off = 0;
  long N = 0;
  std::vector<double> theta;
  std::vector<int> degree;
  double lists_s = 0;  // wall time of the members' list build at creation
  std::vector<sbslpm_panel> panels;
  cudaStream_t user_stream = nullptr, own_stream = nullptr;
  // the members' tree passes run on aux_stream (higher priority) beside the
  // near field, forked and joined by events
  cudaStream_t aux_stream = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  bool user_stream_set = false;
  BliTable tab{};
  StepGeom g{};  // the particle grid (departure search and remap)
  int Lf = 0, Pf = 0, Af = 0, npl = 0, nmax = 0, qmax = 0;

  struct Degree {
    int n = -1, qx = 0;
    TreeTables t;
    double *fpx = nullptr, *fcentre = nullptr, *fbounds = nullptr, *fchild = nullptr, *flx = nullptr, *fly = nullptr;
    int* fface = nullptr;
    std::vector<int> members;
    int* d_idx = nullptr;
    // tensor-core well-separated interactions: union of the members' lists
    CcTcGroup tc{};
    long upairs = 0;
    int cc_auto = 0;              // the autotuner's choice for this group (mode 0, 1 or 3)
    double cc_ms[3] = {0, 0, 0};  // its timings of one launch in modes 0, 1 and 3
  };
  std::vector<Degree> degs;
  std::vector<void*> bufs;  // every device buffer of the batch, freed on destroy
  std::vector<BatchMember> h_mem;
  BatchMember* d_mem = nullptr;
  std::vector<long> near_pairs, cc_pairs;  // leaf pairs / well-separated pairs per member

  double4* psrc = nullptr;
  float4* psrcf = nullptr;
  double *near = nullptr, *vbuf = nullptr, *newvor = nullptr;
  unsigned* err = nullptr;
  unsigned* h_err = nullptr;

  // well-separated interactions: -1 autotuned per proxy-degree group (mixed
  // precision default), 0 CUDA-core pairs per member, 1 tensor cores 3xTF32,
  // 2 tensor cores TF32, 3 CUDA-core pairs shared by groups of members
  // (1-3: mixed precision only)
  int cc_mode = 0;

  // stage-0 near field shared by theta-sorted groups of kNearGroup members
  // (mixed precision; off: every member's own near kernel at every stage)
  bool stage0_shared = false;
  int ngroups = 0;
  int *d_perm = nullptr, *d_gstart = nullptr, *d_gent = nullptr;

  // autotuned near-field launch shape
  bool tuned = false;
  int nt = 128, tpt = 2, splits = 2, candidates = 0;
  double tuned_ms = 0;
  // the mixed near field's pair form (near_expanded_ok for every member's list)
  bool near_expanded = false;
  static constexpr int kMaxSplits = 4;

  cudaGraphExec_t graph = nullptr;
  const void* key[7] = {};
  long launches_per_step = 0;

  cudaStream_t stream() const { return user_stream_set ? user_stream : own_stream; }
};

namespace {

template <class T>
sbslpm_status balloc(sbslpm_batch* b, T** p, size_t count) {
  SB_TRY(dalloc(p, count));
  if (*p) b->bufs.push_back(*p);
  return SBSLPM_OK;
}

template <class T>
sbslpm_status bupload(sbslpm_batch* b, T** p, const std::vector<T>& h) {
  SB_TRY(upload(p, h));
  if (*p) b->bufs.push_back(*p);
  return SBSLPM_OK;
}

sbslpm_status batch_finish(sbslpm_batch* b) {
  cudaStream_t st = b->stream();
  SB_CUDA(cudaGetLastError());
  SB_CUDA(cudaMemcpyAsync(b->h_err, b->err, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
  SB_CUDA(cudaStreamSynchronize(st));
  const unsigned e = *b->h_err;
  if (e) {
    SB_CUDA(cudaMemsetAsync(b->err, 0, sizeof(unsigned), st));
    SB_CUDA(cudaStreamSynchronize(st));
    if (e & kErrTimeout)
      return set_last_error("a tensor-core interaction kernel's bounded wait ran out"), SBSLPM_ERR_TIMEOUT;
    if (e & kErrNonFinite) return set_last_error("non-finite point in a location step"), SBSLPM_ERR_NONFINITE;
    return set_last_error("interpolation point outside its panel"), SBSLPM_ERR_OUT_OF_PANEL;
  }
  return SBSLPM_OK;
}

sbslpm_status batch_setup(sbslpm_batch* b) {
  const sbslpm_config& c = b->cfg;
  b->L = c.levels;
  b->d = c.interp_degree;
  b->q = (b->d + 1) * (b->d + 1);
  b->P = sbslpm_panel_count(b->L);
  b->A = sbslpm_leaf_count(b->L);
  b->off = b->P - b->A;
  b->N = (long)b->A * b->q;
  build_panels(b->L, b->panels);
  bli_table(b->d, b->tab);
  SB_TRY(balloc(b, &b->err, 1));
  SB_CUDA(cudaMemset(b->err, 0, sizeof(unsigned)));
  SB_CUDA(cudaMallocHost(reinterpret_cast<void**>(&b->h_err), sizeof(unsigned)));

  StepGeom& g = b->g;
  g.levels = b->L;
  g.degree = b->d;
  g.q = b->q;
  g.panels = b->P;
  g.leaves = b->A;
  g.offset = b->off;
  g.eps = c.kernel_eps;
  g.omega = c.omega;
  g.err = b->err;

  // one set of tree tables per proxy degree in use
  std::vector<int> uniq(b->degree.begin(), b->degree.end());
  std::sort(uniq.begin(), uniq.end());
  uniq.erase(std::unique(uniq.begin(), uniq.end()), uniq.end());
  b->degs.resize(uniq.size());
  for (size_t k = 0; k < uniq.size(); k++) {
    sbslpm_batch::Degree& D = b->degs[k];
    D.n = uniq[k];
    D.qx = (D.n + 1) * (D.n + 1);
    SB_TRY(build_tree_tables(b->L, b->d, b->panels, c.leaf_size, D.n, D.t));
    SB_TRY(bupload(b, &D.fpx, D.t.fpx));
    SB_TRY(bupload(b, &D.fcentre, D.t.centre));
    SB_TRY(bupload(b, &D.fbounds, D.t.bounds));
    SB_TRY(bupload(b, &D.fface, D.t.face));
    if (!D.t.c1d.empty()) SB_TRY(bupload(b, &D.fchild, D.t.c1d));
    SB_TRY(bupload(b, &D.flx, D.t.lx));
    SB_TRY(bupload(b, &D.fly, D.t.ly));
  }
  b->Lf = b->degs[0].t.Lf;
  b->Pf = b->degs[0].t.Pf;
  b->Af = b->degs[0].t.Af;
  b->npl = b->degs[0].t.npl;
  b->nmax = uniq.back();
  b->qmax = (b->nmax + 1) * (b->nmax + 1);

  const bool mixed = c.precision == SBSLPM_MIXED;
  b->cc_mode = mixed ? -1 : 0;
  // tensor-core member tiling of each degree group, and the union of the
  // group's well-separated lists with one member bit per pair
  std::vector<int> gsize(uniq.size(), 0);
  for (int m = 0; m < b->M; m++) gsize[std::lower_bound(uniq.begin(), uniq.end(), b->degree[m]) - uniq.begin()]++;
  std::vector<std::vector<int>> uidx(uniq.size());
  std::vector<std::vector<std::pair<int, int>>> upair(uniq.size());
  std::vector<std::vector<unsigned>> umask(uniq.size());
  for (size_t k = 0; k < uniq.size(); k++) {
    CcTcGroup& G = b->degs[k].tc;
    G.Q = b->degs[k].qx;
    G.Pf = b->degs[k].t.Pf;
    G.nmem = gsize[k];
    const int maxtile = cc_tc_max_tile(G.Q), r16 = (G.nmem + 15) / 16 * 16;
    const int ntiles = (r16 + maxtile - 1) / maxtile;
    G.ntile = ((G.nmem + ntiles - 1) / ntiles + 15) / 16 * 16;
    G.npad = G.ntile * ntiles;
    G.kch = ((G.Q + 7) / 8 * 8 + cc_tc_kc(G.Q) - 1) / cc_tc_kc(G.Q);
    G.mw = (G.npad + 31) / 32;
    G.eps = c.kernel_eps;
    if (mixed) uidx[k].assign((size_t)G.Pf * G.Pf, -1);
  }
  b->h_mem.resize(b->M);
  std::vector<std::vector<int>> hns(b->M), hnsrc(b->M);  // members' near lists (host)
  b->near_pairs.assign(b->M, 0);
  b->cc_pairs.assign(b->M, 0);
  // members in theta order, so that a degree group's member bits (and the
  // shared-pair groups of consecutive bits) follow theta
  std::vector<int> by_theta(b->M);
  for (int m = 0; m < b->M; m++) by_theta[m] = m;
  std::stable_sort(by_theta.begin(), by_theta.end(), [&](int u, int v) { return b->theta[u] < b->theta[v]; });
  // every member's traversal on the GPU in one launch series (the degree
  // groups share the tree: it depends on the leaf size, not on the degree)
  std::vector<TreeLists> lists;
  {
    const auto t0 = std::chrono::steady_clock::now();
    SB_TRY(device_tree_lists(b->degs[0].t, b->theta, lists, nullptr));
    b->lists_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
  b->near_expanded = mixed;
  for (int m = 0; m < b->M && b->near_expanded; m++)
    b->near_expanded = near_expanded_ok(b->degs[0].t, lists[m], b->cfg.kernel_eps);
  for (int mi = 0; mi < b->M; mi++) {
    const int m = by_theta[mi];
    const size_t k = std::lower_bound(uniq.begin(), uniq.end(), b->degree[m]) - uniq.begin();
    sbslpm_batch::Degree& D = b->degs[k];
    D.members.push_back(m);
    TreeLists& l = lists[m];
    hns[m] = l.ns;
    hnsrc[m] = l.nsrc;
    b->near_pairs[m] = l.ns.back();
    b->cc_pairs[m] = l.cs.back();
    if (mixed) {
      const int j = (int)D.members.size() - 1, mw = D.tc.mw, Pf = D.t.Pf;
      for (int t = 0; t < Pf; t++)
        for (int e = l.cs[t]; e < l.cs[t + 1]; e++) {
          int& u = uidx[k][(size_t)t * Pf + l.csrc[e]];
          if (u < 0) {
            u = (int)upair[k].size();
            upair[k].push_back({t, l.csrc[e]});
            umask[k].resize(umask[k].size() + mw, 0u);
          }
          umask[k][(size_t)u * mw + (j >> 5)] |= 1u << (j & 31);
        }
    }
    int *ns = nullptr, *nsrc = nullptr, *cs = nullptr, *csrc = nullptr;
    SB_TRY(bupload(b, &ns, l.ns));
    SB_TRY(bupload(b, &nsrc, l.nsrc));
    SB_TRY(bupload(b, &cs, l.cs));
    SB_TRY(bupload(b, &csrc, l.csrc));
    const size_t pn = (size_t)b->Pf * D.qx;
    double4* fsrc = nullptr;
    float4* fsrcf = nullptr;
    double* ftgt = nullptr;
    SB_TRY(balloc(b, &fsrc, pn));
    std::vector<double4> init(pn);
    for (size_t i = 0; i < pn; i++) init[i] = make_double4(D.t.fpx[i], D.t.fpx[pn + i], D.t.fpx[2 * pn + i], 0.0);
    SB_CUDA(cudaMemcpy(fsrc, init.data(), sizeof(double4) * pn, cudaMemcpyHostToDevice));
    if (mixed) SB_TRY(balloc(b, &fsrcf, pn));
    SB_TRY(balloc(b, &ftgt, 3 * pn));

    BatchMember& bm = b->h_mem[m];
    StepGeom& fg = bm.fg;
    fg = StepGeom{};
    fg.levels = D.t.Lf;
    fg.degree = D.n;
    fg.q = D.qx;
    fg.panels = D.t.Pf;
    fg.leaves = D.t.Af;
    fg.offset = D.t.Pf - D.t.Af;
    fg.eps = c.kernel_eps;
    fg.omega = c.omega;
    fg.px = D.fpx;
    fg.tgt_start = cs;
    fg.src_panel = csrc;
    fg.child_1d = D.fchild;
    fg.pd_centre = D.fcentre;
    fg.srcf = fsrcf;
    fg.err = b->err;
    TreeGeom& tg = bm.tg;
    tg.n = D.n;
    tg.npl = D.t.npl;
    tg.N = b->N;
    tg.eps = c.kernel_eps;
    tg.omega = c.omega;
    tg.lx = D.flx;
    tg.ly = D.fly;
    tg.fbounds = D.fbounds;
    tg.fface = D.fface;
    tg.near_start = ns;
    tg.near_src = nsrc;
    bm.tab = D.t.ftab;
    bm.fsrc = fsrc;
    bm.ftgt = ftgt;
  }
  for (auto& D : b->degs) SB_TRY(bupload(b, &D.d_idx, D.members));
  SB_TRY(bupload(b, &b->d_mem, b->h_mem));
  if (mixed) {
    // members sorted by theta (their near lists nest), in groups of
    // kNearGroup; per group and target leaf the union of the members' near
    // source leaves in ascending order, each with its members' bits
    constexpr int MB = kNearGroup;
    std::vector<int> perm(b->M);
    for (int m = 0; m < b->M; m++) perm[m] = m;
    std::stable_sort(perm.begin(), perm.end(), [&](int u, int v) { return b->theta[u] < b->theta[v]; });
    b->ngroups = (b->M + MB - 1) / MB;
    const int Af = b->Af;
    std::vector<int> gstart((size_t)b->ngroups * (Af + 1), 0), gent;
    std::vector<int> bits(Af, 0), seen;
    for (int g = 0; g < b->ngroups; g++) {
      gstart[(size_t)g * (Af + 1)] = (int)gent.size();  // offsets into gent, all groups in one array
      for (int f = 0; f < Af; f++) {
        seen.clear();
        for (int j = 0; j < MB && g * MB + j < b->M; j++) {
          const int m = perm[g * MB + j];
          for (int e = hns[m][f]; e < hns[m][f + 1]; e++) {
            const int sl = hnsrc[m][e];
            if (!bits[sl]) seen.push_back(sl);
            bits[sl] |= 1 << j;
          }
        }
        std::sort(seen.begin(), seen.end());
        for (int sl : seen) {
          gent.push_back((int)((unsigned)sl | ((unsigned)bits[sl] << 24)));
          bits[sl] = 0;
        }
        gstart[(size_t)g * (Af + 1) + f + 1] = (int)gent.size();
      }
    }
    if (Af < (1 << 24)) {
      SB_TRY(bupload(b, &b->d_perm, perm));
      SB_TRY(bupload(b, &b->d_gstart, gstart));
      if (!gent.empty()) SB_TRY(bupload(b, &b->d_gent, gent));
      b->stage0_shared = !gent.empty();
    }
  }
  if (mixed) {
    for (size_t k = 0; k < b->degs.size(); k++) {
      sbslpm_batch::Degree& D = b->degs[k];
      CcTcGroup& G = D.tc;
      // CSR by target cluster, sources ascending (the accumulation order)
      std::vector<int> order(upair[k].size());
      for (size_t e = 0; e < order.size(); e++) order[e] = (int)e;
      std::sort(order.begin(), order.end(), [&](int x, int y) { return upair[k][x] < upair[k][y]; });
      std::vector<int> us(G.Pf + 1, 0), usrc(order.size());
      std::vector<unsigned> um(order.size() * G.mw);
      for (size_t e = 0; e < order.size(); e++) {
        const auto& pr = upair[k][order[e]];
        us[pr.first + 1]++;
        usrc[e] = pr.second;
        for (int w = 0; w < G.mw; w++) um[e * G.mw + w] = umask[k][(size_t)order[e] * G.mw + w];
      }
      G.maxlist = 0;
      for (int t = 0; t < G.Pf; t++) G.maxlist = std::max(G.maxlist, us[t + 1]);
      for (int t = 0; t < G.Pf; t++) us[t + 1] += us[t];
      D.upairs = (long)order.size();
      int *dus = nullptr, *dusrc = nullptr;
      unsigned* dum = nullptr;
      SB_TRY(bupload(b, &dus, us));
      if (!usrc.empty()) {
        SB_TRY(bupload(b, &dusrc, usrc));
        SB_TRY(bupload(b, &dum, um));
      }
      const size_t pn = (size_t)G.Pf * G.Q;
      std::vector<float4> pxf(pn);
      for (size_t i = 0; i < pn; i++) {
        const double* cc = &D.t.centre[4 * (i / G.Q)];
        pxf[i] = make_float4((float)((D.t.fpx[i] - cc[0]) * kPackScale), (float)((D.t.fpx[pn + i] - cc[1]) * kPackScale),
                             (float)((D.t.fpx[2 * pn + i] - cc[2]) * kPackScale), 0.f);
      }
      float4* dpxf = nullptr;
      SB_TRY(bupload(b, &dpxf, pxf));
      float *whi = nullptr, *wlo = nullptr;
      const size_t wn = (size_t)G.Pf * G.kch * G.npad * cc_tc_kc(G.Q);
      SB_TRY(balloc(b, &whi, wn));
      SB_TRY(balloc(b, &wlo, wn));
      G.ustart = dus;
      G.usrc = dusrc;
      G.umask = dum;
      G.pxf = dpxf;
      G.centre = D.fcentre;
      G.px = D.fpx;
      G.whi = whi;
      G.wlo = wlo;
      G.idx = D.d_idx;
      G.mem = b->d_mem;
      G.err = b->err;
      SB_CUDA(cc_tc_prepare(G));
    }
  }

  const size_t MN = (size_t)b->M * b->N;
  SB_TRY(balloc(b, &b->psrc, MN));
  if (mixed) SB_TRY(balloc(b, &b->psrcf, MN));
  SB_TRY(balloc(b, &b->near, (size_t)sbslpm_batch::kMaxSplits * 3 * MN));
  SB_TRY(balloc(b, &b->vbuf, 4 * 3 * MN));
  SB_TRY(balloc(b, &b->newvor, MN));
  return SBSLPM_OK;
}

// One velocity evaluation of every member (bve_back_rk4_step's stage, with the
// treecode of section "decoupled proxy degree"), stage velocities into v.
void batch_velocity(sbslpm_batch* b, int stage, double dt_s, const double* vprev, const double* x, const double* y,
                    const double* z, const double* area, const double* vors, double* v) {
  cudaStream_t st = b->stream();
  const int prec = b->cfg.precision;
  const bool mixed = prec == SBSLPM_MIXED;
  launch_bltc_sources_batch(b->d_mem, b->M, b->Af, b->npl, b->nmax, stage, dt_s, vprev, x, y, z, vors, area, b->psrc,
                            b->psrcf, mixed, st);
  // the tree passes need only the leaf proxies, the near field only the
  // particle sources: the tree runs on the auxiliary stream beside it
  cudaStream_t tree_st = b->aux_stream ? b->aux_stream : st;
  if (b->aux_stream) {
    cudaEventRecord(b->ev_fork, st);
    cudaStreamWaitEvent(tree_st, b->ev_fork, 0);
  }
  launch_upward_batch(b->d_mem, b->M, b->Lf, b->qmax, mixed, tree_st);
  for (const auto& D : b->degs) {
    const int mode = mixed ? (b->cc_mode < 0 ? D.cc_auto : b->cc_mode) : 0;
    if (mode == 3) {
      launch_cc_multi(D.tc, tree_st);
    } else if (mode != 0) {
      launch_cc_tc_pack(D.tc, tree_st);
      launch_cc_tc(D.tc, mode == 1 ? 3 : 1, tree_st);
    } else {
      launch_cc_batch(b->d_mem, D.d_idx, (int)D.members.size(), D.qx, b->Pf, b->cfg.kernel_eps, prec, tree_st);
    }
  }
  launch_downward_batch(b->d_mem, b->M, b->Lf, b->qmax, tree_st);
  if (b->aux_stream) cudaEventRecord(b->ev_join, tree_st);
  if (stage == 0 && mixed && b->stage0_shared)
    launch_bltc_near_multi(b->d_mem, b->d_perm, b->M, b->ngroups, b->Af, b->npl, b->cfg.kernel_eps, b->d_gstart,
                           b->d_gent, x, y, z, b->psrcf, b->near, b->splits, st);
  else
    launch_bltc_near_batch(b->d_mem, b->M, b->Af, b->npl, b->cfg.kernel_eps, prec, x, y, z, b->psrc, b->psrcf,
                           b->near, b->splits, b->nt, b->tpt, b->near_expanded, st);
  if (b->aux_stream) cudaStreamWaitEvent(st, b->ev_join, 0);
  launch_bltc_to_particles_batch(b->d_mem, b->M, b->Af, b->nmax, b->near, b->splits, v, st);
}

void batch_enqueue_step(sbslpm_batch* b, const double* x, const double* y, const double* z, const double* area,
                        double* vors, double* vel) {
  NvtxRange step_range("sbslpm batch step");
  cudaStream_t st = b->stream();
  const size_t MN = (size_t)b->M * b->N;
  const double dt = b->cfg.dt;
  double* v[4];
  for (int k = 0; k < 4; k++) v[k] = b->vbuf + (size_t)k * 3 * MN;
  const double stage_dt[4] = {0.0, 0.5 * dt, 0.5 * dt, dt};
  for (int s = 0; s < 4; s++) batch_velocity(b, s, stage_dt[s], s ? v[s - 1] : nullptr, x, y, z, area, vors, v[s]);
  launch_depart_remap_batch(b->g, &b->tab, b->M, x, y, z, v[0], v[1], v[2], v[3], dt, vors, b->newvor, st);
  cudaMemcpyAsync(vors, b->newvor, sizeof(double) * MN, cudaMemcpyDeviceToDevice, st);
  cudaMemcpyAsync(vel, v[0], sizeof(double) * 3 * MN, cudaMemcpyDeviceToDevice, st);
}

// Times every near-field launch shape (threads x targets per thread covering a
// leaf, and 1..4 source-list splits) on the members' stage-0 sources and
// keeps the fastest.  Runs once, before the first step, outside any capture.
sbslpm_status batch_autotune(sbslpm_batch* b, const double* x, const double* y, const double* z, const double* area,
                             const double* vors) {
  if (b->tuned) return SBSLPM_OK;
  cudaStream_t st = b->stream();
  const int prec = b->cfg.precision;
  launch_bltc_sources_batch(b->d_mem, b->M, b->Af, b->npl, b->nmax, 0, 0.0, nullptr, x, y, z, vors, area, b->psrc,
                            b->psrcf, prec == SBSLPM_MIXED, st);
  const int shapes[][2] = {{64, 4}, {128, 2}, {256, 1}, {256, 2}, {64, 2}, {64, 1}, {128, 1}};
  cudaEvent_t e0, e1;
  SB_CUDA(cudaEventCreate(&e0));
  SB_CUDA(cudaEventCreate(&e1));
  double best = 1e30;
  int cand = 0;
  for (const auto& sh : shapes) {
    if (sh[0] * sh[1] < b->npl || sh[0] * sh[1] >= 4 * b->npl) continue;
    for (int sp = 1; sp <= sbslpm_batch::kMaxSplits; sp++) {
      launch_bltc_near_batch(b->d_mem, b->M, b->Af, b->npl, b->cfg.kernel_eps, prec, x, y, z, b->psrc, b->psrcf,
                             b->near, sp, sh[0], sh[1], b->near_expanded, st);  // warm-up
      SB_CUDA(cudaEventRecord(e0, st));
      for (int r = 0; r < 3; r++)
        launch_bltc_near_batch(b->d_mem, b->M, b->Af, b->npl, b->cfg.kernel_eps, prec, x, y, z, b->psrc, b->psrcf,
                               b->near, sp, sh[0], sh[1], b->near_expanded, st);
      SB_CUDA(cudaEventRecord(e1, st));
      SB_CUDA(cudaEventSynchronize(e1));
      float ms = 0;
      SB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      cand++;
      if (ms / 3 < best) {
        best = ms / 3;
        b->nt = sh[0];
        b->tpt = sh[1];
        b->splits = sp;
      }
    }
  }
  // well-separated interactions of each proxy-degree group: CUDA-core pairs
  // or the tensor-core 3xTF32 GEMM, whichever is faster here (needs the
  // proxy sources of the stage-0 upward pass)
  if (prec == SBSLPM_MIXED) {
    launch_upward_batch(b->d_mem, b->M, b->Lf, b->qmax, true, st);
    for (auto& D : b->degs) {
      for (int mi = 0; mi < 3; mi++) {
        const int mode = mi == 2 ? 3 : mi;
        auto run = [&] {
          if (mode == 0)
            launch_cc_batch(b->d_mem, D.d_idx, (int)D.members.size(), D.qx, b->Pf, b->cfg.kernel_eps, prec, st);
          else if (mode == 3)
            launch_cc_multi(D.tc, st);
          else {
            launch_cc_tc_pack(D.tc, st);
            launch_cc_tc(D.tc, 3, st);
          }
        };
        run();  // warm-up
        SB_CUDA(cudaEventRecord(e0, st));
        for (int r = 0; r < 3; r++) run();
        SB_CUDA(cudaEventRecord(e1, st));
        SB_CUDA(cudaEventSynchronize(e1));
        float ms = 0;
        SB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        D.cc_ms[mi] = ms / 3;
      }
      const int modes[3] = {0, 1, 3};
      int best = 0;
      for (int mi = 1; mi < 3; mi++)
        if (D.cc_ms[mi] < D.cc_ms[best]) best = mi;
      D.cc_auto = modes[best];
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  b->candidates = cand;
  b->tuned_ms = best;
  b->tuned = true;
  return batch_finish(b);
}

bool bad(const void* p) { return p == nullptr; }

}  // namespace

extern "C" {

sbslpm_status sbslpm_batch_destroy(sbslpm_batch* b) {
  if (!b) return SBSLPM_OK;
  if (b->graph) cudaGraphExecDestroy(b->graph);
  for (void* p : b->bufs) cudaFree(p);
  if (b->h_err) cudaFreeHost(b->h_err);
  if (b->own_stream) cudaStreamDestroy(b->own_stream);
  if (b->aux_stream) cudaStreamDestroy(b->aux_stream);
  if (b->ev_fork) cudaEventDestroy(b->ev_fork);
  if (b->ev_join) cudaEventDestroy(b->ev_join);
  delete b;
  return SBSLPM_OK;
}

sbslpm_status sbslpm_batch_create(const sbslpm_config* base, int members, const double* theta,
                                  const int* proxy_degree, sbslpm_batch** out) {
  if (!base || !theta || !proxy_degree || !out || members < 1 || members > 65535) return SBSLPM_ERR_ARG;
  *out = nullptr;
  sbslpm_config c = *base;
  c.velocity = SBSLPM_VEL_FMM;
  c.tracer_count = 0;
  for (int m = 0; m < members; m++) {
    if (proxy_degree[m] < 5 || proxy_degree[m] > kMaxDegree)
      return set_last_error("batched members need proxy_degree in 5..10"), SBSLPM_ERR_CONFIG;
    if (!(theta[m] > 0) || !std::isfinite(theta[m]))
      return set_last_error("batched members need a positive finite theta"), SBSLPM_ERR_CONFIG;
  }
  if (c.forcing != SBSLPM_FORCING_NONE)
    return set_last_error("batched members run without forcing"), SBSLPM_ERR_CONFIG;
  c.proxy_degree = proxy_degree[0];
  c.fmm_theta = theta[0];
  if (c.levels < 1 || c.levels > 12 || c.interp_degree < 0 || c.interp_degree > kMaxDegree ||
      (c.precision != SBSLPM_FP64 && c.precision != SBSLPM_MIXED) || !(c.kernel_eps >= 0) || !std::isfinite(c.dt) ||
      !std::isfinite(c.omega))
    return set_last_error("invalid base configuration"), SBSLPM_ERR_CONFIG;
  const int qp = (c.interp_degree + 1) * (c.interp_degree + 1);
  long npl = qp;
  while (npl * 4 <= c.leaf_size) npl *= 4;
  if (c.leaf_size < qp || npl > 512)
    return set_last_error("leaf_size must hold at least one panel's points and at most 512"), SBSLPM_ERR_CONFIG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    set_last_error("no CUDA device available");
    return SBSLPM_ERR_NO_DEVICE;
  }
  sbslpm_batch* b = new sbslpm_batch();
  cudaGetDevice(&b->device);
  b->cfg = c;
  b->M = members;
  b->theta.assign(theta, theta + members);
  b->degree.assign(proxy_degree, proxy_degree + members);
  sbslpm_status s = SBSLPM_OK;
  if (cudaStreamCreateWithFlags(&b->own_stream, cudaStreamNonBlocking) != cudaSuccess) s = SBSLPM_ERR_CUDA;
  {
    int least = 0, greatest = 0;
    if (s == SBSLPM_OK &&
        (cudaDeviceGetStreamPriorityRange(&least, &greatest) != cudaSuccess ||
         cudaStreamCreateWithPriority(&b->aux_stream, cudaStreamNonBlocking, greatest) != cudaSuccess ||
         cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
         cudaEventCreateWithFlags(&b->ev_join, cudaEventDisableTiming) != cudaSuccess))
      s = SBSLPM_ERR_CUDA;
  }
  if (s == SBSLPM_OK) s = batch_setup(b);
  if (s != SBSLPM_OK) {
    sbslpm_batch_destroy(b);
    return s;
  }
  *out = b;
  return SBSLPM_OK;
}

sbslpm_status sbslpm_batch_set_stream(sbslpm_batch* b, void* stream) {
  if (!b) return SBSLPM_ERR_ARG;
  b->user_stream = static_cast<cudaStream_t>(stream);
  b->user_stream_set = true;
  return SBSLPM_OK;
}

sbslpm_status sbslpm_batch_get_sizes(const sbslpm_batch* b, long* sizes) {
  if (!b || !sizes) return SBSLPM_ERR_ARG;
  sizes[0] = b->M;
  sizes[1] = b->A;
  sizes[2] = b->q;
  sizes[3] = b->N;
  return SBSLPM_OK;
}

sbslpm_status sbslpm_batch_step(sbslpm_batch* b, const double* x, const double* y, const double* z,
                                const double* area, double* vors, double* vel, double) {
  if (!b || bad(x) || bad(y) || bad(z) || bad(area) || bad(vors) || bad(vel)) return SBSLPM_ERR_ARG;
  if (any_on_host({x, y, z, area, vors, vel}))
    return set_last_error("device-pointer step given host memory"), SBSLPM_ERR_ARG;
  SB_TRY(on_device(b->device, "the batch"));
  SB_TRY(batch_autotune(b, x, y, z, area, vors));
  batch_enqueue_step(b, x, y, z, area, vors, vel);
  return batch_finish(b);
}

sbslpm_status sbslpm_batch_run(sbslpm_batch* b, const double* x, const double* y, const double* z,
                               const double* area, double* vors, double* vel, double, int nsteps) {
  if (!b || bad(x) || bad(y) || bad(z) || bad(area) || bad(vors) || bad(vel) || nsteps < 0) return SBSLPM_ERR_ARG;
  if (any_on_host({x, y, z, area, vors, vel}))
    return set_last_error("device-pointer step given host memory"), SBSLPM_ERR_ARG;
  SB_TRY(on_device(b->device, "the batch"));
  SB_TRY(batch_autotune(b, x, y, z, area, vors));
  const void* key[7] = {x, y, z, area, vors, vel, nullptr};
  cudaStream_t st = b->stream();
  if (!b->graph || std::memcmp(key, b->key, sizeof key) != 0) {
    if (b->graph) {
      cudaGraphExecDestroy(b->graph);
      b->graph = nullptr;
    }
    cudaStream_t cap = b->own_stream;
    if (st != cap) {
      cudaEvent_t ev;
      SB_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
      SB_CUDA(cudaEventRecord(ev, st));
      SB_CUDA(cudaStreamWaitEvent(cap, ev, 0));
      cudaEventDestroy(ev);
    }
    const bool saved = b->user_stream_set;
    b->user_stream_set = false;
    const long before = launch_counter();
    cudaGraph_t gr;
    SB_CUDA(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
    batch_enqueue_step(b, x, y, z, area, vors, vel);
    cudaError_t ce = cudaStreamEndCapture(cap, &gr);
    b->user_stream_set = saved;
    b->launches_per_step = launch_counter() - before;
    launch_counter() = before;
    SB_CUDA(ce);
    SB_CUDA(cudaGraphInstantiateWithFlags(&b->graph, gr, cudaGraphInstantiateFlagUseNodePriority));
    cudaGraphDestroy(gr);
    std::memcpy(b->key, key, sizeof key);
  }
  for (int s = 0; s < nsteps; s++) {
    SB_CUDA(cudaGraphLaunch(b->graph, st));
    launch_counter() += b->launches_per_step;
  }
  return batch_finish(b);
}

sbslpm_status sbslpm_batch_tuning(const sbslpm_batch* b, int* shape, double* ms_per_launch) {
  if (!b || !shape || !ms_per_launch) return SBSLPM_ERR_ARG;
  shape[0] = b->nt;
  shape[1] = b->tpt;
  shape[2] = b->splits;
  shape[3] = b->candidates;
  *ms_per_launch = b->tuned_ms;
  return SBSLPM_OK;
}

sbslpm_status sbslpm_batch_set_tuning(sbslpm_batch* b, int threads, int targets_per_thread, int splits) {
  if (!b) return SBSLPM_ERR_ARG;
  const bool ok = ((threads == 64 && (targets_per_thread == 1 || targets_per_thread == 2 || targets_per_thread == 4)) ||
                   (threads == 128 && (targets_per_thread == 1 || targets_per_thread == 2)) ||
                   (threads == 256 && (targets_per_thread == 1 || targets_per_thread == 2))) &&
                  threads * targets_per_thread >= b->npl && splits >= 1 && splits <= sbslpm_batch::kMaxSplits;
  if (!ok) return set_last_error("unsupported near-field launch shape"), SBSLPM_ERR_ARG;
  b->nt = threads;
  b->tpt = targets_per_thread;
  b->splits = splits;
  b->candidates = 0;
  b->tuned_ms = 0;
  b->tuned = true;
  if (b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  return SBSLPM_OK;
}

sbslpm_status sbslpm_batch_set_near_form(sbslpm_batch* b, int expanded) {
  if (!b || (expanded != 0 && expanded != 1)) return SBSLPM_ERR_ARG;
  if (expanded && (b->cfg.precision != SBSLPM_MIXED || !(b->cfg.kernel_eps > 0)))
    return set_last_error("the expanded near-field form needs mixed precision and kernel_eps > 0"),
           SBSLPM_ERR_CONFIG;
  if ((bool)expanded != b->near_expanded && b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  b->near_expanded = expanded != 0;
  return SBSLPM_OK;
}

sbslpm_status sbslpm_batch_near_form(const sbslpm_batch* b, int* expanded) {
  if (!b || !expanded) return SBSLPM_ERR_ARG;
  *expanded = b->near_expanded ? 1 : 0;
  return SBSLPM_OK;
}

sbslpm_status sbslpm_batch_set_stage0_shared(sbslpm_batch* b, int shared) {
  if (!b || (shared != 0 && shared != 1)) return SBSLPM_ERR_ARG;
  if (shared && !b->d_gent)
    return set_last_error("the shared stage-0 near field needs a mixed-precision batch"), SBSLPM_ERR_CONFIG;
  if ((bool)shared != b->stage0_shared && b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  b->stage0_shared = shared != 0;
  return SBSLPM_OK;
}

sbslpm_status sbslpm_batch_set_cc_mode(sbslpm_batch* b, int mode) {
  if (!b || mode < -1 || mode > 3) return SBSLPM_ERR_ARG;
  if (mode > 0 && b->cfg.precision != SBSLPM_MIXED)
    return set_last_error("the tensor-core and shared-pair well-separated modes need mixed precision"),
           SBSLPM_ERR_CONFIG;
  if (mode != b->cc_mode && b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  b->cc_mode = mode;
  return SBSLPM_OK;
}

sbslpm_status sbslpm_batch_set_wait_test(sbslpm_batch* b, int on) {
  if (!b) return SBSLPM_ERR_ARG;
  for (auto& D : b->degs) {
    D.tc.withhold = on ? 1 : 0;
    D.tc.wait_ns = on ? 2000000ull : 1000000000ull;
  }
  if (b->graph) {  // the groups are kernel arguments captured in the graph
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  return SBSLPM_OK;
}

sbslpm_status sbslpm_batch_setup_times(const sbslpm_batch* b, double* lists_s) {
  if (!b || !lists_s) return SBSLPM_ERR_ARG;
  *lists_s = b->lists_s;
  return SBSLPM_OK;
}

sbslpm_status sbslpm_batch_cc_info(const sbslpm_batch* b, int* mode, double* union_pairs, double* mma_flops) {
  if (!b || !mode || !union_pairs || !mma_flops) return SBSLPM_ERR_ARG;
  *mode = b->cc_mode;
  double up = 0, fl = 0;
  for (const auto& D : b->degs) {
    const CcTcGroup& G = D.tc;
    const int mode = b->cc_mode < 0 ? D.cc_auto : b->cc_mode;
    up += (double)D.upairs;
    if (mode == 1 || mode == 2) {
      const double tiles = ((3 * G.Q + 127) / 128), ksteps = (G.Q + 7) / 8;
      fl += (double)D.upairs * tiles * ksteps * 2.0 * 128 * 8 * G.npad * (mode == 1 ? 3 : 1);
    }
  }
  *union_pairs = up;
  *mma_flops = fl;
  return SBSLPM_OK;
}

sbslpm_status sbslpm_batch_cc_groups(const sbslpm_batch* b, int n, int* degree, int* members, int* mode,
                                     double* ms_cuda_cores, double* ms_tensor_cores, double* ms_shared) {
  if (!b || n < 0 || !degree || !members || !mode || !ms_cuda_cores || !ms_tensor_cores || !ms_shared)
    return SBSLPM_ERR_ARG;
  for (int k = 0; k < n && k < (int)b->degs.size(); k++) {
    const auto& D = b->degs[k];
    degree[k] = D.n;
    members[k] = (int)D.members.size();
    mode[k] = b->cfg.precision != SBSLPM_MIXED ? 0 : (b->cc_mode < 0 ? D.cc_auto : b->cc_mode);
    ms_cuda_cores[k] = D.cc_ms[0];
    ms_tensor_cores[k] = D.cc_ms[1];
    ms_shared[k] = D.cc_ms[2];
  }
  return (int)b->degs.size() > n ? SBSLPM_ERR_ARG : SBSLPM_OK;
}

sbslpm_status sbslpm_batch_pairs(const sbslpm_batch* b, double* near_pairs, double* far_pairs) {
  if (!b || !near_pairs || !far_pairs) return SBSLPM_ERR_ARG;
  double np = 0, fp = 0;
  for (int m = 0; m < b->M; m++) {
    const double qx = (b->degree[m] + 1.0) * (b->degree[m] + 1.0);
    np += (double)b->near_pairs[m] * b->npl * b->npl;
    fp += (double)b->cc_pairs[m] * qx * qx;
  }
  *near_pairs = np;
  *far_pairs = fp;
  return SBSLPM_OK;
}

}  // extern "C"
