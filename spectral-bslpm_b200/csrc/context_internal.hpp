// Internal: the context object shared by the step orchestration files
// (context.cu: set-up, BVE step, C ABI; swe_context.cu: the shallow-water
// step) and their small host helpers.
#pragma once

#include <cuda_runtime.h>

#include <cstring>
#include <functional>
#include <string>
#include <vector>

#include "bve_kernels.cuh"
#include "internal.hpp"
#include "swe_kernels.cuh"

#define SB_CUDA(call)                                                                      \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess) {                                                               \
      set_last_error(std::string(#call) + ": " + cudaGetErrorString(e_));                 \
      return SBSLPM_ERR_CUDA;                                                              \
    }                                                                                      \
  } while (0)

struct GraphKey {
  const void* p[16];
  bool operator==(const GraphKey& o) const { return std::memcmp(p, o.p, sizeof p) == 0; }
};

struct sbslpm_ctx {
  sbslpm_config cfg{};
  int device = 0;  // the device current at creation: buffers and streams live there
  int L = 0, d = 0, q = 0, P = 0, A = 0, off = 0;
  long I = 0;
  std::vector<sbslpm_panel> panels;
  std::vector<sbslpm_interact_pair> list;
  cudaStream_t user_stream = nullptr, own_stream = nullptr;
  bool user_stream_set = false;  // set_stream(NULL) selects the legacy default stream
  // static device data
  double *px = nullptr, *il_basis = nullptr, *child_mat = nullptr, *centre = nullptr;
  int *tgt_start = nullptr, *src_panel = nullptr, *il_row = nullptr;
  int4* entry32 = nullptr;  // mixed, q <= 32: per list entry source panel + centre offset (StepGeom::entry)
  // workspace
  double4* src = nullptr;
  float4* srcf = nullptr;
  double *tgt = nullptr, *vbuf = nullptr, *partial = nullptr, *newvor = nullptr, *newtr = nullptr, *dep = nullptr;
  int groups = 1;
  unsigned* err = nullptr;
  unsigned* h_err = nullptr;
  sbslpm::BliTable tab{};
  sbslpm::StepGeom geom{};
  cudaGraphExec_t graph = nullptr;
  GraphKey graph_key{};
  long launches_per_step = 0;

  // treecode with decoupled proxy degree (proxy_degree > 0)
  bool tree = false;
  int Lf = 0, n = 0, qx = 0, Pf = 0, Af = 0, npl = 0;
  long n_near = 0, n_cc = 0;
  std::vector<sbslpm_panel> fpanels;
  double *fpx = nullptr, *fchild = nullptr, *fcentre = nullptr, *flx = nullptr, *fly = nullptr, *fbounds = nullptr;
  int *fface = nullptr, *near_start = nullptr, *near_src = nullptr, *cc_start = nullptr, *cc_src = nullptr;
  int4* fentry32 = nullptr;  // the same entry table over the well-separated list (mixed, q <= 32)
  double4 *fsrc = nullptr, *psrc = nullptr;
  // SWE on the treecode: the divergence field's particle sources and proxies
  double4 *fsrc2 = nullptr, *psrc2 = nullptr;
  float4 *fsrcf2 = nullptr, *psrcf2 = nullptr;
  double* gx = nullptr;  // [3][particles]: the particle grid, for timing the near kernel alone
  double* near = nullptr;  // [4][3][particles] near-field partial sums (near_splits in use)
  int near_splits = 2, near_nt = 128, near_tpt = 2;  // near-field launch shape (autotuned on the first step)
  // the mixed near field's pair form: expanded (near_expanded_ok at set-up,
  // or sbslpm_set_near_form) or difference
  bool near_expanded = false;
  bool near_tuned = false;
  int near_candidates = 0;
  double near_tuned_ms = 0;
  // the first stage's two-sided near-field kernel (mixed, 256-particle leaves):
  // its units, float32 slot sums, and whether the first-step timing chose it
  int4* mutual_units = nullptr;
  int n_mutual = 0;
  float* near_slot = nullptr;
  bool near_mutual = false;
  double near_mutual_ms = 0;
  // the well-separated list cut into chunks of 1..4 entries per target panel
  // (k = chunk length - 1), used for q >= 36; threads and chunk length are
  // autotuned with the near field
  int4* cc_chunks[4] = {};
  int* cc_cstart[4] = {};
  int cc_nchunks[4] = {};
  double* cc_partial = nullptr;  // [n_cc][3][qx] chunk sums
  double* swe_cc_partial = nullptr;  // [n_cc][6][qx] chunk sums of both SWE fields (mixed treecode)
  int cc_slots = 1, cc_len = 2;  // chunk slots per block (0: one block per target panel), entries per chunk
  int cc_tpt = 0;                 // 0: sources staged in shared memory; 1 | 2: barrier-free, targets per thread
  float4* fsrcp = nullptr;        // pair-transposed packed proxy sources (barrier-free mixed kernel)
  bool cc_tuned = false;
  int cc_candidates = 0;
  double cc_tuned_ms = 0;
  // treecode stages: the tree passes run on aux_stream (higher priority)
  // beside the near field on the context's stream, forked and joined by events
  cudaStream_t aux_stream = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  sbslpm::BatchMember* self = nullptr;
  double* force = nullptr;   // [leaves*q] forcing of the current step (forcing configured)
  double* d_time = nullptr;  // the step's time on the device, advanced by dt inside each step  // this context's treecode as a one-member table (shaped near-field launches)
  float4 *fsrcf = nullptr, *psrcf = nullptr;
  double* ftgt = nullptr;
  sbslpm::BliTable ftab{};
  sbslpm::StepGeom fgeom{};
  sbslpm::TreeGeom tgeom{};

  // shallow water (SWE v2): static tables and workspace, set up on first use
  bool swe_ready = false;
  double *s_fd = nullptr, *s_ntan = nullptr, *s_pow15 = nullptr, *s_filt = nullptr, *s_ptan = nullptr;
  int *s_pface = nullptr, *s_ustart = nullptr, *s_umem = nullptr;
  std::vector<int> two_d_to_1d, unique_counts;
  double4* src2 = nullptr;
  float4* srcf2 = nullptr;
  double* tend = nullptr;  // [3 stages][3 fields][leaves*q]: vorticity, divergence, height tendencies
  double* avor = nullptr;  // arrival vorticity
  sbslpm::SweGeom sgeom{};
  cudaGraphExec_t swe_graph = nullptr;
  GraphKey swe_graph_key{};
  long swe_launches_per_step = 0;

  // host-array step (sbslpm_bve_step_host): device copies of the inputs and
  // outputs, a second stream for the velocity copy, allocated on first use
  double* hio = nullptr;  // [5 + T][leaves*q]: x, y, z, area, vors, tracers
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t ev_stage0 = nullptr, ev_copied = nullptr;
  // the same step with its copies captured as one CUDA graph, for pinned host
  // arrays (keyed by the host pointers)
  cudaGraphExec_t host_graph = nullptr;
  GraphKey host_graph_key{};
  long host_launches_per_step = 0;

  // adjoint workspace, allocated on first use
  double4* adj_src = nullptr;  // [4 stages][panels*q] stage sources (positions, strengths)
  double *adj_vbar = nullptr, *adj_q = nullptr, *adj_y = nullptr, *adj_part = nullptr, *adj_w = nullptr,
         *adj_vel = nullptr;
  int adj_groups = 1;
  int *adj_near_ts = nullptr, *adj_near_tt = nullptr, *adj_cc_ts = nullptr, *adj_cc_tt = nullptr;
  double *adj_tbar = nullptr, *adj_qbl = nullptr;
  double* adj_ynl = nullptr;  // spectral FMM: [3][non-leaf proxies] position adjoints

  // owner-computes sharding of one treecode problem over ranks (shard.cpp):
  // this rank's slice of the tree leaves, the unfiltered well-separated CSR
  // (rebuilt per slice), and the communicator that all-gathers each stage's
  // velocity (null: the rank computes its own slice only)
  int shard_rank = 0, shard_n = 1;
  std::vector<int> h_ns, h_cs, h_csrc;
  std::vector<double> h_fcentre;  // [tree panels][4] panel centres (entry tables)
  void* nccl_comm = nullptr;
  double shard_timeout_s = 300.0;
  sbslpm_status shard_status = SBSLPM_OK;  // a failed exchange inside an enqueued step
  std::string shard_error;

  cudaStream_t stream() const { return user_stream_set ? user_stream : own_stream; }
};

namespace sbslpm {

template <class T>
sbslpm_status dalloc(T** p, size_t count) {
  *p = nullptr;
  if (count == 0) return SBSLPM_OK;
  SB_CUDA(cudaMalloc(reinterpret_cast<void**>(p), sizeof(T) * count));
  return SBSLPM_OK;
}

template <class T>
sbslpm_status upload(T** p, const std::vector<T>& h) {
  sbslpm_status s = dalloc(p, h.size());
  if (s != SBSLPM_OK) return s;
  if (!h.empty()) SB_CUDA(cudaMemcpy(*p, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice));
  return SBSLPM_OK;
}

#define SB_TRY(expr)                           \
  do {                                         \
    sbslpm_status s_ = (expr);                 \
    if (s_ != SBSLPM_OK) return s_;            \
  } while (0)


sbslpm_status finish(sbslpm_ctx* c);
void enqueue_step(sbslpm_ctx* c, const double* x, const double* y, const double* z, const double* area, double* vors,
                  double* vel_x, double* vel_y, double* vel_z, double* tracers,
                  cudaEvent_t stage0 = nullptr);
void velocity_eval(sbslpm_ctx* c, int stage, double dt_s, const double* vprev, const double* x, const double* y,
                   const double* z, const double* area, const double* vors, double* v);
void launch_add3(const double* t, long n, double* a, double* b, double* cc, cudaStream_t st);
sbslpm_status install_cc_lists(sbslpm_ctx* c, const std::vector<int>& cs, const std::vector<int>& csrc);
// shard.cpp: all-gathers a stage velocity [3][particles] over the context's
// ranks (a no-op on an unsharded context); failures land in shard_status
void shard_exchange(sbslpm_ctx* c, double* v);
void shard_release(sbslpm_ctx* c);
// Entry points that run a whole step: a sharded context (more than one rank)
// needs its communicator; the adjoint and the shallow-water step are not
// sharded.  Returns SBSLPM_OK or the refusal (with its message set).
sbslpm_status shard_allows(const sbslpm_ctx* c, bool step_needs_exchange, const char* what);

// tree_setup.cu: host tables of the decoupled-degree treecode.
struct TreeTables {
  int Lf = 0, Pf = 0, Af = 0, npl = 0, n = 0, qx = 0;
  std::vector<sbslpm_panel> fpanels;
  std::vector<double> fpx, centre, bounds, c1d, lx, ly;
  std::vector<int> face;
  BliTable ftab{};
};
struct TreeLists {
  std::vector<int> ns, nsrc, cs, csrc;
  std::vector<sbslpm_interact_pair> list;
};
void child_basis_1d(const std::vector<sbslpm_panel>& P, const BliTable& tab, int d, std::vector<double>& out,
                    unsigned& err);
void bli_table(int n, BliTable& t);
sbslpm_status build_tree_tables(int L, int d, const std::vector<sbslpm_panel>& grid, int leaf_size, int n,
                                TreeTables& t);
// The treecode's lists from the traversal of its tree (list in traversal
// order, near[e] = 1 for pairs that failed the MAC): on the host
// (build_tree_lists) or from a traversal made elsewhere (tree_lists_from;
// device_tree_lists runs the members' traversals on the GPU in one launch
// series).
void build_tree_lists(const TreeTables& t, double theta, TreeLists& l);
// The mixed near field's pair form for these lists and kernel eps: true = the
// expanded form (8 paired operations per two pairs), false = the difference
// form (10); the expanded form only where its rounding stays far below eps.
bool near_expanded_ok(const TreeTables& t, const TreeLists& l, double eps);
void tree_lists_from(const TreeTables& t, std::vector<sbslpm_interact_pair>&& list, const std::vector<char>& near,
                     TreeLists& l);
sbslpm_status device_tree_lists(const TreeTables& t, const std::vector<double>& theta, std::vector<TreeLists>& out,
                                cudaStream_t st);
sbslpm_status near_autotune(sbslpm_ctx* c, const double* x, const double* y, const double* z, const double* area,
                            const double* vors);
// The treecode's well-separated interactions into ftgt (chunked kernels where q allows).
void launch_tree_cc(sbslpm_ctx* c, cudaStream_t st);
// Target leaves the near-field launches cover: this rank's slice when sharded.
inline int owned_leaves(const sbslpm_ctx* c) { return c->tgeom.owned > 0 ? c->tgeom.owned : c->fgeom.leaves; }
sbslpm_status capture_graph(sbslpm_ctx* c, cudaGraphExec_t* graph, const std::function<void()>& body);
// Releases the captured BVE steps (device-array and host-array forms): their
// launch shapes or lists changed.
void drop_step_graphs(sbslpm_ctx* c);

}  // namespace sbslpm
