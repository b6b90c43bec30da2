// One treecode problem sharded over ranks, one GPU each: owner-computes over
// the target leaves.  The reference spreads a step over MPI ranks by slicing
// its interaction list and summing the partial velocities with MPI_Allreduce
// (src/fmm_interactions/bve_vel.cpp:15-33, src/bve_time_step.cpp:346-348).
// Here rank r of R owns a contiguous slice of the tree leaves -- a contiguous
// slice of the particles, since a tree panel's leaves (and its particles) are
// contiguous in the breadth-first panel order.  Every rank keeps the whole
// problem resident (positions, vorticity and the four stage velocities are a
// few tens of MB at 393,216 particles), builds the particle and proxy sources
// and runs the tree passes in full (a small share of the step), and evaluates
// only what lands on its slice: the near field of its leaves, the
// well-separated pairs whose target panel covers one of its leaves, and its
// particles' velocities.  After each RK stage one all-gather over NCCL puts
// every slice into every rank's copy (3 x particles float64 per stage); the
// departure search and remap are replicated.  Each owned target sums the same
// entries in the same order as the unsharded context, so a sharded step is
// bit-identical to the single-GPU step.
//
// NCCL is loaded at run time (libnccl.so.2: the copy a host process already
// holds, e.g. PyTorch's, else the system's), so the library needs it only when
// a communicator is asked for.  The communicator is non-blocking: its set-up
// and every exchange are polled against a time limit, so a rank that never
// joins ends the others' set-up with SBSLPM_ERR_TIMEOUT instead of a hang.
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nccl.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "context_internal.hpp"

using namespace sbslpm;

namespace {

struct NcclApi {
  bool ok = false;
  std::string why;
  ncclResult_t (*get_version)(int*) = nullptr;
  ncclResult_t (*get_unique_id)(ncclUniqueId*) = nullptr;
  ncclResult_t (*init_rank_config)(ncclComm_t*, int, ncclUniqueId, int, ncclConfig_t*) = nullptr;
  ncclResult_t (*async_error)(ncclComm_t, ncclResult_t*) = nullptr;
  ncclResult_t (*abort_comm)(ncclComm_t) = nullptr;
  ncclResult_t (*finalize)(ncclComm_t) = nullptr;
  ncclResult_t (*destroy)(ncclComm_t) = nullptr;
  ncclResult_t (*all_gather)(const void*, void*, size_t, ncclDataType_t, ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*group_start)() = nullptr;
  ncclResult_t (*group_end)() = nullptr;
  const char* (*error_string)(ncclResult_t) = nullptr;
};

template <class F>
bool bind(void* h, const char* name, F& f, std::string& why) {
  f = reinterpret_cast<F>(dlsym(h, name));
  if (!f && why.empty()) why = std::string("libnccl.so.2 lacks ") + name;
  return f != nullptr;
}

const NcclApi& nccl() {
  static NcclApi api;
  static std::once_flag once;
  std::call_once(once, [] {
    void* h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
    if (!h) {
      const char* e = dlerror();
      api.why = std::string("cannot load libnccl.so.2: ") + (e ? e : "unknown");
      return;
    }
    std::string& w = api.why;
    bool ok = bind(h, "ncclGetVersion", api.get_version, w) & bind(h, "ncclGetUniqueId", api.get_unique_id, w) &
              bind(h, "ncclCommInitRankConfig", api.init_rank_config, w) &
              bind(h, "ncclCommGetAsyncError", api.async_error, w) & bind(h, "ncclCommAbort", api.abort_comm, w) &
              bind(h, "ncclCommFinalize", api.finalize, w) & bind(h, "ncclCommDestroy", api.destroy, w) &
              bind(h, "ncclAllGather", api.all_gather, w) & bind(h, "ncclGroupStart", api.group_start, w) &
              bind(h, "ncclGroupEnd", api.group_end, w) & bind(h, "ncclGetErrorString", api.error_string, w);
    int version = 0;
    if (ok && (api.get_version(&version) != ncclSuccess || version < 21400)) {
      w = "NCCL 2.14 or later is needed (non-blocking communicators)";
      ok = false;
    }
    api.ok = ok;
  });
  return api;
}

std::string nccl_error(const NcclApi& n, ncclResult_t r) {
  return n.error_string ? n.error_string(r) : ("NCCL error " + std::to_string((int)r));
}

// Polls a non-blocking communicator until its last operation has left the
// in-progress state, at most timeout_s seconds.
sbslpm_status wait_comm(const NcclApi& n, ncclComm_t comm, double timeout_s, const char* what, std::string& msg) {
  const auto t0 = std::chrono::steady_clock::now();
  for (long spin = 0;; spin++) {
    ncclResult_t state = ncclInProgress;
    const ncclResult_t r = n.async_error(comm, &state);
    if (r != ncclSuccess) state = r;
    if (state == ncclSuccess) return SBSLPM_OK;
    if (state != ncclInProgress) {
      msg = std::string(what) + ": " + nccl_error(n, state);
      return SBSLPM_ERR_CUDA;
    }
    const double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (s > timeout_s) {
      msg = std::string(what) + ": no answer from every rank within " + std::to_string(timeout_s) + " s";
      return SBSLPM_ERR_TIMEOUT;
    }
    if (spin < 1000) std::this_thread::yield();
    else std::this_thread::sleep_for(std::chrono::microseconds(200));
  }
}

}  // namespace

namespace sbslpm {

// Ends the context's communicator: finalized when it is healthy, aborted
// otherwise (or when finalizing runs out of time).
void shard_release(sbslpm_ctx* c) {
  if (!c->nccl_comm) return;
  const NcclApi& n = nccl();
  ncclComm_t comm = static_cast<ncclComm_t>(c->nccl_comm);
  c->nccl_comm = nullptr;
  ncclResult_t state = ncclSuccess;
  std::string msg;
  bool clean = n.async_error(comm, &state) == ncclSuccess && state == ncclSuccess;
  if (clean) {
    const ncclResult_t r = n.finalize(comm);
    clean = (r == ncclSuccess || r == ncclInProgress) &&
            wait_comm(n, comm, c->shard_timeout_s, "finalize", msg) == SBSLPM_OK;
  }
  if (clean) n.destroy(comm);
  else n.abort_comm(comm);
}

sbslpm_status shard_allows(const sbslpm_ctx* c, bool step_needs_exchange, const char* what) {
  SB_TRY(on_device(c->device, "the context"));
  if (c->shard_n <= 1) return SBSLPM_OK;
  if (!step_needs_exchange)
    return set_last_error(std::string(what) + " is not sharded: set one rank (sbslpm_set_shard(ctx, 0, 1, ...))"),
           SBSLPM_ERR_CONFIG;
  if (!c->nccl_comm)
    return set_last_error(std::string(what) + " on a sharded context needs its communicator (a rank without one "
                                              "evaluates its own slice: sbslpm_bve_velocity)"),
           SBSLPM_ERR_CONFIG;
  return SBSLPM_OK;
}

void shard_exchange(sbslpm_ctx* c, double* v) {
  if (!c->nccl_comm || c->shard_status != SBSLPM_OK) return;
  const NcclApi& n = nccl();
  ncclComm_t comm = static_cast<ncclComm_t>(c->nccl_comm);
  const size_t N = (size_t)c->A * c->q, cnt = N / (size_t)c->shard_n;
  // in place: rank r's slice of each component is its send buffer
  ncclResult_t r = n.group_start();
  for (int k = 0; k < 3 && (r == ncclSuccess || r == ncclInProgress); k++) {
    double* comp = v + (size_t)k * N;
    r = n.all_gather(comp + (size_t)c->shard_rank * cnt, comp, cnt, ncclFloat64, comm, c->stream());
  }
  const ncclResult_t e = n.group_end();
  if (r == ncclSuccess || r == ncclInProgress) r = e;
  sbslpm_status s = SBSLPM_OK;
  if (r == ncclInProgress) s = wait_comm(n, comm, c->shard_timeout_s, "stage velocity all-gather", c->shard_error);
  else if (r != ncclSuccess) {
    c->shard_error = "stage velocity all-gather: " + nccl_error(n, r);
    s = SBSLPM_ERR_CUDA;
  }
  c->shard_status = s;
}

}  // namespace sbslpm

extern "C" {

sbslpm_status sbslpm_shard_unique_id(unsigned char* id) {
  if (!id) return SBSLPM_ERR_ARG;
  const NcclApi& n = nccl();
  if (!n.ok) return set_last_error(n.why), SBSLPM_ERR_NO_DEVICE;
  ncclUniqueId u;
  const ncclResult_t r = n.get_unique_id(&u);
  if (r != ncclSuccess) return set_last_error("ncclGetUniqueId: " + nccl_error(n, r)), SBSLPM_ERR_CUDA;
  static_assert(sizeof(u.internal) == 128, "NCCL unique ids are 128 bytes");
  std::memcpy(id, u.internal, 128);
  return SBSLPM_OK;
}

sbslpm_status sbslpm_set_shard(sbslpm_ctx* c, int rank, int nranks, const unsigned char* id, double timeout_s) {
  if (!c) return SBSLPM_ERR_ARG;
  if (!c->tree) return set_last_error("sharding needs the treecode velocity (proxy_degree > 0)"), SBSLPM_ERR_CONFIG;
  if (nranks < 1 || rank < 0 || rank >= nranks)
    return set_last_error("rank must be in [0, nranks), nranks >= 1"), SBSLPM_ERR_ARG;
  if (c->Af % nranks)
    return set_last_error("nranks must divide the tree's " + std::to_string(c->Af) + " leaves"), SBSLPM_ERR_ARG;
  if (!(timeout_s > 0)) timeout_s = 300.0;
  // earlier work ends first
  SB_CUDA(cudaStreamSynchronize(c->stream()));
  // the new communicator first: a set-up that fails leaves the context as it was
  ncclComm_t comm = nullptr;
  if (id) {  // one rank works too: its all-gather is a copy in place
    const NcclApi& n = nccl();
    if (!n.ok) return set_last_error(n.why), SBSLPM_ERR_NO_DEVICE;
    ncclUniqueId u;
    std::memcpy(u.internal, id, 128);
    ncclConfig_t cfg = NCCL_CONFIG_INITIALIZER;
    cfg.blocking = 0;
    const ncclResult_t r = n.init_rank_config(&comm, nranks, u, rank, &cfg);
    if (r != ncclSuccess && r != ncclInProgress) {
      if (comm) n.abort_comm(comm);
      return set_last_error("ncclCommInitRankConfig: " + nccl_error(n, r)), SBSLPM_ERR_CUDA;
    }
    std::string msg;
    const sbslpm_status s = wait_comm(n, comm, timeout_s, "communicator set-up", msg);
    if (s != SBSLPM_OK) {
      n.abort_comm(comm);
      return set_last_error(msg), s;
    }
  }
  // the old communicator and the captured steps go
  shard_release(c);
  drop_step_graphs(c);
  if (c->swe_graph) cudaGraphExecDestroy(c->swe_graph);
  c->swe_graph = nullptr;
  c->shard_status = SBSLPM_OK;
  c->shard_timeout_s = timeout_s;
  c->nccl_comm = comm;

  // leaves [lo, hi) of this rank; a tree panel's leaf range from its children
  const int per = c->Af / nranks, lo = rank * per, hi = lo + per, off = c->Pf - c->Af;
  std::vector<int> first(c->Pf), last(c->Pf);
  for (int p = c->Pf - 1; p >= 0; p--) {
    if (p >= off) {
      first[p] = last[p] = p - off;
      continue;
    }
    const sbslpm_panel& P = c->fpanels[p];
    const int ch[4] = {P.child1, P.child2, P.child3, P.child4};
    first[p] = c->Af;
    last[p] = -1;
    for (int k : ch) {
      first[p] = std::min(first[p], first[k]);
      last[p] = std::max(last[p], last[k]);
    }
  }
  // the well-separated entries of the panels covering an owned leaf, in list order
  std::vector<int> cs(c->Pf + 1, 0), csrc;
  csrc.reserve(c->h_csrc.size() / nranks + 1);
  for (int p = 0; p < c->Pf; p++) {
    cs[p] = (int)csrc.size();
    if (nranks == 1 || (first[p] < hi && last[p] >= lo))
      csrc.insert(csrc.end(), c->h_csrc.begin() + c->h_cs[p], c->h_csrc.begin() + c->h_cs[p + 1]);
  }
  cs[c->Pf] = (int)csrc.size();
  SB_TRY(install_cc_lists(c, cs, csrc));
  c->shard_rank = rank;
  c->shard_n = nranks;
  c->tgeom.leaf0 = nranks > 1 ? lo : 0;
  c->tgeom.owned = nranks > 1 ? per : 0;
  BatchMember m{};
  m.fg = c->fgeom;
  m.tg = c->tgeom;
  m.tab = c->ftab;
  m.fsrc = c->fsrc;
  m.ftgt = c->ftgt;
  SB_CUDA(cudaMemcpy(c->self, &m, sizeof m, cudaMemcpyHostToDevice));
  // launch shapes are timed again on the new lists (the two-sided first-stage
  // kernel writes both leaves of a pair: unsharded contexts only)
  c->near_tuned = false;
  c->near_mutual = false;
  if (c->cc_partial) c->cc_tuned = false;
  return SBSLPM_OK;
}

sbslpm_status sbslpm_shard_range(const sbslpm_ctx* c, long* first, long* count) {
  if (!c || !first || !count) return SBSLPM_ERR_ARG;
  const long N = (long)c->A * c->q;
  if (c->shard_n <= 1) {
    *first = 0;
    *count = N;
  } else {
    *count = N / c->shard_n;
    *first = *count * c->shard_rank;
  }
  return SBSLPM_OK;
}

sbslpm_status sbslpm_shard_release(sbslpm_ctx* c) {
  if (!c) return SBSLPM_ERR_ARG;
  if (c->nccl_comm) SB_CUDA(cudaStreamSynchronize(c->stream()));
  shard_release(c);
  return SBSLPM_OK;
}

}  // extern "C"
