// Dual tree traversal (dual_tree_traversal, src/fmm_funcs.cpp:17-123) on the
// device.  The reference pops (target, source) pairs from a FIFO queue: a pair
// passing the MAC (r_t + r_s) / gcdist(c_t, c_s) < theta, or a leaf-leaf pair,
// is appended to the list, any other pair pushes its four refinements.  A FIFO
// queue processes the pairs generation by generation (all children of
// generation k are pushed after every pair of generation k), so the list is
// the concatenation over generations of each generation's appended pairs in
// queue order, and generation k+1 is the concatenation of the children of
// generation k's split pairs in queue order.  Each generation here is one
// classification kernel, two exclusive prefix sums (list slots, child slots)
// and one emission kernel: the same list in the same order.  Several
// traversals of one tree with their own theta (the ensemble members' lists)
// run together, and every pair records whether it failed the MAC (a near
// leaf pair) as the treecode's lists need.
//
// Panel centres come from the host (the reference's own libm, as the host
// traversal computes them); the distance's acos is the device's.
#include <cuda_runtime.h>

#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cstring>
#include <vector>

#include "context_internal.hpp"
#include "device_common.cuh"

using namespace sbslpm;

namespace {

struct TPanel {
  double cx, cy, cz, radius;
  int level, is_leaf, child[4];
};

// 0: well separated (appended with its type), 1: leaf-leaf near (appended,
// type 0), 2: target refined, 3: source refined.
__device__ __forceinline__ int classify(const TPanel* __restrict__ p, int t, int s, double theta) {
  const TPanel &pt = p[t], &ps = p[s];
  double dp = pt.cx * ps.cx + pt.cy * ps.cy + pt.cz * ps.cz;
  dp = dp > 1.0 ? 1.0 : (dp < -1.0 ? -1.0 : dp);
  const double dist = acos(dp);
  double sep = 100;
  if (dist > 1e-16) sep = (pt.radius + ps.radius) / dist;
  if (sep < theta) return 0;
  if (pt.is_leaf && ps.is_leaf) return 1;
  if (pt.is_leaf) return 3;
  if (ps.is_leaf) return 2;
  return pt.level <= ps.level ? 2 : 3;
}

// Frontier entries are (target, source, member): the members' traversals
// (one theta each) run in one launch series, member-major within every
// generation, so member m's pairs keep its own FIFO order.
__global__ void k_classify(const TPanel* __restrict__ p, const int3* __restrict__ front, long n,
                           const double* __restrict__ theta, int* __restrict__ state, int* __restrict__ nlist,
                           int* __restrict__ nchild) {
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int c = classify(p, front[k].x, front[k].y, theta[front[k].z]);
  state[k] = c;
  nlist[k] = c <= 1 ? 1 : 0;
  nchild[k] = c >= 2 ? 4 : 0;
}

__global__ void k_emit(const TPanel* __restrict__ p, const int3* __restrict__ front, long n, int levels,
                       const int* __restrict__ state, const int* __restrict__ lofs, const int* __restrict__ cofs,
                       long list_base, sbslpm_interact_pair* __restrict__ list, int2* __restrict__ tag,
                       int3* __restrict__ next) {
  const long k = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int t = front[k].x, s = front[k].y, m = front[k].z, c = state[k];
  if (c <= 1) {
    const int type = c == 0 ? (p[t].level < levels - 1 ? 2 : 0) + (p[s].level < levels - 1 ? 1 : 0) : 0;
    const long o = list_base + lofs[k];
    list[o] = sbslpm_interact_pair{t, s, type};
    tag[o] = make_int2(m, c);  // member, 1 = near (failed the MAC)
  } else {
    int3* o = next + cofs[k];
    for (int i = 0; i < 4; i++) o[i] = c == 2 ? make_int3(p[t].child[i], s, m) : make_int3(t, p[s].child[i], m);
  }
}

// A device buffer freed on scope exit.
template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
  cudaError_t reserve(size_t want) {
    if (want <= n) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
    cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&p), sizeof(T) * want);
    if (e == cudaSuccess) n = want;
    return e;
  }
};

}  // namespace

namespace sbslpm {

sbslpm_status device_dual_tree_traversal_multi(int levels, const std::vector<sbslpm_panel>& P,
                                               const std::vector<double>& theta,
                                               std::vector<std::vector<sbslpm_interact_pair>>& out,
                                               std::vector<std::vector<char>>* near, cudaStream_t st) {
  const int np = (int)P.size(), members = (int)theta.size();
  std::vector<TPanel> tp(np);
  for (int i = 0; i < np; i++) {
    const sbslpm_panel& q = P[i];
    double c[3];
    xyz_from_xieta(kPi / 4.0 * 0.5 * (q.min_xi + q.max_xi), kPi / 4.0 * 0.5 * (q.min_eta + q.max_eta), q.face, c);
    tp[i] = TPanel{c[0], c[1], c[2], q.radius, q.level, q.is_leaf, {q.child1, q.child2, q.child3, q.child4}};
  }
  DevBuf<TPanel> dp;
  DevBuf<double> dth;
  DevBuf<int3> front, next;
  DevBuf<int> state, nl, nc, lo, co;
  DevBuf<sbslpm_interact_pair> list;
  DevBuf<int2> tag;
  DevBuf<unsigned char> tmp;
  SB_CUDA(dp.reserve(np));
  SB_CUDA(cudaMemcpyAsync(dp.p, tp.data(), sizeof(TPanel) * np, cudaMemcpyHostToDevice, st));
  SB_CUDA(dth.reserve(members));
  SB_CUDA(cudaMemcpyAsync(dth.p, theta.data(), sizeof(double) * members, cudaMemcpyHostToDevice, st));
  std::vector<int3> f0;
  for (int m = 0; m < members; m++)
    for (int t = 0; t < 6; t++)
      for (int s = 0; s < 6; s++) f0.push_back(make_int3(t, s, m));
  long n = (long)f0.size(), total = 0;
  SB_CUDA(front.reserve(n));
  SB_CUDA(cudaMemcpyAsync(front.p, f0.data(), sizeof(int3) * n, cudaMemcpyHostToDevice, st));
  while (n > 0) {
    if (n > 0x7fffffffL / 4) return set_last_error("dual tree traversal frontier too large"), SBSLPM_ERR_CONFIG;
    SB_CUDA(state.reserve(n));
    SB_CUDA(nl.reserve(n));
    SB_CUDA(nc.reserve(n));
    SB_CUDA(lo.reserve(n));
    SB_CUDA(co.reserve(n));
    const unsigned grid = dev::blocks_for(n, 256);
    k_classify<<<grid, 256, 0, st>>>(dp.p, front.p, n, dth.p, state.p, nl.p, nc.p);
    SB_CUDA(cudaGetLastError());
    size_t tb = 0;
    SB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, nl.p, lo.p, (int)n, st));
    SB_CUDA(tmp.reserve(tb));
    SB_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, tb, nl.p, lo.p, (int)n, st));
    tb = 0;
    SB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, nc.p, co.p, (int)n, st));
    SB_CUDA(tmp.reserve(tb));
    SB_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, tb, nc.p, co.p, (int)n, st));
    int last[4];
    SB_CUDA(cudaMemcpyAsync(&last[0], lo.p + n - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    SB_CUDA(cudaMemcpyAsync(&last[1], nl.p + n - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    SB_CUDA(cudaMemcpyAsync(&last[2], co.p + n - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    SB_CUDA(cudaMemcpyAsync(&last[3], nc.p + n - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    SB_CUDA(cudaStreamSynchronize(st));
    const long added = (long)last[0] + last[1], children = (long)last[2] + last[3];
    if (list.n < (size_t)(total + added)) {  // grow the list and its tags, keeping what they hold
      DevBuf<sbslpm_interact_pair> bigger;
      DevBuf<int2> btag;
      SB_CUDA(bigger.reserve((size_t)(total + added) * 2));
      SB_CUDA(btag.reserve((size_t)(total + added) * 2));
      if (total) {
        SB_CUDA(cudaMemcpyAsync(bigger.p, list.p, sizeof(sbslpm_interact_pair) * total, cudaMemcpyDeviceToDevice,
                                st));
        SB_CUDA(cudaMemcpyAsync(btag.p, tag.p, sizeof(int2) * total, cudaMemcpyDeviceToDevice, st));
      }
      SB_CUDA(cudaStreamSynchronize(st));
      std::swap(list.p, bigger.p);
      std::swap(list.n, bigger.n);
      std::swap(tag.p, btag.p);
      std::swap(tag.n, btag.n);
    }
    SB_CUDA(next.reserve(children > 0 ? children : 1));
    k_emit<<<grid, 256, 0, st>>>(dp.p, front.p, n, levels, state.p, lo.p, co.p, total, list.p, tag.p, next.p);
    SB_CUDA(cudaGetLastError());
    total += added;
    std::swap(front.p, next.p);
    std::swap(front.n, next.n);
    n = children;
  }
  std::vector<sbslpm_interact_pair> all(total);
  std::vector<int2> tags(total);
  if (total) {
    SB_CUDA(cudaMemcpyAsync(all.data(), list.p, sizeof(sbslpm_interact_pair) * total, cudaMemcpyDeviceToHost, st));
    SB_CUDA(cudaMemcpyAsync(tags.data(), tag.p, sizeof(int2) * total, cudaMemcpyDeviceToHost, st));
  }
  SB_CUDA(cudaStreamSynchronize(st));
  // stable split by member: each member's pairs in generation order, that is
  // in its own FIFO order
  out.assign(members, {});
  if (near) near->assign(members, {});
  for (long i = 0; i < total; i++) {
    out[tags[i].x].push_back(all[i]);
    if (near) (*near)[tags[i].x].push_back((char)tags[i].y);
  }
  return SBSLPM_OK;
}

sbslpm_status device_dual_tree_traversal(int levels, const std::vector<sbslpm_panel>& P, double theta,
                                         std::vector<sbslpm_interact_pair>& out, cudaStream_t st) {
  std::vector<std::vector<sbslpm_interact_pair>> lists;
  SB_TRY(device_dual_tree_traversal_multi(levels, P, std::vector<double>{theta}, lists, nullptr, st));
  out.swap(lists[0]);
  return SBSLPM_OK;
}

}  // namespace sbslpm

extern "C" sbslpm_status sbslpm_dual_tree_traversal_device_multi(int levels, const sbslpm_panel* panels, int members,
                                                                const double* theta, sbslpm_interact_pair* out,
                                                                char* near, long cap, long* counts) {
  if (!panels || !theta || !counts || members < 1 || levels < 1 || levels > 12) return SBSLPM_ERR_ARG;
  for (int m = 0; m < members; m++)
    if (!(theta[m] > 0)) return set_last_error("theta must be positive"), SBSLPM_ERR_ARG;
  std::vector<sbslpm_panel> p(panels, panels + sbslpm_panel_count(levels));
  std::vector<std::vector<sbslpm_interact_pair>> lists;
  std::vector<std::vector<char>> flags;
  SB_TRY(device_dual_tree_traversal_multi(levels, p, std::vector<double>(theta, theta + members), lists, &flags,
                                          nullptr));
  long o = 0;
  for (int m = 0; m < members; m++) {
    counts[m] = (long)lists[m].size();
    for (size_t i = 0; i < lists[m].size(); i++, o++) {
      if (o >= cap) continue;
      if (out) out[o] = lists[m][i];
      if (near) near[o] = flags[m][i];
    }
  }
  return SBSLPM_OK;
}

extern "C" sbslpm_status sbslpm_dual_tree_traversal_device(int levels, const sbslpm_panel* panels, double theta,
                                                          sbslpm_interact_pair* out, long cap, long* count) {
  if (!panels || !count || levels < 1 || levels > 12 || !(theta > 0)) return SBSLPM_ERR_ARG;
  std::vector<sbslpm_panel> p(panels, panels + sbslpm_panel_count(levels));
  std::vector<sbslpm_interact_pair> list;
  SB_TRY(device_dual_tree_traversal(levels, p, theta, list, nullptr));
  *count = (long)list.size();
  if (out && cap > 0)
    std::memcpy(out, list.data(), sizeof(sbslpm_interact_pair) * std::min<size_t>((size_t)cap, list.size()));
  return SBSLPM_OK;
}
