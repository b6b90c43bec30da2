// Batched well-separated (cluster-cluster) proxy interactions of an ensemble
// as a multi-right-hand-side GEMM on the 5th-generation tensor cores.
//
// Members that share a proxy degree share the treecode's proxy points, so for
// a target cluster T and source cluster S the matrix
//     A^c_ab = d^c_ab / (|d_ab|^2 + eps),  d_ab = (s_b - t_a) / sqrt(2)
// (c = x, y, z; the packed form of bve_vel_impl.hpp:49-69's kernel) is the
// same for every member, and member j's proxy-target sum is
//     D^c_a(j) = sum_S sum_b A^c_ab w_b(j)
// with w(j) its proxy source strengths: one GEMM per (T, S) whose right-hand
// sides are the members.  A member whose list (its own theta) lacks (T, S)
// gets a zero row in B.  The GEMM runs as tcgen05.mma kind::tf32 with the
// accumulators in tensor memory; with three passes (A_hi B_hi + A_hi B_lo +
// A_lo B_hi, hi/lo the TF32 split of a float) it keeps float32 accuracy.
#pragma once

#include <cuda_runtime.h>

#include "bve_kernels.cuh"

namespace sbslpm {

// One proxy-degree group of a batch.
struct CcTcGroup {
  int Q;             // proxies per cluster, (n+1)^2 <= 121
  int Pf;            // tree panels
  int nmem;          // members in the group
  int npad;          // members padded to the B row tiling (multiple of 16)
  int ntile;         // members per CTA (multiple of 16, <= npad)
  int kch;           // K chunks (cc_tc_kc(Q) wide) covering Q
  int mw;            // 32-bit mask words per union pair
  int maxlist;       // longest union list of a target (cached in shared memory)
  double eps;
  const int* ustart;     // [Pf+1] CSR of the union of the members' well-separated lists by target
  const int* usrc;       // source cluster of each union pair
  const unsigned* umask; // [pairs][mw] members holding the pair (bit j = group member j)
  const float4* pxf;     // [Pf*Q] proxy points relative to their cluster centre, scaled by 1/sqrt(2)
  const double* centre;  // [Pf][4] cluster centres
  const double* px;      // [3][Pf*Q] proxy points
  float* whi;            // strength image, TF32 high part: [Pf][kch][npad/8][KC/4][8][4]
  float* wlo;            // low part
  const int* idx;        // [nmem] batch index of each group member
  const BatchMember* mem;
  unsigned* err;
  size_t smem3, smem1;  // dynamic shared memory of the 3xTF32 / TF32 kernels (cc_tc_prepare)
  // bound of every mbarrier wait (ns); withhold = 1 keeps one producer
  // thread of every CTA from arriving on the first chunk's barrier, so that
  // the MMA warp's wait runs out (the timeout path's test; no MMA is issued)
  unsigned long long wait_ns = 1000000000ull;
  int withhold = 0;
};

// Kernel attributes and launch shared memory of a group; call once, outside
// any stream capture (sets g.smem3 / g.smem1).
cudaError_t cc_tc_prepare(CcTcGroup& g);
// Pack the members' proxy source strengths (after the upward pass) into the
// B-operand image.
void launch_cc_tc_pack(const CcTcGroup& g, cudaStream_t st);
// D = A W for every target cluster and member, written as the members'
// proxy-target velocities (fg.ftgt).  passes = 3 (3xTF32) or 1 (TF32).
void launch_cc_tc(const CcTcGroup& g, int passes, cudaStream_t st);
// The same interactions on the CUDA cores, the cluster pairs' distances and
// reciprocals shared by groups of 4 consecutive group members
// (cc_chunks.cu; mixed precision; needs ustart/usrc/umask/pxf/centre/px).
void launch_cc_multi(const CcTcGroup& g, cudaStream_t st);
// Dynamic shared memory and tensor-memory columns of one CTA.
size_t cc_tc_smem_bytes(int Q, int ntile, int passes, int maxlist, int mw);
int cc_tc_tmem_cols(int Q, int ntile);
int cc_tc_max_tile(int Q);
int cc_tc_kc(int Q);

}  // namespace sbslpm
