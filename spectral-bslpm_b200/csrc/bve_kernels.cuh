// Device kernels of the BVE step (sm_100a).  Launch wrappers are in
// bve_kernels.cu; the step orchestration is in context.cu.
#pragma once

#include <cuda_runtime.h>

#include <atomic>

#include <vector>

#include "geometry.cuh"

namespace sbslpm {

// Mixed precision stores source coordinates scaled by 1/sqrt(2), so that
// |d'|^2 + eps = |d|^2 / 2 + eps is one chain of fused multiply-adds; the
// accumulated sum is scaled back by sqrt(2) with the Biot-Savart constant.
constexpr double kPackScale = 0.70710678118654752440;
constexpr double kBiotSavartPacked = kBiotSavart * 1.41421356237309504880;

// Static per-problem constants used by the BLI code on the device.
struct BliTable {
  double cosv[kMaxDegree + 1];  // cos(pi*i/d), computed on the host with libm
  double w[kMaxDegree + 1];     // barycentric weights of Chebyshev extrema
};

// Everything the stage kernels need, passed by value.
struct StepGeom {
  int levels, degree, q, panels, leaves, offset;  // offset = panels - leaves
  double eps, omega;
  const double* px;           // proxy positions [panels*q] x, y, z blocks (3 * panels*q)
  const int* tgt_start;       // [panels+1] CSR of the interaction list by target
  const int* src_panel;       // [interactions] source panel, list order within a target
  const int* il_row;          // [(panels-leaves)*q] leaf row interpolating a non-leaf proxy
  const double* il_basis;     // [q][(panels-leaves)*q] BLI basis at that leaf, term-major (coalesced per point)
  const double* child_1d;     // [2][d+1][d+1]: 1-D basis of parent node a at the node i of a child in the upper (0) / lower (1) half
  const double* pd_centre;    // mixed: panel centres [panels][4] (double)
  float4* srcf;               // mixed: packed sources [panels*q] (workspace)
  // mixed, q <= 32: per list entry (CSR order) the source panel and the offset
  // of its centre from the target panel's, (float)((c_S - c_T) kPackScale) as
  // float bits
  const int4* entry;
  unsigned* err;              // device error word
  const double* force;        // forcing added to the leaf vorticity [leaves*q], or null
};

// Treecode with decoupled proxy degree (bltc_kernels.cu).  The treecode tree
// itself is described by a StepGeom over its panels with q = (n+1)^2 proxies.
struct TreeGeom {
  int n;                  // proxy degree
  int npl;                // particles per treecode leaf
  long N;                 // particles
  double eps, omega;
  const double* lx;       // [npl][n+1]: leaf-box BLI basis of each particle's xi (same for every leaf)
  const double* ly;       // [npl][n+1]: the same for eta
  const double* fbounds;  // [tree panels][4]: min_xi, max_xi, min_eta, max_eta (radians)
  const int* fface;       // [tree panels]
  const int* near_start;  // [tree leaves + 1]: CSR of near leaf pairs by target leaf
  const int* near_src;    // source leaf (relative to the first leaf)
  // owner-computes slice of the target leaves (a sharded problem): the near
  // field and the particle velocities are evaluated for leaves
  // [leaf0, leaf0 + owned) only; owned 0 = every leaf
  int leaf0 = 0, owned = 0;
};

// One member of a batched ensemble (treecode velocity, shared particle grid):
// its tree and well-separated list (fg, with fg.srcf its packed proxy
// sources), its near lists and leaf bases (tg), its degree's BLI table, and
// its proxy source / target buffers.  Per-particle buffers of the batch are
// [member][...] with a uniform stride.
struct BatchMember {
  StepGeom fg;
  TreeGeom tg;
  BliTable tab;
  double4* fsrc;  // [tree panels * q] proxy sources
  double* ftgt;   // [3][tree panels * q] proxy targets
};

// Launch wrappers (stream-ordered).
void launch_leaf_sources(const StepGeom& g, int stage, double dt_s, const double* vprev, const double* x,
                         const double* y, const double* z, const double* vors, const double* area, double4* src,
                         cudaStream_t st);
// Fused passes: whole tree in ceil((levels-1)/3) launches.  mode 0 = the
// step's sources (leaf sources, non-leaf positions, strengths, mixed
// packing); mode 1 = strengths area*pots only; mode 2 = leaf strengths
// already in src (treecode proxies), mixed packing.
void launch_upward_fused(const StepGeom& g, int mode, int stage, double dt_s, const double* vprev, const double* x,
                         const double* y, const double* z, const double* vors, const double* area, double4* src,
                         bool mixed, cudaStream_t st);
// leaf_out == nullptr: leaf values stay in tgt.
void launch_downward_fused(const StepGeom& g, double* tgt, double* leaf_out, cudaStream_t st);
void launch_interactions(const StepGeom& g, int precision, const double4* src, double* tgt, bool accumulate,
                         cudaStream_t st);
void launch_direct_leaves(const StepGeom& g, int precision, const double4* src, double* vout, double* partial,
                          int groups, cudaStream_t st);
void launch_depart_remap(const StepGeom& g, const BliTable* tab, const double* x, const double* y, const double* z,
                         const double* v0, const double* v1, const double* v2, const double* v3, double dt,
                         double* dep, const double* vors, const double* tracers, int tracer_count, double* new_vors,
                         double* new_tracers, int mode, cudaStream_t st);
// Raw-array helpers for the piecewise API.
void launch_sources_from_disp(const StepGeom& g, const double* dx, const double* dy, const double* dz,
                              const double* source, double4* src, cudaStream_t st);
void launch_copy_strength(const StepGeom& g, const double4* src, double* out, cudaStream_t st);

// Stand-alone direct sums (no tree).
int direct_groups(long n_targets, long n_sources);
void launch_direct_bve(long nt, const double* tx, const double* ty, const double* tz, long ns, const double* sx,
                       const double* sy, const double* sz, const double* s, double eps, int precision, double* partial,
                       int groups, double* ux, double* uy, double* uz, cudaStream_t st);
// bve_ssw_forcing / bve_ssw_forcing_2 (src/forcing_funcs.cpp:6-80) at the
// device-held time: force[leaf][q]; then time += dt (launch_time_advance).
void launch_ssw_forcing(int leaves, int q, int type, double omega, const double* time, const double* x,
                        const double* y, const double* z, double* force, cudaStream_t st);
void launch_time_advance(double* time, double dt, cudaStream_t st);
void launch_inv_lap(long n, const double* x, const double* y, const double* z, const double* area,
                    const double* pots, double* soln, cudaStream_t st);

// Treecode well-separated interactions over chunks of consecutive list
// entries of one target panel (cc_chunks.cu), for q in {36, 49, 64, 81, 100,
// 121}: blocks of `slots` chunks (slots in {1, 2, 3, 4, 6, 8}, at most 512
// threads with at most a fifth of them idle: cc_chunk_shape_ok) write each
// chunk's raw sums to partial[chunk][3][q], then a reduction adds each
// target's chunks in list order into tgt ([3][panels*q]).  chunks[c] =
// (target, first entry, end entry, 0); cstart[panels+1] is the CSR of chunks
// by target.  Mixed precision with direct_tpt = 1 or 2: the barrier-free
// form (k_cc32d: direct_tpt target proxies per thread, sources read through
// L1 from the pair-transposed copy srcp that launch_cc_pair_sources makes of
// the packed proxy sources; cc_direct_shape_ok); with direct_tpt =
// kCcBulkForm: the same slots as the staged form with each slot's source
// panels brought into shared memory by bulk copies (k_cc32t, double-buffered
// through mbarriers; cc_chunk_shape_ok); with direct_tpt = kCcWarpForm: one
// warp per chunk, ceil(q / 32) target proxies per lane, `slots` warps per
// block (1, 2, 4 or 8; cc_warp_shape_ok), each warp staging its source panels
// from srcp with cp.async and __syncwarp only (k_cc32w).
constexpr int kCcBulkForm = 3;
constexpr int kCcWarpForm = 4;
bool cc_warp_shape_ok(int q, int warps);
bool cc_chunk_supported(int q);
bool cc_chunk_shape_ok(int q, int slots);
bool cc_direct_shape_ok(int q, int slots, int tpt);
int cc_chunk_threads(int q, int slots, int direct_tpt = 0);
void launch_cc_pair_sources(const float4* srcf, int q, int panels, float4* srcp, cudaStream_t st);
void launch_cc_chunks(const StepGeom& g, int precision, int slots, const int4* chunks, int nchunks, const int* cstart,
                      const double4* src, double* partial, double* tgt, cudaStream_t st, int direct_tpt = 0,
                      const float4* srcp = nullptr);
void build_cc_chunks(const std::vector<int>& start, int chunk_len, std::vector<int4>& chunks,
                     std::vector<int>& cstart);

// The interaction kernel alone (no mixed-precision packing), for timing.
void launch_interactions_only(const StepGeom& g, int precision, const double4* src, double* tgt, cudaStream_t st);
void launch_pack_mixed(const StepGeom& g, const double4* src, cudaStream_t st);
// FMA-chain throughput probe: kind 0 float32, 1 float64; iters per thread.
void launch_fma_probe(int kind, int blocks, int iters, float* out32, double* out64, cudaStream_t st);

void launch_bltc_sources(const TreeGeom& tg, const StepGeom& fg, const BliTable& tab, int stage, double dt_s,
                         const double* vprev, const double* x, const double* y, const double* z, const double* vors,
                         const double* area, double4* psrc, float4* psrcf, double4* proxy, bool mixed,
                         cudaStream_t st);
// near: splits x 3 x particles partial sums (splits = source-list splits per target leaf)
// v = near splits summed + far field interpolated from the leaf proxies
void launch_bltc_to_particles(const TreeGeom& tg, const StepGeom& fg, const double* tgt, const double* near,
                              int splits, double* v, cudaStream_t st);
// The first stage's near field with each leaf pair evaluated once for both
// directions (kMutualLeaf-particle leaves, mixed precision): units (T, S,
// slot of T <- S, slot of S <- T or -1), float32 slot sums [near entries][3][leaf]
// added per leaf in list order into split 0 of near.
constexpr int kMutualLeaf = 256;
void launch_bltc_near_mutual(const TreeGeom& tg, const StepGeom& fg, const int4* units, int nunits,
                             const float4* psrcf, float* slot, const double* x, const double* y, const double* z,
                             double* near, cudaStream_t st);
void build_mutual_units(const std::vector<int>& ns, const std::vector<int>& nsrc, std::vector<int4>& units);

// Batched treecode (members on one particle grid; one launch per phase over
// all members, the cc launch once per proxy degree).  mem: device array of
// members; per-particle arrays are [member][...]; nmax = largest proxy degree.
void launch_bltc_sources_batch(const BatchMember* mem, int members, int leaves, int npl, int nmax, int stage,
                               double dt_s, const double* vprev, const double* x, const double* y, const double* z,
                               const double* vors, const double* area, double4* psrc, float4* psrcf, bool mixed,
                               cudaStream_t st);
void launch_upward_batch(const BatchMember* mem, int members, int levels, int qmax, bool mixed, cudaStream_t st);
// Stage-0 near field of groups of kNearGroup members (mixed precision): perm
// lists the members by group (theta-sorted), ustart[group][leaves+1] and uent
// (source leaf | member bits << 24) are the groups' union near lists.
constexpr int kNearGroup = 8;
void launch_bltc_near_multi(const BatchMember* mem, const int* perm, int members, int groups, int leaves, int npl,
                            double eps, const int* ustart, const int* uent, const double* x, const double* y,
                            const double* z, const float4* psrcf, double* near, int splits, cudaStream_t st);
// idx: device array of the member indices whose proxies number q
void launch_cc_batch(const BatchMember* mem, const int* idx, int count, int q, int tree_panels, double eps,
                     int precision, cudaStream_t st);
void launch_downward_batch(const BatchMember* mem, int members, int levels, int qmax, cudaStream_t st);
// expanded: the mixed kernel's expanded pair form (pair32x2_expanded; eps > 0 only)
void launch_bltc_near_batch(const BatchMember* mem, int members, int leaves, int npl, double eps, int precision,
                            const double* x, const double* y, const double* z, const double4* psrc,
                            const float4* psrcf, double* near, int splits, int nt, int tpt, bool expanded,
                            cudaStream_t st);
void launch_bltc_to_particles_batch(const BatchMember* mem, int members, int leaves, int nmax, const double* near,
                                    int splits, double* v, cudaStream_t st);
void launch_depart_remap_batch(const StepGeom& g, const BliTable* tab, int members, const double* x,
                               const double* y, const double* z, const double* v0, const double* v1,
                               const double* v2, const double* v3, double dt, const double* vors, double* new_vors,
                               cudaStream_t st);

// Counts every kernel launched through the wrappers above.
// Kernel launches made by the library (a process-wide diagnostic count).
std::atomic<long>& launch_counter();

}  // namespace sbslpm
