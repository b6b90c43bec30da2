// Device kernels of the BVE backward semi-Lagrangian step, sm_100a.
//
// Data layout in HBM (all row-major, [panel][q] as in the reference):
//   src   : double4 [panels*q]  displaced source position (x, y, z) and
//           strength w = area * vorticity (leaves) or its anterpolation
//           (non-leaf proxies).  32 B per proxy point, one load per pair block.
//   srcf  : float4  [panels*q]  mixed precision: position relative to the
//           panel centre (float) and strength (float).
//   tgt   : double  [3][panels*q] proxy-target velocities.
//   v_k   : double  [3][leaves*q] stage velocities (x, y, z blocks).
// Every kernel is owner-computes (no atomics), so results are deterministic.
#include <cuda_runtime.h>

#include <cstdio>
#include <type_traits>

#include "../../include/sbslpm.h"
#include "bve_kernels.cuh"
#include "device_common.cuh"

namespace sbslpm {

std::atomic<long>& launch_counter() {
  static std::atomic<long> n{0};
  return n;
}

namespace {

using namespace dev;

constexpr int kWarpsPerBlock = 4;

// ---------------------------------------------------------------------------
// Source preparation.

// Leaves (bve_disp_update, src/bve_time_step.cpp:69-105, with the forcing
// copy of src/forcing_funcs.cpp:93-95 and base_pots, src/fmm_funcs_impl.hpp:17-34):
// stage 0: strength area*vor at proj(proxy); stage s > 0: disp = dt_s v,
// strength area*(vor + 2 Omega z - 2 Omega z'), z' from proj(x + v dt_s),
// position proj(proxy + disp).
__global__ void k_leaf_sources(StepGeom g, int stage, double dt_s, const double* __restrict__ vprev,
                               const double* __restrict__ x, const double* __restrict__ y,
                               const double* __restrict__ z, const double* __restrict__ vors,
                               const double* __restrict__ area, double4* __restrict__ src) {
  long n = (long)g.leaves * g.q;
  long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  long pn = (long)g.panels * g.q;
  long o = (long)g.offset * g.q + i;
  double px = g.px[o], py = g.px[pn + o], pz = g.px[2 * pn + o];
  double w;
  if (stage == 0) {
    w = area[i] * (g.force ? vors[i] + g.force[i] : vors[i]);
  } else {
    double vx = vprev[i], vy = vprev[n + i], vz = vprev[2 * n + i];
    double xx = x[i] + vx * dt_s, yy = y[i] + vy * dt_s, zz = z[i] + vz * dt_s;
    project_to_sphere(xx, yy, zz);
    double dvor = vors[i] + 2 * g.omega * z[i] - 2 * g.omega * zz;
    w = area[i] * (g.force ? dvor + g.force[i] : dvor);
    px += dt_s * vx;
    py += dt_s * vy;
    pz += dt_s * vz;
  }
  project_to_sphere(px, py, pz);
  src[o] = make_double4(px, py, pz, w);
}

// Piecewise API: sources from explicit displacements and strengths
// (the inputs of bve_vel_interactions).
__global__ void k_sources_from_disp(StepGeom g, const double* __restrict__ dx, const double* __restrict__ dy,
                                    const double* __restrict__ dz, const double* __restrict__ s,
                                    double4* __restrict__ src) {
  long pn = (long)g.panels * g.q;
  long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= pn) return;
  double px = g.px[i] + dx[i], py = g.px[pn + i] + dy[i], pz = g.px[2 * pn + i] + dz[i];
  project_to_sphere(px, py, pz);
  src[i] = make_double4(px, py, pz, s[i]);
}

__global__ void k_copy_strength(StepGeom g, const double4* __restrict__ src, double* __restrict__ out) {
  long pn = (long)g.panels * g.q;
  long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= pn) return;
  out[i] = src[i].w;
}

// ---------------------------------------------------------------------------
// Tree passes (upward_pass / downward_pass_3, src/fmm_funcs.cpp:341-392;
// child_to_parent / parent_to_child_3, src/fmm_funcs_impl.hpp:36-172).
// The BLI basis of parent node (a,b) at child c's node (i,j) is the product
// Lx_c[i][a] Ly_c[j][b] of one-dimensional bases, and the uniform quadtree has
// only two of them: child_1d[h][i][a] for the child in the upper (h = 0) or
// lower (h = 1) half of its parent.  The passes contract one direction at a
// time:
//   upward:   T[c][i][b] = sum_j Ly_c[j][b] S_c[i][j];  S[a][b] = sum_c sum_i Lx_c[i][a] T[c][i][b]
//   downward: U[c][a][j] = sum_b Ly_c[j][b] T[a][b];    T_c[i][j] += sum_a Lx_c[i][a] U[c][a][j]
//
// One CTA owns the subtree of depth D below one panel of level r and keeps
// the strengths (upward) or target values (downward) of all its levels in
// shared memory, so a pass over the whole tree takes ceil((L-1)/3) launches.
//
// Upward, mode 0 (the step): when the subtree reaches the leaves, the leaf
// sources are computed here (bve_disp_update, src/bve_time_step.cpp:69-105,
// with the forcing copy and base_pots folded in); the non-leaf proxies of the
// subtree get their displaced positions (bve_disp_interp,
// src/bve_time_step.cpp:107-160, leaf row and BLI basis precomputed on the
// host); strengths are anterpolated level by level; in mixed precision the
// packed float4 sources are written for every panel the CTA owns.
// Mode 1 (sbslpm_upward_pass): leaf strengths area * pots, positions untouched.
// Mode 2 (treecode): leaf strengths already anterpolated into src, fixed
// proxy positions untouched, mixed packing as in mode 0.

__device__ __forceinline__ void upward_subtree_body(const StepGeom& g, int root_rel, int r, int D, int mode,
                                                    int positions, int stage, double dt_s,
                                                    const double* __restrict__ vprev,
                                                    const double* __restrict__ x, const double* __restrict__ y,
                                                    const double* __restrict__ z, const double* __restrict__ vors,
                                                    const double* __restrict__ area, double4* __restrict__ src,
                                                    int mixed) {
  extern __shared__ double sh[];  // strengths of levels r..r+D (level k at q*(4^k-1)/3), then scratch
  const int q = g.q, n1 = g.degree + 1;
  const bool leaves_here = (r + D == g.levels - 1);
  const long ln = (long)g.leaves * g.q, pn = (long)g.panels * g.q;
  auto lvl = [&](int k) { return sh + q * (((1 << (2 * k)) - 1) / 3); };

  // bottom level of the subtree: leaf sources, or strengths computed by the previous launch
  {
    const int first = subtree_first(r, root_rel, D), npts = (1 << (2 * D)) * q;
    double* bot = lvl(D);
    for (int t = threadIdx.x; t < npts; t += blockDim.x) {
      const long o = (long)first * q + t;
      if (leaves_here && mode != 2) {
        const long i = o - (long)g.offset * q;
        double w;
        if (mode == 1) {
          w = area[i] * vors[i];
          src[o].w = w;
        } else {
          double px = g.px[o], py = g.px[pn + o], pz = g.px[2 * pn + o];
          if (stage == 0) {
            w = area[i] * (g.force ? vors[i] + g.force[i] : vors[i]);
          } else {
            double vx = vprev[i], vy = vprev[ln + i], vz = vprev[2 * ln + i];
            double xx = x[i] + vx * dt_s, yy = y[i] + vy * dt_s, zz = z[i] + vz * dt_s;
            project_to_sphere(xx, yy, zz);
            double dvor = vors[i] + 2 * g.omega * z[i] - 2 * g.omega * zz;
            w = area[i] * (g.force ? dvor + g.force[i] : dvor);
            px += dt_s * vx;
            py += dt_s * vy;
            pz += dt_s * vz;
          }
          project_to_sphere(px, py, pz);
          src[o] = make_double4(px, py, pz, w);
        }
        bot[t] = w;
      } else {
        bot[t] = src[o].w;
      }
    }
  }
  // displaced positions of the subtree's non-leaf proxies (levels r..r+D-1),
  // unless k_nonleaf_positions wrote them before the pass
  if (mode == 0 && positions) {
    for (int k = 0; k < D; k++) {
      const int first = subtree_first(r, root_rel, k), npts = (1 << (2 * k)) * q;
      for (int t = threadIdx.x; t < npts; t += blockDim.x) {
        const long i = (long)first * q + t;
        double px, py, pz;
        nonleaf_position(g, i, stage, dt_s, vprev, px, py, pz);
        src[i] = make_double4(px, py, pz, 0.0);
      }
    }
  }
  __syncthreads();
  // anterpolation, deepest parents first, one direction at a time
  double* scratch = sh + q * (((1 << (2 * (D + 1))) - 1) / 3);
  for (int k = D - 1; k >= 0; k--) {
    const double* ch = lvl(k + 1);
    double* pa = lvl(k);
    const int np = 1 << (2 * k), first = subtree_first(r, root_rel, k);
    for (int t = threadIdx.x; t < 4 * np * q; t += blockDim.x) {  // T[cc][i][b]
      const int cc = t / q, rem = t % q, i = rem / n1, b = rem % n1;
      const double* ly = g.child_1d + ((cc & 3) >= 2 ? n1 * n1 : 0);
      const double* sc = ch + cc * q + i * n1;
      double acc = 0;
      for (int j = 0; j < n1; j++) acc = fma(__ldg(ly + j * n1 + b), sc[j], acc);
      scratch[t] = acc;
    }
    __syncthreads();
    for (int t = threadIdx.x; t < np * q; t += blockDim.x) {  // S[p][a][b]
      const int p = t / q, rem = t % q, a = rem / n1, b = rem % n1;
      double acc = 0;
      for (int c = 0; c < 4; c++) {
        const double* lx = g.child_1d + ((c == 1 || c == 2) ? n1 * n1 : 0);
        const double* tc = scratch + (4 * p + c) * q + b;
        for (int i = 0; i < n1; i++) acc = fma(__ldg(lx + i * n1 + a), tc[i * n1], acc);
      }
      pa[t] = acc;
      src[(long)first * q + t].w = acc;
    }
    __syncthreads();
  }
  // mixed precision: float4 sources relative to the panel centre, for every panel this CTA owns
  if (mixed && mode != 1) {
    const int kmax = leaves_here ? D : D - 1;
    for (int k = 0; k <= kmax; k++) {
      const int first = subtree_first(r, root_rel, k), npts = (1 << (2 * k)) * q;
      for (int t = threadIdx.x; t < npts; t += blockDim.x) {
        const long i = (long)first * q + t;
        const double* cc = g.pd_centre + 4 * (i / q);
        double4 sv = src[i];
        g.srcf[i] = make_float4((float)((sv.x - cc[0]) * kPackScale), (float)((sv.y - cc[1]) * kPackScale),
                                (float)((sv.z - cc[2]) * kPackScale), (float)sv.w);
      }
    }
  }
}

__global__ void k_upward_subtree(StepGeom g, int r, int D, int mode, int positions, int stage, double dt_s,
                                 const double* __restrict__ vprev, const double* __restrict__ x,
                                 const double* __restrict__ y, const double* __restrict__ z,
                                 const double* __restrict__ vors, const double* __restrict__ area,
                                 double4* __restrict__ src, int mixed) {
  upward_subtree_body(g, blockIdx.x, r, D, mode, positions, stage, dt_s, vprev, x, y, z, vors, area, src, mixed);
}

// The displaced positions of every non-leaf proxy (bve_disp_interp,
// src/bve_time_step.cpp:107-160) in one flat launch, a thread per point, ahead
// of the subtree passes of mode 0: the same arithmetic as nonleaf_position,
// with the q-term interpolation unrolled for q = 16, so that the passes
// themselves no longer wait on these gathers level by level.
template <int Q>
__global__ void k_nonleaf_positions(StepGeom g, int stage, double dt_s, const double* __restrict__ vprev,
                                    double4* __restrict__ src) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const int q = Q > 0 ? Q : g.q;
  if (i >= (long)g.offset * q) return;
  const long pn = (long)g.panels * q, ln = (long)g.leaves * q;
  double px = g.px[i], py = g.px[pn + i], pz = g.px[2 * pn + i];
  if (stage > 0) {
    const long np = (long)g.offset * q;
    const long row = (long)g.il_row[i] * q;
    double ax = 0, ay = 0, az = 0;
#pragma unroll
    for (int m = 0; m < (Q > 0 ? Q : q); m++) {
      const double bm = g.il_basis[m * np + i];
      ax += (dt_s * vprev[row + m]) * bm;
      ay += (dt_s * vprev[ln + row + m]) * bm;
      az += (dt_s * vprev[2 * ln + row + m]) * bm;
    }
    px += ax;
    py += ay;
    pz += az;
  }
  project_to_sphere(px, py, pz);
  src[i] = make_double4(px, py, pz, 0.0);
}

// Batched treecode members (mode 2): member blockIdx.z.
__global__ void k_upward_subtree_batch(const BatchMember* __restrict__ mem, int r, int D, int mixed) {
  const StepGeom g = mem[blockIdx.z].fg;
  upward_subtree_body(g, blockIdx.x, r, D, 2, 0, 0, 0.0, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                      mem[blockIdx.z].fsrc, mixed);
}

// Downward: the root's targets are final; children of levels r+1..r+D get
// own + interpolated parent values.  Leaves go to leaf_out when given (the
// stage velocity), intermediate levels stay in shared memory, and the
// deepest non-leaf level is written back for the next launch.
__device__ __forceinline__ void downward_subtree_body(const StepGeom& g, int root_rel, int r, int D,
                                                      double* __restrict__ tgt, double* __restrict__ leaf_out) {
  extern __shared__ double sh[];  // 3 fields x levels r..r+D, then 3 x 4^D q scratch
  const int q = g.q, n1 = g.degree + 1;
  const long pn = (long)g.panels * g.q, ln = (long)g.leaves * g.q;
  const int per_field = q * (((1 << (2 * (D + 1))) - 1) / 3);
  auto lvl = [&](int f, int k) { return sh + f * per_field + q * (((1 << (2 * k)) - 1) / 3); };
  double* scratch = sh + 3 * per_field;
  const int sstride = (1 << (2 * D)) * q;
  {
    const int first = subtree_first(r, root_rel, 0);
    for (int t = threadIdx.x; t < q; t += blockDim.x)
      for (int f = 0; f < 3; f++) lvl(f, 0)[t] = tgt[f * pn + (long)first * q + t];
  }
  __syncthreads();
  for (int k = 1; k <= D; k++) {
    const int level = r + k, npts = (1 << (2 * k)) * q, first = subtree_first(r, root_rel, k);
    const bool is_leaf = (level == g.levels - 1);
    for (int t = threadIdx.x; t < npts; t += blockDim.x) {  // U[cc][a][j]
      const int cc = t / q, rem = t % q, a = rem / n1, j = rem % n1;
      const double* ly = g.child_1d + ((cc & 3) >= 2 ? n1 * n1 : 0) + j * n1;
      const int pp = cc >> 2;
      const double *p0 = lvl(0, k - 1) + pp * q + a * n1, *p1 = lvl(1, k - 1) + pp * q + a * n1,
                   *p2 = lvl(2, k - 1) + pp * q + a * n1;
      double u0 = 0, u1 = 0, u2 = 0;
      for (int b = 0; b < n1; b++) {
        const double l = __ldg(ly + b);
        u0 = fma(l, p0[b], u0);
        u1 = fma(l, p1[b], u1);
        u2 = fma(l, p2[b], u2);
      }
      scratch[t] = u0;
      scratch[sstride + t] = u1;
      scratch[2 * sstride + t] = u2;
    }
    __syncthreads();
    for (int t = threadIdx.x; t < npts; t += blockDim.x) {  // T_c[i][j] += sum_a Lx[i][a] U[a][j]
      const int cc = t / q, rem = t % q, i = rem / n1, j = rem % n1, c = cc & 3;
      const double* lx = g.child_1d + ((c == 1 || c == 2) ? n1 * n1 : 0) + i * n1;
      const double* u = scratch + cc * q + j;
      double a0 = 0, a1 = 0, a2 = 0;
      for (int a = 0; a < n1; a++) {
        const double l = __ldg(lx + a);
        a0 = fma(l, u[a * n1], a0);
        a1 = fma(l, u[sstride + a * n1], a1);
        a2 = fma(l, u[2 * sstride + a * n1], a2);
      }
      const long o = (long)first * q + t;
      a0 += tgt[o];
      a1 += tgt[pn + o];
      a2 += tgt[2 * pn + o];
      lvl(0, k)[t] = a0;
      lvl(1, k)[t] = a1;
      lvl(2, k)[t] = a2;
      if (is_leaf && leaf_out != nullptr) {
        const long lo = o - (long)g.offset * q;
        leaf_out[lo] = a0;
        leaf_out[ln + lo] = a1;
        leaf_out[2 * ln + lo] = a2;
      } else if (k == D || is_leaf || leaf_out == nullptr) {
        tgt[o] = a0;
        tgt[pn + o] = a1;
        tgt[2 * pn + o] = a2;
      }
    }
    __syncthreads();
  }
}

__global__ void k_downward_subtree(StepGeom g, int r, int D, double* __restrict__ tgt,
                                   double* __restrict__ leaf_out) {
  downward_subtree_body(g, blockIdx.x, r, D, tgt, leaf_out);
}

__global__ void k_downward_subtree_batch(const BatchMember* __restrict__ mem, int r, int D) {
  const StepGeom g = mem[blockIdx.z].fg;
  downward_subtree_body(g, blockIdx.x, r, D, mem[blockIdx.z].ftgt, nullptr);
}

// ---------------------------------------------------------------------------
// Interactions (bve_vel_panel_interaction, src/fmm_interactions/bve_vel_impl.hpp:85-122).
//
// One warp owns one target panel and walks its sources (CSR list, or all
// leaves in direct mode).  For q <= 16 the warp's lanes are (split h,
// target node j): split h takes every S-th source panel, stages its q
// points in shared memory and every lane of the split runs over them.  For
// q > 32 each lane owns ceil(q/32) target nodes and the whole warp stages
// one source panel at a time.  Partial sums of the splits are combined in a
// fixed order, so the result is deterministic.
//
// Direct mode (ALL_LEAVES) splits the source leaves into gridDim.y groups
// and writes per-group partials that k_reduce_groups sums in order.

template <int Q>
struct WarpShape {
  static constexpr int S = Q <= 16 ? 32 / Q : 1;          // source splits per warp
  static constexpr int STAGE = (S * Q > Q ? S * Q : Q);    // staged points per warp
  static constexpr int Q2 = (Q + 1) / 2;                    // source pairs per panel
  static constexpr int STAGE2 = (S > 1 ? S : 1) * 2 * Q2;   // float4 slots per warp, paired layout
};

template <int Q, bool ALL_LEAVES, bool GUARD>
__global__ void __launch_bounds__(32 * kWarpsPerBlock) k_interact64(StepGeom g, const double4* __restrict__ src,
                                                                    double* __restrict__ out, long out_stride) {
  using W = WarpShape<Q>;
  __shared__ double4 stage[kWarpsPerBlock][W::STAGE];
  __shared__ double red[kWarpsPerBlock][3][32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int tp_first = ALL_LEAVES ? g.offset : 0;
  const int tp_count = ALL_LEAVES ? g.leaves : g.panels;
  const int tix = blockIdx.x * kWarpsPerBlock + warp;
  if (tix >= tp_count) return;
  const int t = tp_first + tix;
  const long pn = (long)g.panels * g.q;

  int e0, e1;
  if (ALL_LEAVES) {
    int per = (g.leaves + gridDim.y - 1) / gridDim.y;
    e0 = blockIdx.y * per;
    e1 = min(g.leaves, e0 + per);
  } else {
    e0 = g.tgt_start[t];
    e1 = g.tgt_start[t + 1];
  }
  auto source_of = [&](int e) { return ALL_LEAVES ? g.offset + e : __ldg(g.src_panel + e); };

  if constexpr (Q <= 32) {
    const int h = lane / Q, j = lane % Q;
    const bool active = h < W::S;
    double tx = 0, ty = 0, tz = 0;
    if (active) {
      long o = (long)t * Q + j;
      tx = g.px[o];
      ty = g.px[pn + o];
      tz = g.px[2 * pn + o];
    }
    double ax = 0, ay = 0, az = 0;
    if constexpr (ALL_LEAVES) {
      for (int e = e0; e < e1; e += W::S) {
        if (active && e + h < e1) stage[warp][h * Q + j] = src[(long)source_of(e + h) * Q + j];
        __syncwarp();
        if (active && e + h < e1) {
          const double4* sp = &stage[warp][h * Q];
#pragma unroll
          for (int k = 0; k < Q; k++) pair64<GUARD>(tx, ty, tz, sp[k], g.eps, ax, ay, az);
        }
        __syncwarp();
      }
    } else {
      // the list in batches of 32 entries, one source index per lane, handed
      // to the splits by shuffles; the next entry's sources are loaded while
      // the current ones are evaluated
      for (int eb = e0; eb < e1; eb += 32) {
        const int nb = min(32, e1 - eb);
        const int idx = lane < nb ? __ldg(g.src_panel + eb + lane) : 0;
        const int iters = (nb + W::S - 1) / W::S;
        double4 sv = make_double4(0, 0, 0, 0);
        {
          const int sp = __shfl_sync(0xffffffffu, idx, h & 31);
          if (active && h < nb) sv = src[(long)sp * Q + j];
        }
        for (int it = 0; it < iters; it++) {
          const bool on = active && it * W::S + h < nb;
          const int ns = (it + 1) * W::S + h;
          const int sp_n = __shfl_sync(0xffffffffu, idx, ns & 31);
          double4 sv_n = make_double4(0, 0, 0, 0);
          if (active && ns < nb) sv_n = src[(long)sp_n * Q + j];
          if (on) stage[warp][h * Q + j] = sv;
          __syncwarp();
          if (on) {
            const double4* sp = &stage[warp][h * Q];
#pragma unroll
            for (int k = 0; k < Q; k++) pair64<GUARD>(tx, ty, tz, sp[k], g.eps, ax, ay, az);
          }
          __syncwarp();
          sv = sv_n;
        }
      }
    }
    if (W::S > 1) {
      red[warp][0][lane] = ax;
      red[warp][1][lane] = ay;
      red[warp][2][lane] = az;
      __syncwarp();
      if (h == 0) {
        for (int hh = 1; hh < W::S; hh++) {
          ax += red[warp][0][hh * Q + j];
          ay += red[warp][1][hh * Q + j];
          az += red[warp][2][hh * Q + j];
        }
      }
    }
    if (h == 0) {
      double ux = kBiotSavart * (ty * az - tz * ay);
      double uy = kBiotSavart * (tz * ax - tx * az);
      double uz = kBiotSavart * (tx * ay - ty * ax);
      long o = ALL_LEAVES ? (long)blockIdx.y * 3 * out_stride + (long)tix * Q + j : (long)t * Q + j;
      long s = ALL_LEAVES ? out_stride : pn;
      out[o] = ux;
      out[s + o] = uy;
      out[2 * s + o] = uz;
    }
  } else {
    constexpr int TPL = Q <= 32 ? 1 : (Q + 31) / 32;  // target nodes per lane
    double tx[TPL], ty[TPL], tz[TPL], ax[TPL], ay[TPL], az[TPL];
#pragma unroll
    for (int r = 0; r < TPL; r++) {
      int j = lane + 32 * r;
      long o = (long)t * Q + (j < Q ? j : 0);
      tx[r] = g.px[o];
      ty[r] = g.px[pn + o];
      tz[r] = g.px[2 * pn + o];
      ax[r] = ay[r] = az[r] = 0;
    }
    for (int e = e0; e < e1; e++) {
      const long sb = (long)source_of(e) * Q;
      for (int k = lane; k < Q; k += 32) stage[warp][k] = src[sb + k];
      __syncwarp();
      for (int k = 0; k < Q; k++) {
        const double4 s = stage[warp][k];
#pragma unroll
        for (int r = 0; r < TPL; r++) pair64<GUARD>(tx[r], ty[r], tz[r], s, g.eps, ax[r], ay[r], az[r]);
      }
      __syncwarp();
    }
#pragma unroll
    for (int r = 0; r < TPL; r++) {
      int j = lane + 32 * r;
      if (j >= Q) continue;
      double ux = kBiotSavart * (ty[r] * az[r] - tz[r] * ay[r]);
      double uy = kBiotSavart * (tz[r] * ax[r] - tx[r] * az[r]);
      double uz = kBiotSavart * (tx[r] * ay[r] - ty[r] * ax[r]);
      long o = ALL_LEAVES ? (long)blockIdx.y * 3 * out_stride + (long)tix * Q + j : (long)t * Q + j;
      long s = ALL_LEAVES ? out_stride : pn;
      out[o] = ux;
      out[s + o] = uy;
      out[2 * s + o] = uz;
    }
  }
}

// Mixed precision: positions relative to panel centres in float, pair
// arithmetic in float32, per-source-panel partial sums in float32 added into
// float64 accumulators.  For q <= 32 the two float32 halves of a panel's sum
// are added in float32 before the conversion: with 16 sources per panel the
// float64 conversions would otherwise load the MUFU/conversion pipe more than
// the reciprocals do.
__global__ void k_pack_mixed(StepGeom g, const double4* __restrict__ src, float4* __restrict__ srcf) {
  long pn = (long)g.panels * g.q;
  long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= pn) return;
  const double* c = g.pd_centre + 4 * (i / g.q);
  double4 s = src[i];
  srcf[i] = make_float4((float)((s.x - c[0]) * kPackScale), (float)((s.y - c[1]) * kPackScale),
                        (float)((s.z - c[2]) * kPackScale), (float)s.w);
}

template <int Q, bool ALL_LEAVES, bool GUARD>
__global__ void __launch_bounds__(32 * kWarpsPerBlock) k_interact32(StepGeom g, const float4* __restrict__ srcf,
                                                                    double* __restrict__ out, long out_stride) {
  using W = WarpShape<Q>;
  __shared__ float4 stage[kWarpsPerBlock][W::STAGE2];
  __shared__ double red[kWarpsPerBlock][3][32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int tp_first = ALL_LEAVES ? g.offset : 0;
  const int tp_count = ALL_LEAVES ? g.leaves : g.panels;
  const int tix = blockIdx.x * kWarpsPerBlock + warp;
  if (tix >= tp_count) return;
  const int t = tp_first + tix;
  const long pn = (long)g.panels * g.q;
  int e0, e1;
  if (ALL_LEAVES) {
    int per = (g.leaves + gridDim.y - 1) / gridDim.y;
    e0 = blockIdx.y * per;
    e1 = min(g.leaves, e0 + per);
  } else {
    e0 = g.tgt_start[t];
    e1 = g.tgt_start[t + 1];
  }
  const double* ct = g.pd_centre + 4 * (long)t;
  const double ctx = ct[0], cty = ct[1], ctz = ct[2];
  const float eps = (float)g.eps;
  if constexpr (Q <= 32) {
    const int h = lane / Q, j = lane % Q;
    const bool active = h < W::S;
    double tx = 0, ty = 0, tz = 0;
    float dtx = 0, dty = 0, dtz = 0;
    if (active) {
      long o = (long)t * Q + j;
      tx = g.px[o];
      ty = g.px[pn + o];
      tz = g.px[2 * pn + o];
      dtx = (float)((tx - ctx) * kPackScale);
      dty = (float)((ty - cty) * kPackScale);
      dtz = (float)((tz - ctz) * kPackScale);
    }
    double ax = 0, ay = 0, az = 0;
    const float2 eps2 = make_float2(eps, eps);
    // each split's panel staged two sources per pair slot, transposed as
    // (x0,x1,y0,y1),(z0,z1,w0,w1); a missing partner (odd q) has zero strength
    float* sl = reinterpret_cast<float*>(&stage[warp][0]) + h * 8 * W::Q2;
    if constexpr (ALL_LEAVES) {
      for (int e = e0; e < e1; e += W::S) {
        int sp = 0;
        if (active && e + h < e1) {
          sp = g.offset + e + h;
          const float4 sv = srcf[(long)sp * Q + j];
          const int k2 = j >> 1, o = j & 1;
          sl[8 * k2 + o] = sv.x;
          sl[8 * k2 + 2 + o] = sv.y;
          sl[8 * k2 + 4 + o] = sv.z;
          sl[8 * k2 + 6 + o] = sv.w;
          if ((Q & 1) && j == Q - 1) {
            sl[8 * k2 + 1] = 0.f;
            sl[8 * k2 + 3] = 0.f;
            sl[8 * k2 + 5] = 0.f;
            sl[8 * k2 + 7] = 0.f;
          }
        }
        __syncwarp();
        if (active && e + h < e1) {
          const double* cs = g.pd_centre + 4 * (long)sp;
          const float b0 = (float)((cs[0] - ctx) * kPackScale) - dtx, b1 = (float)((cs[1] - cty) * kPackScale) - dty,
                      b2 = (float)((cs[2] - ctz) * kPackScale) - dtz;
          const float2 bx = make_float2(b0, b0), by = make_float2(b1, b1), bz = make_float2(b2, b2);
          float2 fx = make_float2(0.f, 0.f), fy = fx, fz = fx;
          const float4* sb = reinterpret_cast<const float4*>(sl);
#pragma unroll
          for (int k2 = 0; k2 < W::Q2; k2++) {
            const float4 A = sb[2 * k2], B = sb[2 * k2 + 1];
            pair32x2<GUARD>(bx, by, bz, make_float2(A.x, A.y), make_float2(A.z, A.w), make_float2(B.x, B.y),
                            make_float2(B.z, B.w), eps2, fx, fy, fz);
          }
          ax += (double)(fx.x + fx.y);
          ay += (double)(fy.x + fy.y);
          az += (double)(fz.x + fz.y);
        }
        __syncwarp();
      }
    } else {
      // The list in batches of 32 entries (g.entry: source panel and its
      // centre's offset from the target's, one entry per lane), handed to the
      // splits by shuffles; the next entry's sources are loaded while the
      // current ones are evaluated.  A source pair is staged by one store per
      // lane: the even node of a pair writes (x0,x1,y0,y1), the odd one
      // (z0,z1,w0,w1), each taking its partner's half by a shuffle.
      const unsigned full = 0xffffffffu;
      float4* st4 = reinterpret_cast<float4*>(sl);
      const bool odd = j & 1, last_odd = (Q & 1) && j == Q - 1;
      const int partner = (odd ? lane - 1 : lane + 1) & 31;
      for (int eb = e0; eb < e1; eb += 32) {
        const int nb = min(32, e1 - eb);
        int4 en = make_int4(0, 0, 0, 0);
        if (lane < nb) en = __ldg(g.entry + eb + lane);
        const int iters = (nb + W::S - 1) / W::S;
        float cbx = __int_as_float(__shfl_sync(full, en.y, h & 31));
        float cby = __int_as_float(__shfl_sync(full, en.z, h & 31));
        float cbz = __int_as_float(__shfl_sync(full, en.w, h & 31));
        float4 sv = make_float4(0.f, 0.f, 0.f, 0.f);
        {
          const int sp = __shfl_sync(full, en.x, h & 31);
          if (active && h < nb) sv = srcf[(long)sp * Q + j];
        }
        for (int it = 0; it < iters; it++) {
          const bool on = active && it * W::S + h < nb;
          const int ns = (it + 1) * W::S + h;
          const int sp_n = __shfl_sync(full, en.x, ns & 31);
          const float nbx = __int_as_float(__shfl_sync(full, en.y, ns & 31));
          const float nby = __int_as_float(__shfl_sync(full, en.z, ns & 31));
          const float nbz = __int_as_float(__shfl_sync(full, en.w, ns & 31));
          float4 sv_n = make_float4(0.f, 0.f, 0.f, 0.f);
          if (active && ns < nb) sv_n = srcf[(long)sp_n * Q + j];
          const float r0 = __shfl_sync(full, odd ? sv.x : sv.z, partner);
          const float r1 = __shfl_sync(full, odd ? sv.y : sv.w, partner);
          if (on) {
            const int k2 = j >> 1;
            if (last_odd) {
              st4[2 * k2] = make_float4(sv.x, 0.f, sv.y, 0.f);
              st4[2 * k2 + 1] = make_float4(sv.z, 0.f, sv.w, 0.f);
            } else if (!odd) {
              st4[2 * k2] = make_float4(sv.x, r0, sv.y, r1);
            } else {
              st4[2 * k2 + 1] = make_float4(r0, sv.z, r1, sv.w);
            }
          }
          __syncwarp();
          if (on) {
            const float b0 = cbx - dtx, b1 = cby - dty, b2 = cbz - dtz;
            const float2 bx = make_float2(b0, b0), by = make_float2(b1, b1), bz = make_float2(b2, b2);
            float2 fx = make_float2(0.f, 0.f), fy = fx, fz = fx;
#pragma unroll
            for (int k2 = 0; k2 < W::Q2; k2++) {
              const float4 A = st4[2 * k2], B = st4[2 * k2 + 1];
              pair32x2<GUARD>(bx, by, bz, make_float2(A.x, A.y), make_float2(A.z, A.w), make_float2(B.x, B.y),
                              make_float2(B.z, B.w), eps2, fx, fy, fz);
            }
            ax += (double)(fx.x + fx.y);
            ay += (double)(fy.x + fy.y);
            az += (double)(fz.x + fz.y);
          }
          __syncwarp();
          sv = sv_n;
          cbx = nbx;
          cby = nby;
          cbz = nbz;
        }
      }
    }
    if (W::S > 1) {
      red[warp][0][lane] = ax;
      red[warp][1][lane] = ay;
      red[warp][2][lane] = az;
      __syncwarp();
      if (h == 0)
        for (int hh = 1; hh < W::S; hh++) {
          ax += red[warp][0][hh * Q + j];
          ay += red[warp][1][hh * Q + j];
          az += red[warp][2][hh * Q + j];
        }
    }
    if (h == 0) {
      long o = ALL_LEAVES ? (long)blockIdx.y * 3 * out_stride + (long)tix * Q + j : (long)t * Q + j;
      long s = ALL_LEAVES ? out_stride : pn;
      out[o] = kBiotSavartPacked * (ty * az - tz * ay);
      out[s + o] = kBiotSavartPacked * (tz * ax - tx * az);
      out[2 * s + o] = kBiotSavartPacked * (tx * ay - ty * ax);
    }
  } else {
    constexpr int TPL = Q <= 32 ? 1 : (Q + 31) / 32;  // target nodes per lane
    double tx[TPL], ty[TPL], tz[TPL], ax[TPL], ay[TPL], az[TPL];
    float dtx[TPL], dty[TPL], dtz[TPL];
#pragma unroll
    for (int r = 0; r < TPL; r++) {
      int j = lane + 32 * r;
      long o = (long)t * Q + (j < Q ? j : 0);
      tx[r] = g.px[o];
      ty[r] = g.px[pn + o];
      tz[r] = g.px[2 * pn + o];
      dtx[r] = (float)((tx[r] - ctx) * kPackScale);
      dty[r] = (float)((ty[r] - cty) * kPackScale);
      dtz[r] = (float)((tz[r] - ctz) * kPackScale);
      ax[r] = ay[r] = az[r] = 0;
    }
    for (int e = e0; e < e1; e++) {
      const int sp = ALL_LEAVES ? g.offset + e : __ldg(g.src_panel + e);
      const long sb = (long)sp * Q;
      for (int k = lane; k < Q; k += 32) stage[warp][k] = srcf[sb + k];
      const double* cs = g.pd_centre + 4 * (long)sp;
      const float bx0 = (float)((cs[0] - ctx) * kPackScale), by0 = (float)((cs[1] - cty) * kPackScale),
                  bz0 = (float)((cs[2] - ctz) * kPackScale);
      float fx[TPL], fy[TPL], fz[TPL], bx[TPL], by[TPL], bz[TPL];
#pragma unroll
      for (int r = 0; r < TPL; r++) {
        fx[r] = fy[r] = fz[r] = 0.f;
        bx[r] = bx0 - dtx[r];
        by[r] = by0 - dty[r];
        bz[r] = bz0 - dtz[r];
      }
      __syncwarp();
      for (int k = 0; k < Q; k++) {
        const float4 s = stage[warp][k];
#pragma unroll
        for (int r = 0; r < TPL; r++) pair32<GUARD>(bx[r], by[r], bz[r], s, eps, fx[r], fy[r], fz[r]);
      }
#pragma unroll
      for (int r = 0; r < TPL; r++) {
        ax[r] += fx[r];
        ay[r] += fy[r];
        az[r] += fz[r];
      }
      __syncwarp();
    }
#pragma unroll
    for (int r = 0; r < TPL; r++) {
      int j = lane + 32 * r;
      if (j >= Q) continue;
      long o = ALL_LEAVES ? (long)blockIdx.y * 3 * out_stride + (long)tix * Q + j : (long)t * Q + j;
      long s = ALL_LEAVES ? out_stride : pn;
      out[o] = kBiotSavartPacked * (ty[r] * az[r] - tz[r] * ay[r]);
      out[s + o] = kBiotSavartPacked * (tz[r] * ax[r] - tx[r] * az[r]);
      out[2 * s + o] = kBiotSavartPacked * (tx[r] * ay[r] - ty[r] * ax[r]);
    }
  }
}

// The list kernel of the reference's default degree 3 (q = 16) in mixed
// precision, two targets per lane: a warp holds one target panel as 4
// source splits x 8 lanes, lane jj of a split owns target nodes jj and
// jj + 8, stages the source pair (2 jj, 2 jj + 1) of its split's panel
// ((x0,x1,y0,y1),(z0,z1,w0,w1), one pair slot per lane) and evaluates the
// split's 16 sources against both targets, so every shared-memory read feeds
// two targets' pairs.  Entries come in batches of 32 (g.entry) handed out by
// shuffles, the next entry's sources are loaded while the current ones are
// evaluated, and the four splits' float64 sums are added in split order.
template <bool GUARD>
__global__ void __launch_bounds__(32 * kWarpsPerBlock) k_interact32_q16(StepGeom g, const float4* __restrict__ srcf,
                                                                        double* __restrict__ out) {
  constexpr int Q = 16, S = 4;
  __shared__ float4 stage[kWarpsPerBlock][S][Q];
  __shared__ double red[kWarpsPerBlock][6][32];
  const unsigned full = 0xffffffffu;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int t = blockIdx.x * kWarpsPerBlock + warp;
  if (t >= g.panels) return;
  const long pn = (long)g.panels * Q;
  const int e0 = g.tgt_start[t], e1 = g.tgt_start[t + 1];
  const int h = lane >> 3, jj = lane & 7;
  const double* ct = g.pd_centre + 4 * (long)t;
  float dtx[2], dty[2], dtz[2];
#pragma unroll
  for (int r = 0; r < 2; r++) {
    const long o = (long)t * Q + jj + 8 * r;
    dtx[r] = (float)((g.px[o] - ct[0]) * kPackScale);
    dty[r] = (float)((g.px[pn + o] - ct[1]) * kPackScale);
    dtz[r] = (float)((g.px[2 * pn + o] - ct[2]) * kPackScale);
  }
  double ax[2] = {0, 0}, ay[2] = {0, 0}, az[2] = {0, 0};
  const float feps = (float)g.eps;
  const float2 eps2 = make_float2(feps, feps);
  float4* tile = stage[warp][h];
  for (int eb = e0; eb < e1; eb += 32) {
    const int nb = min(32, e1 - eb);
    int4 en = make_int4(0, 0, 0, 0);
    if (lane < nb) en = __ldg(g.entry + eb + lane);
    const int iters = (nb + S - 1) / S;
    float cbx = __int_as_float(__shfl_sync(full, en.y, h));
    float cby = __int_as_float(__shfl_sync(full, en.z, h));
    float cbz = __int_as_float(__shfl_sync(full, en.w, h));
    float4 s0 = make_float4(0.f, 0.f, 0.f, 0.f), s1 = s0;
    {
      const int sp = __shfl_sync(full, en.x, h);
      if (h < nb) {
        s0 = srcf[(long)sp * Q + 2 * jj];
        s1 = srcf[(long)sp * Q + 2 * jj + 1];
      }
    }
    for (int it = 0; it < iters; it++) {
      const bool on = it * S + h < nb;
      const int ns = (it + 1) * S + h;
      const int sp_n = __shfl_sync(full, en.x, ns & 31);
      const float nbx = __int_as_float(__shfl_sync(full, en.y, ns & 31));
      const float nby = __int_as_float(__shfl_sync(full, en.z, ns & 31));
      const float nbz = __int_as_float(__shfl_sync(full, en.w, ns & 31));
      float4 n0 = make_float4(0.f, 0.f, 0.f, 0.f), n1 = n0;
      if (ns < nb) {
        n0 = srcf[(long)sp_n * Q + 2 * jj];
        n1 = srcf[(long)sp_n * Q + 2 * jj + 1];
      }
      if (on) {
        tile[2 * jj] = make_float4(s0.x, s1.x, s0.y, s1.y);
        tile[2 * jj + 1] = make_float4(s0.z, s1.z, s0.w, s1.w);
      }
      __syncwarp();
      if (on) {
        float2 bx[2], by[2], bz[2], fx[2], fy[2], fz[2];
#pragma unroll
        for (int r = 0; r < 2; r++) {
          const float b0 = cbx - dtx[r], b1 = cby - dty[r], b2 = cbz - dtz[r];
          bx[r] = make_float2(b0, b0);
          by[r] = make_float2(b1, b1);
          bz[r] = make_float2(b2, b2);
          fx[r] = fy[r] = fz[r] = make_float2(0.f, 0.f);
        }
#pragma unroll
        for (int k2 = 0; k2 < Q / 2; k2++) {
          const float4 A = tile[2 * k2], B = tile[2 * k2 + 1];
          const float2 sx = make_float2(A.x, A.y), sy = make_float2(A.z, A.w), sz = make_float2(B.x, B.y),
                       sw = make_float2(B.z, B.w);
#pragma unroll
          for (int r = 0; r < 2; r++) pair32x2<GUARD>(bx[r], by[r], bz[r], sx, sy, sz, sw, eps2, fx[r], fy[r], fz[r]);
        }
#pragma unroll
        for (int r = 0; r < 2; r++) {
          ax[r] += (double)(fx[r].x + fx[r].y);
          ay[r] += (double)(fy[r].x + fy[r].y);
          az[r] += (double)(fz[r].x + fz[r].y);
        }
      }
      __syncwarp();
      s0 = n0;
      s1 = n1;
      cbx = nbx;
      cby = nby;
      cbz = nbz;
    }
  }
#pragma unroll
  for (int r = 0; r < 2; r++) {
    red[warp][3 * r][lane] = ax[r];
    red[warp][3 * r + 1][lane] = ay[r];
    red[warp][3 * r + 2][lane] = az[r];
  }
  __syncwarp();
  if (h == 0) {
#pragma unroll
    for (int r = 0; r < 2; r++) {
      double sx = ax[r], sy = ay[r], sz = az[r];
      for (int hh = 1; hh < S; hh++) {
        sx += red[warp][3 * r][hh * 8 + jj];
        sy += red[warp][3 * r + 1][hh * 8 + jj];
        sz += red[warp][3 * r + 2][hh * 8 + jj];
      }
      const long o = (long)t * Q + jj + 8 * r;
      const double tx = g.px[o], ty = g.px[pn + o], tz = g.px[2 * pn + o];
      out[o] = kBiotSavartPacked * (ty * sz - tz * sy);
      out[pn + o] = kBiotSavartPacked * (tz * sx - tx * sz);
      out[2 * pn + o] = kBiotSavartPacked * (tx * sy - ty * sx);
    }
  }
}

// Wide panels (q > 32, e.g. 81 treecode proxies): one CTA of four warps per
// target panel; the warps take every fourth source panel, each lane owns
// ceil(q/32) target nodes, and the four partial sums are added in warp order
// (deterministic).  MIXED: float32 pairs on packed sources (kPackScale),
// per-source-panel float32 sums added into float64.
template <int Q, bool ALL_LEAVES, bool GUARD, bool MIXED>
__device__ __forceinline__ void interact_wide_body(const StepGeom& g, int tix, int gy, int ngy,
                                                   const double4* __restrict__ src, const float4* __restrict__ srcf,
                                                   double* __restrict__ out, long out_stride) {
  constexpr int TPL = (Q + 31) / 32, NW = 4, Q2 = (Q + 1) / 2;
  using Src = typename std::conditional<MIXED, float4, double4>::type;
  // MIXED: sources staged two at a time, transposed, (x0,x1,y0,y1),(z0,z1,w0,w1)
  __shared__ Src stage[NW][MIXED ? 2 * Q2 : Q];
  __shared__ double red[NW][3][Q];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int t = (ALL_LEAVES ? g.offset : 0) + tix;
  const long pn = (long)g.panels * g.q;
  int e0, e1;
  if (ALL_LEAVES) {
    int per = (g.leaves + ngy - 1) / ngy;
    e0 = gy * per;
    e1 = min(g.leaves, e0 + per);
  } else {
    e0 = g.tgt_start[t];
    e1 = g.tgt_start[t + 1];
  }
  const double* ct = g.pd_centre + 4 * (long)t;
  const double ctx = ct[0], cty = ct[1], ctz = ct[2];
  double tx[TPL], ty[TPL], tz[TPL], ax[TPL], ay[TPL], az[TPL];
  float dtx[TPL], dty[TPL], dtz[TPL];
#pragma unroll
  for (int r = 0; r < TPL; r++) {
    int j = lane + 32 * r;
    long o = (long)t * Q + (j < Q ? j : 0);
    tx[r] = g.px[o];
    ty[r] = g.px[pn + o];
    tz[r] = g.px[2 * pn + o];
    dtx[r] = (float)((tx[r] - ctx) * kPackScale);
    dty[r] = (float)((ty[r] - cty) * kPackScale);
    dtz[r] = (float)((tz[r] - ctz) * kPackScale);
    ax[r] = ay[r] = az[r] = 0;
  }
  const float feps = (float)g.eps;
  for (int e = e0 + warp; e < e1; e += NW) {
    const int sp = ALL_LEAVES ? g.offset + e : __ldg(g.src_panel + e);
    const long sb = (long)sp * Q;
    if constexpr (MIXED) {
      for (int k2 = lane; k2 < Q2; k2 += 32) {
        const float4 s0 = srcf[sb + 2 * k2];
        const float4 s1 = (2 * k2 + 1 < Q) ? srcf[sb + 2 * k2 + 1] : make_float4(0.f, 0.f, 0.f, 0.f);
        stage[warp][2 * k2] = make_float4(s0.x, s1.x, s0.y, s1.y);
        stage[warp][2 * k2 + 1] = make_float4(s0.z, s1.z, s0.w, s1.w);
      }
    } else {
      for (int k = lane; k < Q; k += 32) stage[warp][k] = src[sb + k];
    }
    __syncwarp();
    if constexpr (MIXED) {
      const double* cs = g.pd_centre + 4 * (long)sp;
      const float bx0 = (float)((cs[0] - ctx) * kPackScale), by0 = (float)((cs[1] - cty) * kPackScale),
                  bz0 = (float)((cs[2] - ctz) * kPackScale);
      const float2 eps2 = make_float2(feps, feps);
      float2 fx[TPL], fy[TPL], fz[TPL], bx[TPL], by[TPL], bz[TPL];
#pragma unroll
      for (int r = 0; r < TPL; r++) {
        fx[r] = fy[r] = fz[r] = make_float2(0.f, 0.f);
        const float b0 = bx0 - dtx[r], b1 = by0 - dty[r], b2 = bz0 - dtz[r];
        bx[r] = make_float2(b0, b0);
        by[r] = make_float2(b1, b1);
        bz[r] = make_float2(b2, b2);
      }
#pragma unroll 3
      for (int k2 = 0; k2 < Q2; k2++) {
        const float4 A = stage[warp][2 * k2], B = stage[warp][2 * k2 + 1];
        const float2 sx = make_float2(A.x, A.y), sy = make_float2(A.z, A.w), sz = make_float2(B.x, B.y),
                     sw = make_float2(B.z, B.w);
#pragma unroll
        for (int r = 0; r < TPL; r++)
          pair32x2<GUARD>(bx[r], by[r], bz[r], sx, sy, sz, sw, eps2, fx[r], fy[r], fz[r]);
      }
#pragma unroll
      for (int r = 0; r < TPL; r++) {
        ax[r] += (double)fx[r].x + (double)fx[r].y;
        ay[r] += (double)fy[r].x + (double)fy[r].y;
        az[r] += (double)fz[r].x + (double)fz[r].y;
      }
    } else {
#pragma unroll 3
      for (int k = 0; k < Q; k++) {
        const double4 s = stage[warp][k];
#pragma unroll
        for (int r = 0; r < TPL; r++) pair64<GUARD>(tx[r], ty[r], tz[r], s, g.eps, ax[r], ay[r], az[r]);
      }
    }
    __syncwarp();
  }
#pragma unroll
  for (int r = 0; r < TPL; r++) {
    int j = lane + 32 * r;
    if (j < Q) {
      red[warp][0][j] = ax[r];
      red[warp][1][j] = ay[r];
      red[warp][2][j] = az[r];
    }
  }
  __syncthreads();
  const double cb = MIXED ? kBiotSavartPacked : kBiotSavart;
  for (int j = threadIdx.x; j < Q; j += blockDim.x) {
    double sx = red[0][0][j], sy = red[0][1][j], sz = red[0][2][j];
    for (int w = 1; w < NW; w++) {
      sx += red[w][0][j];
      sy += red[w][1][j];
      sz += red[w][2][j];
    }
    long o = (long)t * Q + j;
    const double px = g.px[o], py = g.px[pn + o], pz = g.px[2 * pn + o];
    long oo = ALL_LEAVES ? (long)gy * 3 * out_stride + (long)tix * Q + j : o;
    long st = ALL_LEAVES ? out_stride : pn;
    out[oo] = cb * (py * sz - pz * sy);
    out[st + oo] = cb * (pz * sx - px * sz);
    out[2 * st + oo] = cb * (px * sy - py * sx);
  }
}

template <int Q, bool ALL_LEAVES, bool GUARD, bool MIXED>
__global__ void __launch_bounds__(128) k_interact_wide(StepGeom g, const double4* __restrict__ src,
                                                       const float4* __restrict__ srcf, double* __restrict__ out,
                                                       long out_stride) {
  interact_wide_body<Q, ALL_LEAVES, GUARD, MIXED>(g, blockIdx.x, blockIdx.y, gridDim.y, src, srcf, out, out_stride);
}

// Batched treecode members with q = Q: member idx[blockIdx.z], well-separated pairs.
template <int Q, bool GUARD, bool MIXED>
__global__ void __launch_bounds__(128) k_interact_wide_batch(const BatchMember* __restrict__ mem,
                                                             const int* __restrict__ idx) {
  const BatchMember& m = mem[idx[blockIdx.z]];
  const StepGeom g = m.fg;
  interact_wide_body<Q, false, GUARD, MIXED>(g, blockIdx.x, 0, 1, m.fsrc, g.srcf, m.ftgt, 0);
}

// Sum of per-group partials (group gi at partial + gi * gstride) in group order.
__global__ void k_reduce_groups(const double* __restrict__ partial, int groups, long n, long gstride,
                                double* __restrict__ out) {
  long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double a = 0;
  for (int gi = 0; gi < groups; gi++) a += partial[(long)gi * gstride + i];
  out[i] = a;
}

// ---------------------------------------------------------------------------
// Departure points and remap.
//
// bve_find_departure_points (src/bve_time_step.cpp:172-309): backward RK4
// with k1 = v3 at x, k2 = v2 at proj(x - dt/2 k1), k3 = v1 at
// proj(x - dt/2 k2), k4 = v0 at proj(x - dt k3), and the re-projected
// combination.  bve_departure_to_target (src/bve_time_step.cpp:15-67):
// new vorticity = BLI(vor)(dep) + 2 Omega dep_z - 2 Omega z, tracers by BLI.
// mode bit 1: compute departure points (else read dep); bit 2: remap (else
// write dep).  The locations use locate_basis_rcp (one division per
// direction of the barycentric basis, reciprocals in the projections): the
// kernel is bound by float64 division and atan latency, not by its 136 bytes
// of traffic per particle.

template <int D>
__device__ __forceinline__ void depart_remap_body(const StepGeom& g, const BliTable& tab, long o,
                                                  const double* __restrict__ x, const double* __restrict__ y,
                                                  const double* __restrict__ z, const double* __restrict__ v0,
                                                  const double* __restrict__ v1, const double* __restrict__ v2,
                                                  const double* __restrict__ v3, double dt, double* __restrict__ dep,
                                                  const double* __restrict__ vors, const double* __restrict__ tracers,
                                                  int T, double* __restrict__ new_vors,
                                                  double* __restrict__ new_tracers, int mode) {
  const long n = (long)g.leaves * g.q;
  unsigned err = 0;
  Basis<D> b;
  double dx, dy, dz;
  if (mode & 1) {
    const double x0 = x[o], y0 = y[o], z0 = z[o];
    const double k1x = v3[o], k1y = v3[n + o], k1z = v3[2 * n + o];
    double xx = x0 - 0.5 * dt * k1x, yy = y0 - 0.5 * dt * k1y, zz = z0 - 0.5 * dt * k1z;
    project_to_sphere_rcp(xx, yy, zz);
    locate_basis_rcp<D>(g, tab, xx, yy, zz, b, err);
    double k2x, k2y, k2z;
    gather3<D>(b, v2, n, k2x, k2y, k2z);
    xx = x0 - 0.5 * dt * k2x, yy = y0 - 0.5 * dt * k2y, zz = z0 - 0.5 * dt * k2z;
    project_to_sphere_rcp(xx, yy, zz);
    locate_basis_rcp<D>(g, tab, xx, yy, zz, b, err);
    double k3x, k3y, k3z;
    gather3<D>(b, v1, n, k3x, k3y, k3z);
    xx = x0 - dt * k3x, yy = y0 - dt * k3y, zz = z0 - dt * k3z;
    project_to_sphere_rcp(xx, yy, zz);
    locate_basis_rcp<D>(g, tab, xx, yy, zz, b, err);
    double k4x, k4y, k4z;
    gather3<D>(b, v0, n, k4x, k4y, k4z);
    xx = x0 - 1.0 / 6.0 * dt * k1x, yy = y0 - 1.0 / 6.0 * dt * k1y, zz = z0 - 1.0 / 6.0 * dt * k1z;
    project_to_sphere_rcp(xx, yy, zz);
    xx -= -1.0 / 3.0 * dt * k2x, yy -= -1.0 / 3.0 * dt * k2y, zz -= -1.0 / 3.0 * dt * k2z;
    project_to_sphere_rcp(xx, yy, zz);
    xx -= -1.0 / 3.0 * dt * k3x, yy -= -1.0 / 3.0 * dt * k3y, zz -= -1.0 / 3.0 * dt * k3z;
    project_to_sphere_rcp(xx, yy, zz);
    xx -= -1.0 / 6.0 * dt * k4x, yy -= -1.0 / 6.0 * dt * k4y, zz -= -1.0 / 6.0 * dt * k4z;
    project_to_sphere_rcp(xx, yy, zz);
    dx = xx;
    dy = yy;
    dz = zz;
    if (!(mode & 2)) {
      dep[o] = dx;
      dep[n + o] = dy;
      dep[2 * n + o] = dz;
    }
  } else {
    dx = dep[o];
    dy = dep[n + o];
    dz = dep[2 * n + o];
  }
  if (mode & 2) {
    locate_basis_rcp<D>(g, tab, dx, dy, dz, b, err);
    double vor = gather<D>(b, vors);
    for (int k = 0; k < T; k++) new_tracers[o * T + k] = gather<D>(b, tracers, T, k);
    vor += 2 * g.omega * dz;
    new_vors[o] = vor - 2 * g.omega * z[o];
  }
  flag(g.err, err);
}

// 128 threads held to 64 registers (eight blocks per SM; a few bytes spill):
// the chain of four locate -> gather rounds per particle is latency-bound,
// and the extra resident warps measured 9 us per launch faster at 393,216
// particles (78 vs 87 us) than the 76-register build.
template <int D>
__global__ void __launch_bounds__(128, 8) k_depart_remap(StepGeom g, BliTable tab, const double* __restrict__ x, const double* __restrict__ y,
                               const double* __restrict__ z, const double* __restrict__ v0,
                               const double* __restrict__ v1, const double* __restrict__ v2,
                               const double* __restrict__ v3, double dt, double* __restrict__ dep,
                               const double* __restrict__ vors, const double* __restrict__ tracers, int T,
                               double* __restrict__ new_vors, double* __restrict__ new_tracers, int mode) {
  const long o = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (o >= (long)g.leaves * g.q) return;
  depart_remap_body<D>(g, tab, o, x, y, z, v0, v1, v2, v3, dt, dep, vors, tracers, T, new_vors, new_tracers, mode);
}

// Batched members on one particle grid (member blockIdx.y): departure and
// remap in one pass (mode 3), stage velocities v_k + m * 3n, vorticity + m * n.
template <int D>
__global__ void k_depart_remap_batch(StepGeom g, BliTable tab, const double* __restrict__ x,
                                     const double* __restrict__ y, const double* __restrict__ z,
                                     const double* __restrict__ v0, const double* __restrict__ v1,
                                     const double* __restrict__ v2, const double* __restrict__ v3, double dt,
                                     const double* __restrict__ vors, double* __restrict__ new_vors) {
  const long n = (long)g.leaves * g.q;
  const long o = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (o >= n) return;
  const long m = blockIdx.y, vo = m * 3 * n, so = m * n;
  depart_remap_body<D>(g, tab, o, x, y, z, v0 + vo, v1 + vo, v2 + vo, v3 + vo, dt, nullptr, vors + so, nullptr, 0,
                       new_vors + so, nullptr, 3);
}

// ---------------------------------------------------------------------------
// Stand-alone direct sums over arbitrary points: blocks own 128 targets and
// stage 128 sources at a time in shared memory; gridDim.y source groups write
// partials reduced by k_reduce_groups.

constexpr int kDirectThreads = 128;

__global__ void __launch_bounds__(kDirectThreads)
    k_direct_bve64(long nt, const double* __restrict__ tx, const double* __restrict__ ty,
                   const double* __restrict__ tz, long ns, const double* __restrict__ sx,
                   const double* __restrict__ sy, const double* __restrict__ sz, const double* __restrict__ sw,
                   double eps, double* __restrict__ partial) {
  __shared__ double4 tile[kDirectThreads];
  long i = blockIdx.x * (long)kDirectThreads + threadIdx.x;
  double x = 0, y = 0, z = 0;
  if (i < nt) {
    x = tx[i];
    y = ty[i];
    z = tz[i];
  }
  long per = (ns + gridDim.y - 1) / gridDim.y;
  long s0 = blockIdx.y * per, s1 = min(ns, s0 + per);
  double ax = 0, ay = 0, az = 0;
  for (long b = s0; b < s1; b += kDirectThreads) {
    long k = b + threadIdx.x;
    tile[threadIdx.x] = k < s1 ? make_double4(sx[k], sy[k], sz[k], sw[k]) : make_double4(0, 0, 0, 0);
    __syncthreads();
    int cnt = (int)min((long)kDirectThreads, s1 - b);
    for (int m = 0; m < cnt; m++) pair64<true>(x, y, z, tile[m], eps, ax, ay, az);
    __syncthreads();
  }
  if (i < nt) {
    long o = (long)blockIdx.y * 3 * nt + i;
    partial[o] = kBiotSavart * (y * az - z * ay);
    partial[nt + o] = kBiotSavart * (z * ax - x * az);
    partial[2 * nt + o] = kBiotSavart * (x * ay - y * ax);
  }
}

// Mixed: each block measures both tiles relative to their first point (in
// float64), so float32 carries only the small in-tile offsets.
__global__ void __launch_bounds__(kDirectThreads)
    k_direct_bve32(long nt, const double* __restrict__ tx, const double* __restrict__ ty,
                   const double* __restrict__ tz, long ns, const double* __restrict__ sx,
                   const double* __restrict__ sy, const double* __restrict__ sz, const double* __restrict__ sw,
                   double eps, double* __restrict__ partial) {
  __shared__ float4 tile[kDirectThreads];
  long i = blockIdx.x * (long)kDirectThreads + threadIdx.x;
  long i0 = blockIdx.x * (long)kDirectThreads;
  const double tcx = tx[i0], tcy = ty[i0], tcz = tz[i0];
  double x = tcx, y = tcy, z = tcz;
  if (i < nt) {
    x = tx[i];
    y = ty[i];
    z = tz[i];
  }
  const float dtx = (float)((x - tcx) * kPackScale), dty = (float)((y - tcy) * kPackScale),
              dtz = (float)((z - tcz) * kPackScale);
  long per = (ns + gridDim.y - 1) / gridDim.y;
  long s0 = blockIdx.y * per, s1 = min(ns, s0 + per);
  double ax = 0, ay = 0, az = 0;
  const float feps = (float)eps;
  for (long b = s0; b < s1; b += kDirectThreads) {
    const double scx = sx[b], scy = sy[b], scz = sz[b];
    long k = b + threadIdx.x;
    tile[threadIdx.x] = k < s1 ? make_float4((float)((sx[k] - scx) * kPackScale), (float)((sy[k] - scy) * kPackScale),
                                             (float)((sz[k] - scz) * kPackScale), (float)sw[k])
                               : make_float4(0, 0, 0, 0);
    __syncthreads();
    float bx = (float)((scx - tcx) * kPackScale) - dtx, by = (float)((scy - tcy) * kPackScale) - dty,
          bz = (float)((scz - tcz) * kPackScale) - dtz;
    float fx = 0, fy = 0, fz = 0;
    int cnt = (int)min((long)kDirectThreads, s1 - b);
    for (int m = 0; m < cnt; m++) pair32<true>(bx, by, bz, tile[m], feps, fx, fy, fz);
    ax += fx;
    ay += fy;
    az += fz;
    __syncthreads();
  }
  if (i < nt) {
    long o = (long)blockIdx.y * 3 * nt + i;
    partial[o] = kBiotSavartPacked * (y * az - z * ay);
    partial[nt + o] = kBiotSavartPacked * (z * ax - x * az);
    partial[2 * nt + o] = kBiotSavartPacked * (x * ay - y * ax);
  }
}

// inv_lap (src/direct_sum_impl.hpp:20-27): soln_i += sum_{j != i}
// -1/(4 pi) log(1 - x_i.x_j) area_j pots_j.
__global__ void __launch_bounds__(kDirectThreads)
    k_inv_lap(long n, const double* __restrict__ x, const double* __restrict__ y, const double* __restrict__ z,
              const double* __restrict__ area, const double* __restrict__ pots, double* __restrict__ soln) {
  __shared__ double4 tile[kDirectThreads];
  long i = blockIdx.x * (long)kDirectThreads + threadIdx.x;
  double xi = 0, yi = 0, zi = 0;
  if (i < n) {
    xi = x[i];
    yi = y[i];
    zi = z[i];
  }
  double acc = 0;
  for (long b = 0; b < n; b += kDirectThreads) {
    long k = b + threadIdx.x;
    tile[threadIdx.x] = k < n ? make_double4(x[k], y[k], z[k], area[k] * pots[k]) : make_double4(0, 0, 0, 0);
    __syncthreads();
    int cnt = (int)min((long)kDirectThreads, n - b);
    for (int m = 0; m < cnt; m++) {
      if (b + m == i) continue;
      double4 s = tile[m];
      double dp = xi * s.x + yi * s.y + zi * s.z;
      acc += -0.07957747154594767 * log(1 - dp) * s.w;
    }
    __syncthreads();
  }
  if (i < n) soln[i] += acc;
}

// The forcing of bve_ssw_forcing (type 1) / bve_ssw_forcing_2 (type 2),
// src/forcing_funcs.cpp:6-80: one thread per leaf panel walking its points
// in order as the reference's functor does, so that bcomp carries over from
// the panel's previous point where lat <= 0 (the reference sets it only for
// lat > 0).  force = 0.6 omega a b cos(lon) (type 1) or 1.2 omega a b
// cos(2 lon) (type 2), added to the vorticity by the source kernels.
__global__ void k_ssw_forcing(int leaves, int q, int type, double omega, const double* __restrict__ time,
                              const double* __restrict__ x, const double* __restrict__ y,
                              const double* __restrict__ z, double* __restrict__ force) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= leaves) return;
  const double t = *time, Tp = 4.0, Tf = 4.0 + 11.0, theta1 = kPi / 3.0;
  double acomp, bcomp = 0;
  if (t / 86400.0 < Tp) acomp = 0.5 * (1.0 - cos(kPi * (t / 86400.0) / Tp));
  else if (t / 86400.0 < Tf - Tp) acomp = 1.0;
  else if (t / 86400.0 < Tf) acomp = 0.5 * (1.0 - cos(kPi + kPi * ((t / 86400.0) - Tf + Tp) / Tp));
  else acomp = 0.0;
  for (int j = 0; j < q; j++) {
    const long o = (long)i * q + j;
    const double xx = x[o], yy = y[o], zz = z[o];
    // xyz_to_latlon, src/general_utils_impl.hpp:230-235
    const double lat = kPi / 2.0 - atan2(sqrt(xx * xx + yy * yy), zz), lon = atan2(yy, xx);
    if (lat > 0) {
      const double tt = tan(theta1), tl = tan(lat);
      const double ccomp = (tt * tt) / (tl * tl);
      bcomp = ccomp * exp(1.0 - ccomp);
    }
    force[o] = type == 1 ? 0.6 * omega * acomp * bcomp * cos(lon) : 1.2 * omega * acomp * bcomp * cos(2.0 * lon);
  }
}

__global__ void k_time_advance(double* time, double dt) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *time += dt;
}

}  // namespace

// ---------------------------------------------------------------------------
// Launch wrappers.

using dev::blocks_for;

void launch_leaf_sources(const StepGeom& g, int stage, double dt_s, const double* vprev, const double* x,
                         const double* y, const double* z, const double* vors, const double* area, double4* src,
                         cudaStream_t st) {
  long n = (long)g.leaves * g.q;
  SB_LAUNCH(k_leaf_sources, blocks_for(n, 256), 256, 0, st, g, stage, dt_s, vprev, x, y, z, vors, area, src);
}

void launch_sources_from_disp(const StepGeom& g, const double* dx, const double* dy, const double* dz,
                              const double* s, double4* src, cudaStream_t st) {
  long n = (long)g.panels * g.q;
  SB_LAUNCH(k_sources_from_disp, blocks_for(n, 256), 256, 0, st, g, dx, dy, dz, s, src);
}

void launch_copy_strength(const StepGeom& g, const double4* src, double* out, cudaStream_t st) {
  long n = (long)g.panels * g.q;
  SB_LAUNCH(k_copy_strength, blocks_for(n, 256), 256, 0, st, g, src, out);
}

// Subtree depth per launch: three levels (85 panels) for small q, one level
// for large q so that a pass has enough CTAs; shared memory holds the levels
// plus one scratch level.
static int subtree_depth(int q) { return q <= 25 ? 3 : 1; }

static size_t subtree_smem(int q, int fields, int D) {
  return (size_t)q * fields * 8 * ((((1L << (2 * (D + 1))) - 1) / 3) + (1L << (2 * D)));
}

void launch_upward_fused(const StepGeom& g, int mode, int stage, double dt_s, const double* vprev, const double* x,
                         const double* y, const double* z, const double* vors, const double* area, double4* src,
                         bool mixed, cudaStream_t st) {
  static std::atomic<unsigned long long> attr{0};
  raise_smem_once(attr, 164 * 1024, k_upward_subtree);
  const int Dmax = subtree_depth(g.q);
  int r = g.levels - 1;  // the bottom of the next subtree
  const long nl = (long)g.offset * g.q;  // non-leaf proxy points
  const bool flat = mode == 0 && nl > 0;
  if (flat) {
    if (g.q == 16) SB_LAUNCH(k_nonleaf_positions<16>, blocks_for(nl, 256), 256, 0, st, g, stage, dt_s, vprev, src);
    else SB_LAUNCH(k_nonleaf_positions<0>, blocks_for(nl, 256), 256, 0, st, g, stage, dt_s, vprev, src);
  }
  bool first = true;
  while (first || r > 0) {
    int D = first ? (r < Dmax ? r : Dmax) : (r < Dmax ? r : Dmax);
    int root = r - D;
    SB_LAUNCH(k_upward_subtree, (unsigned)(6 << (2 * root)), 256, subtree_smem(g.q, 1, D), st, g, root, D, mode,
              flat ? 0 : 1, stage, dt_s, vprev, x, y, z, vors, area, src, mixed ? 1 : 0);
    r = root;
    first = false;
  }
}

void launch_upward_batch(const BatchMember* mem, int members, int levels, int qmax, bool mixed, cudaStream_t st) {
  static std::atomic<unsigned long long> attr{0};
  raise_smem_once(attr, 164 * 1024, k_upward_subtree_batch);
  const int Dmax = subtree_depth(qmax);
  int r = levels - 1;
  do {
    const int D = r < Dmax ? r : Dmax;
    const int root = r - D;
    SB_LAUNCH(k_upward_subtree_batch, dim3((unsigned)(6 << (2 * root)), 1, (unsigned)members), 256,
              subtree_smem(qmax, 1, D), st, mem, root, D, mixed ? 1 : 0);
    r = root;
  } while (r > 0);
}

void launch_downward_batch(const BatchMember* mem, int members, int levels, int qmax, cudaStream_t st) {
  static std::atomic<unsigned long long> attr{0};
  raise_smem_once(attr, 164 * 1024, k_downward_subtree_batch);
  const int Dmax = subtree_depth(qmax);
  int r = 0;
  while (r < levels - 1) {
    const int D = (levels - 1 - r) < Dmax ? (levels - 1 - r) : Dmax;
    SB_LAUNCH(k_downward_subtree_batch, dim3((unsigned)(6 << (2 * r)), 1, (unsigned)members), 256,
              subtree_smem(qmax, 3, D), st, mem, r, D);
    r += D;
  }
}

void launch_cc_batch(const BatchMember* mem, const int* idx, int count, int q, int tree_panels, double eps,
                     int precision, cudaStream_t st) {
  if (count <= 0) return;
  const dim3 grid((unsigned)tree_panels, 1, (unsigned)count);
  const bool mixed = precision == SBSLPM_MIXED, guard = !(eps > 0);
#define SB_CCB(Q)                                                                                              \
  case Q:                                                                                                      \
    if (mixed) {                                                                                               \
      if (guard) SB_LAUNCH((k_interact_wide_batch<Q, true, true>), grid, 128, 0, st, mem, idx);                \
      else SB_LAUNCH((k_interact_wide_batch<Q, false, true>), grid, 128, 0, st, mem, idx);                     \
    } else {                                                                                                   \
      if (guard) SB_LAUNCH((k_interact_wide_batch<Q, true, false>), grid, 128, 0, st, mem, idx);               \
      else SB_LAUNCH((k_interact_wide_batch<Q, false, false>), grid, 128, 0, st, mem, idx);                    \
    }                                                                                                          \
    break;
  switch (q) {
    SB_CCB(36) SB_CCB(49) SB_CCB(64) SB_CCB(81) SB_CCB(100) SB_CCB(121)
  }
#undef SB_CCB
}

void launch_downward_fused(const StepGeom& g, double* tgt, double* leaf_out, cudaStream_t st) {
  static std::atomic<unsigned long long> attr{0};
  raise_smem_once(attr, 164 * 1024, k_downward_subtree);
  const int Dmax = subtree_depth(g.q);
  int r = 0;
  while (r < g.levels - 1) {
    int D = (g.levels - 1 - r) < Dmax ? (g.levels - 1 - r) : Dmax;
    SB_LAUNCH(k_downward_subtree, (unsigned)(6 << (2 * r)), 256, subtree_smem(g.q, 3, D), st, g, r, D, tgt,
              leaf_out);
    r += D;
  }
}

namespace {
template <int Q, bool GUARD>
void interact_qg(const StepGeom& g, int precision, const double4* src, double* out, bool all_leaves, int groups,
                 long out_stride, cudaStream_t st, bool pack) {
  int tp = all_leaves ? g.leaves : g.panels;
  if constexpr (Q > 32) {
    dim3 wgrid((unsigned)tp, all_leaves ? groups : 1);
    const bool mixed = precision == SBSLPM_MIXED;
    if (mixed && pack) {
      long pn = (long)g.panels * g.q;
      SB_LAUNCH(k_pack_mixed, blocks_for(pn, 256), 256, 0, st, g, src, g.srcf);
    }
    if (mixed) {
      if (all_leaves) SB_LAUNCH((k_interact_wide<Q, true, GUARD, true>), wgrid, 128, 0, st, g, src, g.srcf, out, out_stride);
      else SB_LAUNCH((k_interact_wide<Q, false, GUARD, true>), wgrid, 128, 0, st, g, src, g.srcf, out, out_stride);
    } else {
      if (all_leaves) SB_LAUNCH((k_interact_wide<Q, true, GUARD, false>), wgrid, 128, 0, st, g, src, g.srcf, out, out_stride);
      else SB_LAUNCH((k_interact_wide<Q, false, GUARD, false>), wgrid, 128, 0, st, g, src, g.srcf, out, out_stride);
    }
    return;
  }
  dim3 grid(blocks_for(tp, kWarpsPerBlock), all_leaves ? groups : 1);
  if (precision == SBSLPM_MIXED) {
    long pn = (long)g.panels * g.q;
    if (pack) SB_LAUNCH(k_pack_mixed, blocks_for(pn, 256), 256, 0, st, g, src, g.srcf);
    if (all_leaves)
      SB_LAUNCH((k_interact32<Q, true, GUARD>), grid, 32 * kWarpsPerBlock, 0, st, g, g.srcf, out, out_stride);
    else if constexpr (Q == 16)
      SB_LAUNCH((k_interact32_q16<GUARD>), grid, 32 * kWarpsPerBlock, 0, st, g, g.srcf, out);
    else
      SB_LAUNCH((k_interact32<Q, false, GUARD>), grid, 32 * kWarpsPerBlock, 0, st, g, g.srcf, out, out_stride);
    return;
  }
  if (all_leaves)
    SB_LAUNCH((k_interact64<Q, true, GUARD>), grid, 32 * kWarpsPerBlock, 0, st, g, src, out, out_stride);
  else
    SB_LAUNCH((k_interact64<Q, false, GUARD>), grid, 32 * kWarpsPerBlock, 0, st, g, src, out, out_stride);
}

// The coincident-point guard is compiled in only when kernel_eps = 0.
template <int Q>
void interact_q(const StepGeom& g, int precision, const double4* src, double* out, bool, bool all_leaves,
                int groups, long out_stride, cudaStream_t st, bool pack = true) {
  if (g.eps > 0)
    interact_qg<Q, false>(g, precision, src, out, all_leaves, groups, out_stride, st, pack);
  else
    interact_qg<Q, true>(g, precision, src, out, all_leaves, groups, out_stride, st, pack);
}

void interact_dispatch(const StepGeom& g, int precision, const double4* src, double* out, bool accumulate,
                       bool all_leaves, int groups, long out_stride, cudaStream_t st, bool pack = true) {
#define SB_IQ(Q) \
  case Q: interact_q<Q>(g, precision, src, out, accumulate, all_leaves, groups, out_stride, st, pack); break;
  switch (g.q) {
    SB_IQ(1) SB_IQ(4) SB_IQ(9) SB_IQ(16) SB_IQ(25) SB_IQ(36) SB_IQ(49) SB_IQ(64) SB_IQ(81) SB_IQ(100)
    default: interact_q<121>(g, precision, src, out, accumulate, all_leaves, groups, out_stride, st, pack); break;
  }
#undef SB_IQ
}

// Independent FMA chains (8 per thread) so the pipe, not latency, limits throughput.
__global__ void k_fma_probe32(int iters, float* out) {
  float a[8];
  for (int k = 0; k < 8; k++) a[k] = threadIdx.x * 1e-7f + k;
  const float m = 0.999999f, c = 1e-7f;
  for (int i = 0; i < iters; i++)
#pragma unroll
    for (int k = 0; k < 8; k++) a[k] = fmaf(a[k], m, c);
  float s = 0;
  for (int k = 0; k < 8; k++) s += a[k];
  if (s == 12345.678f) out[0] = s;  // keeps the chains live
}
__global__ void k_fma_probe64(int iters, double* out) {
  double a[8];
  for (int k = 0; k < 8; k++) a[k] = threadIdx.x * 1e-7 + k;
  const double m = 0.999999, c = 1e-7;
  for (int i = 0; i < iters; i++)
#pragma unroll
    for (int k = 0; k < 8; k++) a[k] = fma(a[k], m, c);
  double s = 0;
  for (int k = 0; k < 8; k++) s += a[k];
  if (s == 12345.678) out[0] = s;
}
}  // namespace

void launch_interactions(const StepGeom& g, int precision, const double4* src, double* tgt, bool accumulate,
                         cudaStream_t st) {
  interact_dispatch(g, precision, src, tgt, accumulate, false, 1, 0, st);
}

void launch_interactions_only(const StepGeom& g, int precision, const double4* src, double* tgt, cudaStream_t st) {
  interact_dispatch(g, precision, src, tgt, false, false, 1, 0, st, false);
}

void launch_pack_mixed(const StepGeom& g, const double4* src, cudaStream_t st) {
  long pn = (long)g.panels * g.q;
  SB_LAUNCH(k_pack_mixed, blocks_for(pn, 256), 256, 0, st, g, src, g.srcf);
}

void launch_fma_probe(int kind, int blocks, int iters, float* out32, double* out64, cudaStream_t st) {
  if (kind == 0)
    SB_LAUNCH(k_fma_probe32, blocks, 256, 0, st, iters, out32);
  else
    SB_LAUNCH(k_fma_probe64, blocks, 256, 0, st, iters, out64);
}

void launch_direct_leaves(const StepGeom& g, int precision, const double4* src, double* vout, double* partial,
                          int groups, cudaStream_t st) {
  long n = (long)g.leaves * g.q;
  interact_dispatch(g, precision, src, partial, false, true, groups, n, st);
  SB_LAUNCH(k_reduce_groups, blocks_for(3 * n, 256), 256, 0, st, partial, groups, 3 * n, 3 * n, vout);
}

void launch_depart_remap(const StepGeom& g, const BliTable* tab, const double* x, const double* y, const double* z,
                         const double* v0, const double* v1, const double* v2, const double* v3, double dt,
                         double* dep, const double* vors, const double* tracers, int T, double* new_vors,
                         double* new_tracers, int mode, cudaStream_t st) {
  long n = (long)g.leaves * g.q;
  unsigned grid = blocks_for(n, 128);
#define SB_DR(D)                                                                                                   \
  case D:                                                                                                          \
    SB_LAUNCH(k_depart_remap<D>, grid, 128, 0, st, g, *tab, x, y, z, v0, v1, v2, v3, dt, dep, vors, tracers, T,   \
              new_vors, new_tracers, mode);                                                                        \
    break;
  switch (g.degree) {
    SB_DR(0) SB_DR(1) SB_DR(2) SB_DR(3) SB_DR(4) SB_DR(5) SB_DR(6) SB_DR(7) SB_DR(8) SB_DR(9) SB_DR(10)
  }
#undef SB_DR
}

void launch_depart_remap_batch(const StepGeom& g, const BliTable* tab, int members, const double* x,
                               const double* y, const double* z, const double* v0, const double* v1,
                               const double* v2, const double* v3, double dt, const double* vors, double* new_vors,
                               cudaStream_t st) {
  const long n = (long)g.leaves * g.q;
  const dim3 grid(blocks_for(n, 128), (unsigned)members);
#define SB_DRB(D)                                                                                               \
  case D:                                                                                                       \
    SB_LAUNCH(k_depart_remap_batch<D>, grid, 128, 0, st, g, *tab, x, y, z, v0, v1, v2, v3, dt, vors, new_vors); \
    break;
  switch (g.degree) {
    SB_DRB(0) SB_DRB(1) SB_DRB(2) SB_DRB(3) SB_DRB(4) SB_DRB(5) SB_DRB(6) SB_DRB(7) SB_DRB(8) SB_DRB(9) SB_DRB(10)
  }
#undef SB_DRB
}

int direct_groups(long nt, long ns) {
  // enough blocks to fill 148 SMs a few times over, without tiny groups
  long tblocks = (nt + kDirectThreads - 1) / kDirectThreads;
  long want = (4L * 148 * 8 + tblocks - 1) / tblocks;
  long maxg = (ns + 1023) / 1024;
  long gsel = want < maxg ? want : maxg;
  return (int)(gsel < 1 ? 1 : (gsel > 64 ? 64 : gsel));
}

void launch_direct_bve(long nt, const double* tx, const double* ty, const double* tz, long ns, const double* sx,
                       const double* sy, const double* sz, const double* s, double eps, int precision, double* partial,
                       int groups, double* ux, double* uy, double* uz, cudaStream_t st) {
  dim3 grid(blocks_for(nt, kDirectThreads), groups);
  if (precision == SBSLPM_MIXED)
    SB_LAUNCH(k_direct_bve32, grid, kDirectThreads, 0, st, nt, tx, ty, tz, ns, sx, sy, sz, s, eps, partial);
  else
    SB_LAUNCH(k_direct_bve64, grid, kDirectThreads, 0, st, nt, tx, ty, tz, ns, sx, sy, sz, s, eps, partial);
  // reduce into the three output arrays (they need not be contiguous)
  double* outs[3] = {ux, uy, uz};
  for (int c = 0; c < 3; c++)
    SB_LAUNCH(k_reduce_groups, blocks_for(nt, 256), 256, 0, st, partial + (long)c * nt, groups, nt, 3 * nt, outs[c]);
}

void launch_ssw_forcing(int leaves, int q, int type, double omega, const double* time, const double* x,
                        const double* y, const double* z, double* force, cudaStream_t st) {
  SB_LAUNCH(k_ssw_forcing, blocks_for(leaves, 128), 128, 0, st, leaves, q, type, omega, time, x, y, z, force);
}

void launch_time_advance(double* time, double dt, cudaStream_t st) {
  SB_LAUNCH(k_time_advance, 1, 32, 0, st, time, dt);
}

void launch_inv_lap(long n, const double* x, const double* y, const double* z, const double* area,
                    const double* pots, double* soln, cudaStream_t st) {
  SB_LAUNCH(k_inv_lap, blocks_for(n, kDirectThreads), kDirectThreads, 0, st, n, x, y, z, area, pots, soln);
}

}  // namespace sbslpm
