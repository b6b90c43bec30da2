// Shallow-water (SWE v2) velocity kernels, sm_100a: the two-field sources and
// upward pass, and the proxy interactions of swe_vel_panel_interaction_2
// (src/fmm_interactions/swe_vel_impl.hpp:80-147):
//
//   u(x) += 1/(4 pi) [ -S_vor (x cross y')/(1 - x.y' + eps)
//                      + S_div (y - x (x.y))/(1 - x.y + eps) ]
//
// with y' the displaced, re-projected source proxy and y the fixed one.  Both
// denominators are computed as |y - x|^2/2 + eps (|x| = |y| = 1), the
// rotational part as x cross sum g (y' - x), and the divergent part as the
// tangential projection (I - x x^T) of sum g2 (y - x), which equals
// sum g2 (y - x (x.y)) for |x| = 1.  Sources (double4, 32 B per proxy):
//   src  = (y'_x, y'_y, y'_z, S_vor),   src2 = (y_x, y_y, y_z, S_div).
// Every kernel is owner-computes (no atomics) and deterministic.
#include <cuda_runtime.h>

#include <type_traits>

#include "../../include/sbslpm.h"
#include "device_common.cuh"
#include "swe_kernels.cuh"

namespace sbslpm {
namespace {

using namespace dev;

constexpr int kWarps = 4;

// ---------------------------------------------------------------------------
// Sources.

// Strengths of leaf point i (relative index) at a stage: swe_apply_tendencies_2
// (src/swe_time_step_2.cpp:390-414) folded into base_pots
// (src/fmm_funcs_impl.hpp:17-34): w_vor = area (1 + dts div) (vor + dts tv),
// w_div = area (div + dts td).
__device__ __forceinline__ void leaf_strengths(long i, long ln, int stage, double dts, const double* tprev,
                                               const double* vors, const double* divs, const double* area,
                                               double& wv, double& wd) {
  const double a = area[i], vor = vors[i], div = divs[i];
  if (stage == 0) {
    wv = a * vor;
    wd = a * div;
  } else {
    const double dvor = vor + dts * tprev[i];
    const double ddiv = div + dts * tprev[ln + i];
    wv = (a * (1.0 + dts * div)) * dvor;
    wd = a * ddiv;
  }
}

__device__ __forceinline__ float4 pack(const double* c, double x, double y, double z, double w) {
  return make_float4((float)((x - c[0]) * kPackScale), (float)((y - c[1]) * kPackScale),
                     (float)((z - c[2]) * kPackScale), (float)w);
}

// Fused upward pass over one subtree (the SWE form of k_upward_subtree): leaf
// sources of both fields when the subtree reaches the leaves, displaced
// positions of its non-leaf proxies (swe_disp_interp_2,
// src/swe_time_step_2.cpp:436-476, identical to the BVE form), both strengths
// anterpolated level by level (upward_pass, src/fmm_funcs.cpp:341-355), and
// the packed float sources in mixed precision.
__global__ void k_swe_upward_subtree(StepGeom g, SweGeom sw, int r, int D, int positions, int stage, double dtd,
                                     double dts,
                                     const double* __restrict__ vprev, const double* __restrict__ tprev,
                                     const double* __restrict__ vors, const double* __restrict__ divs,
                                     const double* __restrict__ area, double4* __restrict__ src,
                                     double4* __restrict__ src2, int mixed) {
  extern __shared__ double sh[];  // 2 fields x levels r..r+D, then 2 x 4^D q scratch
  const int q = g.q, root_rel = blockIdx.x, n1 = g.degree + 1;
  const bool leaves_here = (r + D == g.levels - 1);
  const long ln = (long)g.leaves * g.q, pn = (long)g.panels * g.q;
  const int per_field = q * (((1 << (2 * (D + 1))) - 1) / 3);
  auto lvl = [&](int f, int k) { return sh + f * per_field + q * (((1 << (2 * k)) - 1) / 3); };
  double* scratch = sh + 2 * per_field;
  const int sstride = (1 << (2 * D)) * q;

  {
    const int first = subtree_first(r, root_rel, D), npts = (1 << (2 * D)) * q;
    for (int t = threadIdx.x; t < npts; t += blockDim.x) {
      const long o = (long)first * q + t;
      double wv, wd;
      if (leaves_here) {
        const long i = o - (long)g.offset * q;
        leaf_strengths(i, ln, stage, dts, tprev, vors, divs, area, wv, wd);
        double px = g.px[o], py = g.px[pn + o], pz = g.px[2 * pn + o];
        src2[o] = make_double4(px, py, pz, wd);
        if (stage > 0) {
          px += dtd * vprev[i];
          py += dtd * vprev[ln + i];
          pz += dtd * vprev[2 * ln + i];
        }
        project_to_sphere(px, py, pz);
        src[o] = make_double4(px, py, pz, wv);
      } else {
        wv = src[o].w;
        wd = src2[o].w;
      }
      lvl(0, D)[t] = wv;
      lvl(1, D)[t] = wd;
    }
  }
  for (int k = 0; positions && k < D; k++) {  // else k_swe_nonleaf_positions wrote them
    const int first = subtree_first(r, root_rel, k), npts = (1 << (2 * k)) * q;
    for (int t = threadIdx.x; t < npts; t += blockDim.x) {
      const long i = (long)first * q + t;
      double px, py, pz;
      nonleaf_position(g, i, stage, dtd, vprev, px, py, pz);
      src[i] = make_double4(px, py, pz, 0.0);
      src2[i] = make_double4(g.px[i], g.px[pn + i], g.px[2 * pn + i], 0.0);
    }
  }
  __syncthreads();
  for (int k = D - 1; k >= 0; k--) {
    const int np = 1 << (2 * k), first = subtree_first(r, root_rel, k);
    for (int t = threadIdx.x; t < 2 * 4 * np * q; t += blockDim.x) {  // T[f][cc][i][b]
      const int f = t / (4 * np * q), tt = t % (4 * np * q);
      const int cc = tt / q, rem = tt % q, i = rem / n1, b = rem % n1;
      const double* ly = g.child_1d + ((cc & 3) >= 2 ? n1 * n1 : 0);
      const double* sc = lvl(f, k + 1) + cc * q + i * n1;
      double acc = 0;
      for (int j = 0; j < n1; j++) acc = fma(__ldg(ly + j * n1 + b), sc[j], acc);
      scratch[f * sstride + tt] = acc;
    }
    __syncthreads();
    for (int t = threadIdx.x; t < 2 * np * q; t += blockDim.x) {  // S[f][p][a][b]
      const int f = t / (np * q), tt = t % (np * q);
      const int p = tt / q, rem = tt % q, a = rem / n1, b = rem % n1;
      double acc = 0;
      for (int c = 0; c < 4; c++) {
        const double* lx = g.child_1d + ((c == 1 || c == 2) ? n1 * n1 : 0);
        const double* tc = scratch + f * sstride + (4 * p + c) * q + b;
        for (int i = 0; i < n1; i++) acc = fma(__ldg(lx + i * n1 + a), tc[i * n1], acc);
      }
      lvl(f, k)[tt] = acc;
      if (f == 0) src[(long)first * q + tt].w = acc;
      else src2[(long)first * q + tt].w = acc;
    }
    __syncthreads();
  }
  if (mixed) {
    const int kmax = leaves_here ? D : D - 1;
    for (int k = 0; k <= kmax; k++) {
      const int first = subtree_first(r, root_rel, k), npts = (1 << (2 * k)) * q;
      for (int t = threadIdx.x; t < npts; t += blockDim.x) {
        const long i = (long)first * q + t;
        const double* cc = g.pd_centre + 4 * (i / q);
        const double4 a = src[i], b = src2[i];
        g.srcf[i] = pack(cc, a.x, a.y, a.z, a.w);
        sw.srcf2[i] = pack(cc, b.x, b.y, b.z, b.w);
      }
    }
  }
}

// Positions of every non-leaf proxy of both fields in one flat launch ahead
// of the subtree passes, a thread per point: the vorticity sources displaced
// by the interpolated leaf velocity (nonleaf_position's arithmetic, q = 16
// unrolled), the divergence sources at the fixed proxies.
template <int Q>
__global__ void k_swe_nonleaf_positions(StepGeom g, int stage, double dtd, const double* __restrict__ vprev,
                                        double4* __restrict__ src, double4* __restrict__ src2) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const int q = Q > 0 ? Q : g.q;
  if (i >= (long)g.offset * q) return;
  const long pn = (long)g.panels * q, ln = (long)g.leaves * q;
  const double x0 = g.px[i], y0 = g.px[pn + i], z0 = g.px[2 * pn + i];
  double px = x0, py = y0, pz = z0;
  if (stage > 0) {
    const long np = (long)g.offset * q;
    const long row = (long)g.il_row[i] * q;
    double ax = 0, ay = 0, az = 0;
#pragma unroll
    for (int m = 0; m < (Q > 0 ? Q : q); m++) {
      const double bm = g.il_basis[m * np + i];
      ax += (dtd * vprev[row + m]) * bm;
      ay += (dtd * vprev[ln + row + m]) * bm;
      az += (dtd * vprev[2 * ln + row + m]) * bm;
    }
    px += ax;
    py += ay;
    pz += az;
  }
  project_to_sphere(px, py, pz);
  src[i] = make_double4(px, py, pz, 0.0);
  src2[i] = make_double4(x0, y0, z0, 0.0);
}

// Direct velocity: leaf sources of both fields (no tree).
__global__ void k_swe_leaf_sources(StepGeom g, SweGeom sw, int stage, double dtd, double dts,
                                   const double* __restrict__ vprev, const double* __restrict__ tprev,
                                   const double* __restrict__ vors, const double* __restrict__ divs,
                                   const double* __restrict__ area, double4* __restrict__ src,
                                   double4* __restrict__ src2, int mixed) {
  const long ln = (long)g.leaves * g.q, pn = (long)g.panels * g.q;
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= ln) return;
  const long o = (long)g.offset * g.q + i;
  double wv, wd;
  leaf_strengths(i, ln, stage, dts, tprev, vors, divs, area, wv, wd);
  double px = g.px[o], py = g.px[pn + o], pz = g.px[2 * pn + o];
  src2[o] = make_double4(px, py, pz, wd);
  if (mixed) sw.srcf2[o] = pack(g.pd_centre + 4 * (o / g.q), px, py, pz, wd);
  if (stage > 0) {
    px += dtd * vprev[i];
    py += dtd * vprev[ln + i];
    pz += dtd * vprev[2 * ln + i];
  }
  project_to_sphere(px, py, pz);
  src[o] = make_double4(px, py, pz, wv);
  if (mixed) g.srcf[o] = pack(g.pd_centre + 4 * (o / g.q), px, py, pz, wv);
}

// Piecewise API: sources from explicit displacements (swe_vel_panel_interaction_2
// displaces every proxy, src/fmm_interactions/swe_vel_impl.hpp:124-128) and strengths.
__global__ void k_swe_sources_from_disp(StepGeom g, SweGeom sw, const double* __restrict__ dx,
                                        const double* __restrict__ dy, const double* __restrict__ dz,
                                        const double* __restrict__ sv, const double* __restrict__ sd,
                                        double4* __restrict__ src, double4* __restrict__ src2, int mixed) {
  const long pn = (long)g.panels * g.q;
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= pn) return;
  const double x0 = g.px[i], y0 = g.px[pn + i], z0 = g.px[2 * pn + i];
  double px = x0 + dx[i], py = y0 + dy[i], pz = z0 + dz[i];
  project_to_sphere(px, py, pz);
  src[i] = make_double4(px, py, pz, sv[i]);
  src2[i] = make_double4(x0, y0, z0, sd[i]);
  if (mixed) {
    const double* c = g.pd_centre + 4 * (i / g.q);
    g.srcf[i] = pack(c, px, py, pz, sv[i]);
    sw.srcf2[i] = pack(c, x0, y0, z0, sd[i]);
  }
}

// ---------------------------------------------------------------------------
// Interactions.  One warp per target panel; for q <= 16 the warp's lanes are
// (32/q source splits) x (q target nodes), for larger q each lane owns
// ceil(q/32) target nodes.  A source panel's q proxies of both fields are
// staged in shared memory and every lane sweeps them (mixed: two proxies per
// paired float32 instruction, each panel's two interleaved float32 halves
// added before the float64 conversion).  ALL_LEAVES: every
// leaf against every leaf, source leaves split into gridDim.y groups whose
// partials are reduced in order afterwards.

template <int Q>
struct Shape {
  static constexpr int S = Q <= 16 ? 32 / Q : 1;
  static constexpr int TPL = Q <= 32 ? 1 : (Q + 31) / 32;
  static constexpr int STAGE = S * Q > Q ? S * Q : Q;
};

// u = K x cross A - K (B - x (x.B)); K = -1/(4 pi), or scaled by sqrt(2)
// for the packed float sums.
__device__ __forceinline__ void swe_epilogue(double K, double tx, double ty, double tz, double ax, double ay,
                                             double az, double bx, double by, double bz, double& ux, double& uy,
                                             double& uz) {
  const double tb = tx * bx + ty * by + tz * bz;
  ux = K * (ty * az - tz * ay) - K * (bx - tx * tb);
  uy = K * (tz * ax - tx * az) - K * (by - ty * tb);
  uz = K * (tx * ay - ty * ax) - K * (bz - tz * tb);
}

template <int Q, bool ALL_LEAVES, bool GUARD, bool MIXED>
__global__ void __launch_bounds__(32 * kWarps)
    k_swe_interact(StepGeom g, SweGeom sw, const double4* __restrict__ src, const double4* __restrict__ src2,
                   double* __restrict__ out, long out_stride) {
  using W = Shape<Q>;
  using Src = typename std::conditional<MIXED, float4, double4>::type;
  // mixed: a split's Q proxies as ceil(Q/2) source pairs of two float4
  // (x0,x1,y0,y1),(z0,z1,w0,w1), an odd Q closing on a zero-strength source
  // at the panel's centre (which adds exactly zero)
  constexpr int HQ = (Q + 1) / 2, SPLIT = MIXED ? 2 * HQ : Q, STG = MIXED ? W::S * 2 * HQ : W::STAGE;
  __shared__ Src stage[kWarps][2][STG];
  __shared__ double red[kWarps][6][32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int tp_first = ALL_LEAVES ? g.offset : 0;
  const int tp_count = ALL_LEAVES ? g.leaves : g.panels;
  const int tix = blockIdx.x * kWarps + warp;
  if (tix >= tp_count) return;
  const int t = tp_first + tix;
  const long pn = (long)g.panels * g.q;
  int e0, e1;
  if (ALL_LEAVES) {
    const int per = (g.leaves + gridDim.y - 1) / gridDim.y;
    e0 = blockIdx.y * per;
    e1 = min(g.leaves, e0 + per);
  } else {
    e0 = g.tgt_start[t];
    e1 = g.tgt_start[t + 1];
  }
  auto source_of = [&](int e) { return ALL_LEAVES ? g.offset + e : __ldg(g.src_panel + e); };
  const Src* s1 = nullptr;
  const Src* s2 = nullptr;
  if constexpr (MIXED) {
    s1 = g.srcf;
    s2 = sw.srcf2;
  } else {
    s1 = src;
    s2 = src2;
  }
  const double* ct = g.pd_centre + 4 * (long)t;
  const float eps32 = (float)g.eps;
  constexpr double K = MIXED ? kBiotSavartPacked : kBiotSavart;
  constexpr int TPL = W::TPL;
  const int h = Q <= 32 ? lane / Q : 0;
  const bool active = Q <= 32 ? h < W::S : true;

  double tx[TPL], ty[TPL], tz[TPL], ax[TPL], ay[TPL], az[TPL], bx[TPL], by[TPL], bz[TPL];
  float dtx[TPL], dty[TPL], dtz[TPL];
#pragma unroll
  for (int r = 0; r < TPL; r++) {
    const int j = Q <= 32 ? lane % Q : lane + 32 * r;
    const long o = (long)t * Q + (j < Q ? j : 0);
    tx[r] = g.px[o];
    ty[r] = g.px[pn + o];
    tz[r] = g.px[2 * pn + o];
    if (MIXED) {
      dtx[r] = (float)((tx[r] - ct[0]) * kPackScale);
      dty[r] = (float)((ty[r] - ct[1]) * kPackScale);
      dtz[r] = (float)((tz[r] - ct[2]) * kPackScale);
    }
    ax[r] = ay[r] = az[r] = bx[r] = by[r] = bz[r] = 0;
  }
  constexpr int STEP = Q <= 32 ? W::S : 1;
  // a lane's share of the staging: a proxy (float64) or a source pair (mixed)
  auto stage_one = [&](int sp, int k, int slot) {
    if constexpr (MIXED) {
      const long b = (long)sp * Q + 2 * k;
      const bool two = 2 * k + 1 < Q;
      const float4 none = make_float4(0.f, 0.f, 0.f, 0.f);
      const float4 a0 = s1[b], a1 = two ? s1[b + 1] : none, c0 = s2[b], c1 = two ? s2[b + 1] : none;
      stage[warp][0][slot + 2 * k] = make_float4(a0.x, a1.x, a0.y, a1.y);
      stage[warp][0][slot + 2 * k + 1] = make_float4(a0.z, a1.z, a0.w, a1.w);
      stage[warp][1][slot + 2 * k] = make_float4(c0.x, c1.x, c0.y, c1.y);
      stage[warp][1][slot + 2 * k + 1] = make_float4(c0.z, c1.z, c0.w, c1.w);
    } else {
      stage[warp][0][slot + k] = s1[(long)sp * Q + k];
      stage[warp][1][slot + k] = s2[(long)sp * Q + k];
    }
  };
  constexpr int PER = MIXED ? HQ : Q;  // staging items per source panel
  for (int e = e0; e < e1; e += STEP) {
    int sp = 0;
    if (Q <= 32) {
      if (active && e + h < e1) {
        sp = source_of(e + h);
        const int j = lane % Q;
        if (j < PER) stage_one(sp, j, h * SPLIT);
      }
    } else {
      sp = source_of(e);
      for (int k = lane; k < PER; k += 32) stage_one(sp, k, 0);
    }
    __syncwarp();
    if (active && e + h < e1) {
      const Src* st1 = &stage[warp][0][h * SPLIT];
      const Src* st2 = &stage[warp][1][h * SPLIT];
      if constexpr (MIXED) {
        const double* cs = g.pd_centre + 4 * (long)sp;
        const float c0 = (float)((cs[0] - ct[0]) * kPackScale), c1 = (float)((cs[1] - ct[1]) * kPackScale),
                    c2 = (float)((cs[2] - ct[2]) * kPackScale);
        const float2 eps2 = make_float2(eps32, eps32);
        float2 fa[TPL][3], fb[TPL][3], b0[TPL], b1[TPL], b2[TPL];
#pragma unroll
        for (int r = 0; r < TPL; r++) {
          b0[r] = make_float2(c0 - dtx[r], c0 - dtx[r]);
          b1[r] = make_float2(c1 - dty[r], c1 - dty[r]);
          b2[r] = make_float2(c2 - dtz[r], c2 - dtz[r]);
          fa[r][0] = fa[r][1] = fa[r][2] = fb[r][0] = fb[r][1] = fb[r][2] = make_float2(0.f, 0.f);
        }
#pragma unroll 4
        for (int k = 0; k < HQ; k++) {
          const float4 A = st1[2 * k], B = st1[2 * k + 1], C = st2[2 * k], D = st2[2 * k + 1];
#pragma unroll
          for (int r = 0; r < TPL; r++) {
            pair32x2<GUARD>(b0[r], b1[r], b2[r], make_float2(A.x, A.y), make_float2(A.z, A.w),
                            make_float2(B.x, B.y), make_float2(B.z, B.w), eps2, fa[r][0], fa[r][1], fa[r][2]);
            pair32x2<GUARD>(b0[r], b1[r], b2[r], make_float2(C.x, C.y), make_float2(C.z, C.w),
                            make_float2(D.x, D.y), make_float2(D.z, D.w), eps2, fb[r][0], fb[r][1], fb[r][2]);
          }
        }
#pragma unroll
        for (int r = 0; r < TPL; r++) {
          ax[r] += (double)(fa[r][0].x + fa[r][0].y);
          ay[r] += (double)(fa[r][1].x + fa[r][1].y);
          az[r] += (double)(fa[r][2].x + fa[r][2].y);
          bx[r] += (double)(fb[r][0].x + fb[r][0].y);
          by[r] += (double)(fb[r][1].x + fb[r][1].y);
          bz[r] += (double)(fb[r][2].x + fb[r][2].y);
        }
      } else {
#pragma unroll 4
        for (int k = 0; k < Q; k++) {
          const double4 v1 = st1[k], v2 = st2[k];
#pragma unroll
          for (int r = 0; r < TPL; r++) {
            pair64<GUARD>(tx[r], ty[r], tz[r], v1, g.eps, ax[r], ay[r], az[r]);
            pair64<GUARD>(tx[r], ty[r], tz[r], v2, g.eps, bx[r], by[r], bz[r]);
          }
        }
      }
    }
    __syncwarp();
  }
  if (Q <= 32 && W::S > 1) {
    red[warp][0][lane] = ax[0];
    red[warp][1][lane] = ay[0];
    red[warp][2][lane] = az[0];
    red[warp][3][lane] = bx[0];
    red[warp][4][lane] = by[0];
    red[warp][5][lane] = bz[0];
    __syncwarp();
    if (h == 0)
      for (int hh = 1; hh < W::S; hh++) {
        const int l = hh * Q + lane % Q;
        ax[0] += red[warp][0][l];
        ay[0] += red[warp][1][l];
        az[0] += red[warp][2][l];
        bx[0] += red[warp][3][l];
        by[0] += red[warp][4][l];
        bz[0] += red[warp][5][l];
      }
  }
  if (h != 0) return;
#pragma unroll
  for (int r = 0; r < TPL; r++) {
    const int j = Q <= 32 ? lane % Q : lane + 32 * r;
    if (j >= Q) continue;
    double ux, uy, uz;
    const long ot = (long)t * Q + j;  // the target's position again: not held in registers across the sweep
    swe_epilogue(K, g.px[ot], g.px[pn + ot], g.px[2 * pn + ot], ax[r], ay[r], az[r], bx[r], by[r], bz[r], ux, uy,
                 uz);
    const long o = ALL_LEAVES ? (long)blockIdx.y * 3 * out_stride + (long)tix * Q + j : (long)t * Q + j;
    const long s = ALL_LEAVES ? out_stride : pn;
    out[o] = ux;
    out[s + o] = uy;
    out[2 * s + o] = uz;
  }
}

// Mixed precision, q <= 32, list mode: the BVE list kernel's organisation
// (k_interact32) with both source fields.  List entries come 32 at a time
// from the static entry table (source panel, centre offset as float) and are
// handed to the splits by shuffles; the next entry's sources of both fields
// are loaded while the current ones are evaluated; each field's source pair
// is staged (x0,x1,y0,y1),(z0,z1,w0,w1) by one store per lane, and both
// fields' pairs run on the paired float32 instructions (pair32x2), two
// sources per instruction.  A panel's float32 halves are added before the
// float64 conversion.
template <int Q, bool GUARD>
__global__ void __launch_bounds__(32 * kWarps) k_swe_interact32_list(StepGeom g, SweGeom sw,
                                                                     double* __restrict__ out) {
  using W = Shape<Q>;
  constexpr int Q2 = (Q + 1) / 2;
  __shared__ float4 stage[kWarps][2][W::S * 2 * Q2];
  __shared__ double red[kWarps][6][32];
  const unsigned full = 0xffffffffu;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int t = blockIdx.x * kWarps + warp;
  if (t >= g.panels) return;
  const long pn = (long)g.panels * Q;
  const int e0 = g.tgt_start[t], e1 = g.tgt_start[t + 1];
  const int h = lane / Q, j = lane % Q;
  const bool active = h < W::S;
  const double* ct = g.pd_centre + 4 * (long)t;
  double tx = 0, ty = 0, tz = 0;
  float dtx = 0, dty = 0, dtz = 0;
  if (active) {
    const long o = (long)t * Q + j;
    tx = g.px[o];
    ty = g.px[pn + o];
    tz = g.px[2 * pn + o];
    dtx = (float)((tx - ct[0]) * kPackScale);
    dty = (float)((ty - ct[1]) * kPackScale);
    dtz = (float)((tz - ct[2]) * kPackScale);
  }
  double ax = 0, ay = 0, az = 0, bx = 0, by = 0, bz = 0;
  const float feps = (float)g.eps;
  const float2 eps2 = make_float2(feps, feps);
  float4* t1 = &stage[warp][0][(active ? h : 0) * 2 * Q2];
  float4* t2 = &stage[warp][1][(active ? h : 0) * 2 * Q2];
  const bool odd = j & 1, last_odd = (Q & 1) && j == Q - 1;
  const int partner = (odd ? lane - 1 : lane + 1) & 31;
  auto put = [&](float4* tl, const float4& v, float r0, float r1) {
    const int k2 = j >> 1;
    if (last_odd) {
      tl[2 * k2] = make_float4(v.x, 0.f, v.y, 0.f);
      tl[2 * k2 + 1] = make_float4(v.z, 0.f, v.w, 0.f);
    } else if (!odd) {
      tl[2 * k2] = make_float4(v.x, r0, v.y, r1);
    } else {
      tl[2 * k2 + 1] = make_float4(r0, v.z, r1, v.w);
    }
  };
  for (int eb = e0; eb < e1; eb += 32) {
    const int nb = min(32, e1 - eb);
    int4 en = make_int4(0, 0, 0, 0);
    if (lane < nb) en = __ldg(g.entry + eb + lane);
    const int iters = (nb + W::S - 1) / W::S;
    float cbx = __int_as_float(__shfl_sync(full, en.y, h & 31));
    float cby = __int_as_float(__shfl_sync(full, en.z, h & 31));
    float cbz = __int_as_float(__shfl_sync(full, en.w, h & 31));
    float4 v1 = make_float4(0.f, 0.f, 0.f, 0.f), v2 = v1;
    {
      const int sp = __shfl_sync(full, en.x, h & 31);
      if (active && h < nb) {
        v1 = g.srcf[(long)sp * Q + j];
        v2 = sw.srcf2[(long)sp * Q + j];
      }
    }
    for (int it = 0; it < iters; it++) {
      const bool on = active && it * W::S + h < nb;
      const int ns = (it + 1) * W::S + h;
      const int sp_n = __shfl_sync(full, en.x, ns & 31);
      const float nbx = __int_as_float(__shfl_sync(full, en.y, ns & 31));
      const float nby = __int_as_float(__shfl_sync(full, en.z, ns & 31));
      const float nbz = __int_as_float(__shfl_sync(full, en.w, ns & 31));
      float4 n1 = make_float4(0.f, 0.f, 0.f, 0.f), n2 = n1;
      if (active && ns < nb) {
        n1 = g.srcf[(long)sp_n * Q + j];
        n2 = sw.srcf2[(long)sp_n * Q + j];
      }
      const float p0 = __shfl_sync(full, odd ? v1.x : v1.z, partner);
      const float p1 = __shfl_sync(full, odd ? v1.y : v1.w, partner);
      const float q0 = __shfl_sync(full, odd ? v2.x : v2.z, partner);
      const float q1 = __shfl_sync(full, odd ? v2.y : v2.w, partner);
      if (on) {
        put(t1, v1, p0, p1);
        put(t2, v2, q0, q1);
      }
      __syncwarp();
      if (on) {
        const float b0 = cbx - dtx, b1 = cby - dty, b2 = cbz - dtz;
        const float2 px2 = make_float2(b0, b0), py2 = make_float2(b1, b1), pz2 = make_float2(b2, b2);
        float2 fax = make_float2(0.f, 0.f), fay = fax, faz = fax, fbx = fax, fby = fax, fbz = fax;
#pragma unroll
        for (int k2 = 0; k2 < Q2; k2++) {
          const float4 A = t1[2 * k2], B = t1[2 * k2 + 1], C = t2[2 * k2], D = t2[2 * k2 + 1];
          pair32x2<GUARD>(px2, py2, pz2, make_float2(A.x, A.y), make_float2(A.z, A.w), make_float2(B.x, B.y),
                          make_float2(B.z, B.w), eps2, fax, fay, faz);
          pair32x2<GUARD>(px2, py2, pz2, make_float2(C.x, C.y), make_float2(C.z, C.w), make_float2(D.x, D.y),
                          make_float2(D.z, D.w), eps2, fbx, fby, fbz);
        }
        ax += (double)(fax.x + fax.y);
        ay += (double)(fay.x + fay.y);
        az += (double)(faz.x + faz.y);
        bx += (double)(fbx.x + fbx.y);
        by += (double)(fby.x + fby.y);
        bz += (double)(fbz.x + fbz.y);
      }
      __syncwarp();
      v1 = n1;
      v2 = n2;
      cbx = nbx;
      cby = nby;
      cbz = nbz;
    }
  }
  if (W::S > 1) {
    red[warp][0][lane] = ax;
    red[warp][1][lane] = ay;
    red[warp][2][lane] = az;
    red[warp][3][lane] = bx;
    red[warp][4][lane] = by;
    red[warp][5][lane] = bz;
    __syncwarp();
    if (h == 0)
      for (int hh = 1; hh < W::S; hh++) {
        const int l = hh * Q + j;
        ax += red[warp][0][l];
        ay += red[warp][1][l];
        az += red[warp][2][l];
        bx += red[warp][3][l];
        by += red[warp][4][l];
        bz += red[warp][5][l];
      }
  }
  if (h != 0) return;
  double ux, uy, uz;
  swe_epilogue(kBiotSavartPacked, tx, ty, tz, ax, ay, az, bx, by, bz, ux, uy, uz);
  const long o = (long)t * Q + j;
  out[o] = ux;
  out[pn + o] = uy;
  out[2 * pn + o] = uz;
}

__global__ void k_swe_reduce(const double* __restrict__ partial, int groups, long n, long gstride,
                             double* __restrict__ out) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double s = 0;
  for (int k = 0; k < groups; k++) s += partial[k * gstride + i];
  out[i] = s;
}

template <int Q, bool GUARD>
void swe_interact_qg(const StepGeom& g, const SweGeom& s, int precision, const double4* src, const double4* src2,
                     double* out, bool all_leaves, int groups, long out_stride, cudaStream_t st) {
  const int tp = all_leaves ? g.leaves : g.panels;
  dim3 grid(blocks_for(tp, kWarps), all_leaves ? groups : 1);
  const bool mixed = precision == SBSLPM_MIXED;
#define SB_SWE_K(AL, MX) \
  SB_LAUNCH((k_swe_interact<Q, AL, GUARD, MX>), grid, 32 * kWarps, 0, st, g, s, src, src2, out, out_stride)
  if (all_leaves) {
    if (mixed) SB_SWE_K(true, true);
    else SB_SWE_K(true, false);
  } else {
    if constexpr (Q <= 32) {
      if (mixed && g.entry) {
        SB_LAUNCH((k_swe_interact32_list<Q, GUARD>), grid, 32 * kWarps, 0, st, g, s, out);
        return;
      }
    }
    if (mixed) SB_SWE_K(false, true);
    else SB_SWE_K(false, false);
  }
#undef SB_SWE_K
}

void swe_interact_dispatch(const StepGeom& g, const SweGeom& s, int precision, const double4* src,
                           const double4* src2, double* out, bool all_leaves, int groups, long out_stride,
                           cudaStream_t st) {
#define SB_SQ(Q)                                                                                   \
  case Q:                                                                                          \
    if (g.eps > 0) swe_interact_qg<Q, false>(g, s, precision, src, src2, out, all_leaves, groups, out_stride, st); \
    else swe_interact_qg<Q, true>(g, s, precision, src, src2, out, all_leaves, groups, out_stride, st);            \
    break;
  switch (g.q) {
    SB_SQ(1) SB_SQ(4) SB_SQ(9) SB_SQ(16) SB_SQ(25) SB_SQ(36) SB_SQ(49) SB_SQ(64) SB_SQ(81) SB_SQ(100) SB_SQ(121)
  }
#undef SB_SQ
}

size_t swe_subtree_smem(int q, int D) {
  return (size_t)q * 2 * 8 * ((((1L << (2 * (D + 1))) - 1) / 3) + (1L << (2 * D)));
}

}  // namespace

void launch_swe_upward(const StepGeom& g, const SweGeom& s, int stage, double dtd, double dts, const double* vprev,
                       const double* tprev, const double*, const double*, const double*, const double* vors,
                       const double* divs, const double* area, double4* src, double4* src2, bool mixed,
                       cudaStream_t st) {
  static std::atomic<unsigned long long> attr{0};
  raise_smem_once(attr, 200 * 1024, k_swe_upward_subtree);
  const int Dmax = g.q <= 25 ? 3 : 1;
  int r = g.levels - 1;
  const long nl = (long)g.offset * g.q;  // non-leaf proxy points
  if (nl > 0) {
    if (g.q == 16)
      SB_LAUNCH(k_swe_nonleaf_positions<16>, blocks_for(nl, 256), 256, 0, st, g, stage, dtd, vprev, src, src2);
    else
      SB_LAUNCH(k_swe_nonleaf_positions<0>, blocks_for(nl, 256), 256, 0, st, g, stage, dtd, vprev, src, src2);
  }
  do {
    const int D = r < Dmax ? r : Dmax;
    const int root = r - D;
    SB_LAUNCH(k_swe_upward_subtree, (unsigned)(6 << (2 * root)), 256, swe_subtree_smem(g.q, D), st, g, s, root, D,
              nl > 0 ? 0 : 1, stage, dtd, dts, vprev, tprev, vors, divs, area, src, src2, mixed ? 1 : 0);
    r = root;
  } while (r > 0);
}

void launch_swe_leaf_sources(const StepGeom& g, const SweGeom& s, int stage, double dtd, double dts,
                             const double* vprev, const double* tprev, const double* vors, const double* divs,
                             const double* area, double4* src, double4* src2, bool mixed, cudaStream_t st) {
  const long ln = (long)g.leaves * g.q;
  SB_LAUNCH(k_swe_leaf_sources, blocks_for(ln, 256), 256, 0, st, g, s, stage, dtd, dts, vprev, tprev, vors, divs,
            area, src, src2, mixed ? 1 : 0);
}

void launch_swe_interactions(const StepGeom& g, const SweGeom& s, int precision, const double4* src,
                             const double4* src2, double* tgt, cudaStream_t st) {
  swe_interact_dispatch(g, s, precision, src, src2, tgt, false, 1, 0, st);
}

void launch_swe_direct(const StepGeom& g, const SweGeom& s, int precision, const double4* src, const double4* src2,
                       double* vout, double* partial, int groups, cudaStream_t st) {
  const long n = (long)g.leaves * g.q;
  swe_interact_dispatch(g, s, precision, src, src2, partial, true, groups, n, st);
  SB_LAUNCH(k_swe_reduce, blocks_for(3 * n, 256), 256, 0, st, partial, groups, 3 * n, 3 * n, vout);
}

void launch_swe_sources_from_disp(const StepGeom& g, const SweGeom& s, const double* dx, const double* dy,
                                  const double* dz, const double* s_vor, const double* s_div, double4* src,
                                  double4* src2, bool mixed, cudaStream_t st) {
  const long pn = (long)g.panels * g.q;
  SB_LAUNCH(k_swe_sources_from_disp, blocks_for(pn, 256), 256, 0, st, g, s, dx, dy, dz, s_vor, s_div, src, src2,
            mixed ? 1 : 0);
}

}  // namespace sbslpm
