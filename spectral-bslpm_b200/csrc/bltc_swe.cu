// Treecode velocity of the shallow-water step (decoupled proxy degree), sm_100a.
//
// The SWE velocity (swe_vel_panel_interaction_2, src/fmm_interactions/swe_vel_impl.hpp:80-147)
// has two source fields: vorticity at the displaced positions (rotational
// part, x cross y' / (1 - x.y' + eps)) and divergence at the grid positions
// (divergent part, (y - x (x.y)) / (1 - x.y + eps)).  On the treecode of the
// BVE step (bltc_kernels.cu) each field gets its own proxy strengths on the
// same fixed proxies: the vorticity anterpolated from the displaced
// particles, the divergence from the grid particles (the leaf-box basis of
// the grid, the same for every leaf).  Near leaf pairs evaluate both fields
// particle x particle; well-separated pairs run the SWE proxy kernel
// (k_swe_interact) on the tree; the downward pass and the leaf interpolation
// are the BVE treecode's.  This is the reference's irregular-point design
// (swe_vel_panel_interaction_ll, src/fmm_interactions/swe_vel_impl.hpp:149-288,
// whose pairs carry both fields) with every well-separated pair proxy x proxy.
#include <cuda_runtime.h>

#include <type_traits>

#include "../../include/sbslpm.h"
#include "device_common.cuh"
#include "swe_kernels.cuh"

namespace sbslpm {
namespace {

using namespace dev;

constexpr int kThreads = 256;

// Barycentric basis of degree n on Chebyshev extrema of [lo, hi], extended
// past the interval (displaced sources may leave their leaf); one division
// (the second barycentric form multiplied through by prod_j (t - c_j)).
__device__ __forceinline__ void swe_bli_free(double t, double lo, double hi, int n, const double* cosv,
                                             const double* w, double* f) {
  if (n == 0) {
    f[0] = 1;
    return;
  }
  const double range = 0.5 * (hi - lo), offset = 0.5 * (hi + lo);
  double dl[kMaxDegree + 1];
  int hit = -1;
#pragma unroll
  for (int i = 0; i <= kMaxDegree; i++) {
    dl[i] = i <= n ? t - (cosv[i] * range + offset) : 1.0;
    if (i <= n && hit < 0 && fabs(dl[i]) < 1e-15) hit = i;
  }
  if (hit >= 0) {
    for (int i = 0; i <= n; i++) f[i] = (i == hit) ? 1.0 : 0.0;
    return;
  }
  double pre[kMaxDegree + 1];
  pre[0] = 1.0;
#pragma unroll
  for (int i = 1; i <= kMaxDegree; i++) pre[i] = pre[i - 1] * dl[i - 1];
  double suf = 1.0, den = 0.0, v[kMaxDegree + 1];
#pragma unroll
  for (int i = kMaxDegree; i >= 0; i--) {
    v[i] = i <= n ? w[i] * (pre[i] * suf) : 0.0;
    den += v[i];
    suf *= dl[i];
  }
  const double inv = 1.0 / den;
#pragma unroll
  for (int i = 0; i <= kMaxDegree; i++)
    if (i <= n) f[i] = v[i] * inv;
}

// One CTA per treecode leaf: both fields' particle sources and their
// anterpolation onto the leaf's proxies.  Step mode (no displacement arrays): the
// strengths of swe_apply_tendencies_2 folded into base_pots
// (src/swe_time_step_2.cpp:390-414, src/fmm_funcs_impl.hpp:17-34), w_vor =
// area (1 + dts div)(vor + dts tv) at x + dtd vprev (re-projected), w_div =
// area (div + dts td) at x; stage 0: area vor and area div, undisplaced.
// Piecewise mode: positions x + disp (re-projected) and strengths given.
__global__ void __launch_bounds__(kThreads)
    k_bltc_swe_sources(TreeGeom tg, StepGeom fg, BliTable tab, int stage, double dtd, double dts,
                       const double* __restrict__ vprev, const double* __restrict__ tprev,
                       const double* __restrict__ x, const double* __restrict__ y, const double* __restrict__ z,
                       const double* __restrict__ vors, const double* __restrict__ divs,
                       const double* __restrict__ area, const double* __restrict__ dispx,
                       const double* __restrict__ dispy, const double* __restrict__ dispz,
                       const double* __restrict__ wv_in, const double* __restrict__ wd_in, double4* __restrict__ psrc,
                       float4* __restrict__ psrcf, double4* __restrict__ psrc2, float4* __restrict__ psrcf2,
                       double4* __restrict__ proxy, double4* __restrict__ proxy2, int mixed,
                       const double* __restrict__ gcentre, int gq) {
  extern __shared__ double sh[];
  const int f = blockIdx.x, n1 = tg.n + 1, npl = tg.npl;
  double* lx = sh;              // [npl][n1] basis of the displaced vorticity sources
  double* ly = lx + npl * n1;   // [npl][n1]
  double* sw = ly + npl * n1;   // [npl] vorticity strengths
  double* sd = sw + npl;        // [npl] divergence strengths
  double* part = sd + npl;      // [2][G][qx] group partials
  const int panel = fg.offset + f;
  const double* bd = tg.fbounds + 4 * panel;
  const int face = tg.fface[panel];
  const long N = tg.N;
  for (int k = threadIdx.x; k < npl; k += blockDim.x) {
    const long i = (long)f * npl + k;
    const double gx = x[i], gy = y[i], gz = z[i];
    double xx = gx, yy = gy, zz = gz, wv, wd;
    if (dispx) {
      xx += dispx[i];
      yy += dispy[i];
      zz += dispz[i];
      wv = wv_in[i];
      wd = wd_in[i];
    } else {
      const double a = area[i], vor = vors[i], div = divs[i];
      if (stage == 0) {
        wv = a * vor;
        wd = a * div;
      } else {
        xx += dtd * vprev[i];
        yy += dtd * vprev[N + i];
        zz += dtd * vprev[2 * N + i];
        wv = (a * (1.0 + dts * div)) * (vor + dts * tprev[i]);
        wd = a * (div + dts * tprev[N + i]);
      }
    }
    project_to_sphere(xx, yy, zz);
    psrc[i] = make_double4(xx, yy, zz, wv);
    psrc2[i] = make_double4(gx, gy, gz, wd);
    if (mixed) {  // packed relative to the particle's grid leaf (see k_bltc_swe_near)
      const double* gc = gcentre + 4 * (i / gq);
      psrcf[i] = make_float4((float)((xx - gc[0]) * kPackScale), (float)((yy - gc[1]) * kPackScale),
                             (float)((zz - gc[2]) * kPackScale), (float)wv);
      psrcf2[i] = make_float4((float)((gx - gc[0]) * kPackScale), (float)((gy - gc[1]) * kPackScale),
                              (float)((gz - gc[2]) * kPackScale), (float)wd);
    }
    double xi, eta;
    xieta_from_xyz_face(xx, yy, zz, face, xi, eta);
    swe_bli_free(xi, bd[0], bd[1], tg.n, tab.cosv, tab.w, lx + k * n1);
    swe_bli_free(eta, bd[2], bd[3], tg.n, tab.cosv, tab.w, ly + k * n1);
    sw[k] = wv;
    sd[k] = wd;
  }
  __syncthreads();
  // S[a][b] = sum_k lx[k][a] ly[k][b] w_k over G contiguous particle groups,
  // the partials added in group order (as k_bltc_sources); the divergence
  // uses the grid's leaf-box basis tg.lx / tg.ly
  const int qx = n1 * n1, G = blockDim.x / qx > 0 ? blockDim.x / qx : 1;
  const int per = (npl + G - 1) / G;
  for (int t = threadIdx.x; t < 2 * G * qx; t += blockDim.x) {
    const int fld = t / (G * qx), tt = t - fld * G * qx;
    const int gi = tt / qx, m = tt - gi * qx, a = m / n1, b = m % n1;
    const int k0 = gi * per, k1 = min(npl, k0 + per);
    double acc = 0;
    if (fld == 0)
      for (int k = k0; k < k1; k++) acc = fma(lx[k * n1 + a] * ly[k * n1 + b], sw[k], acc);
    else
      for (int k = k0; k < k1; k++) acc = fma(__ldg(tg.lx + k * n1 + a) * __ldg(tg.ly + k * n1 + b), sd[k], acc);
    part[t] = acc;
  }
  __syncthreads();
  for (int m = threadIdx.x; m < 2 * qx; m += blockDim.x) {
    const int fld = m / qx, mm = m - fld * qx;
    double acc = part[fld * G * qx + mm];
    for (int gi = 1; gi < G; gi++) acc += part[fld * G * qx + gi * qx + mm];
    (fld == 0 ? proxy : proxy2)[(long)panel * qx + mm].w = acc;
  }
}

// u = K x cross A - K (B - x (x.B)) (swe_kernels.cu's epilogue)
__device__ __forceinline__ void swe_tree_epilogue(double K, double tx, double ty, double tz, double ax, double ay,
                                                  double az, double bx, double by, double bz, double& ux, double& uy,
                                                  double& uz) {
  const double tb = tx * bx + ty * by + tz * bz;
  ux = K * (ty * az - tz * ay) - K * (bx - tx * tb);
  uy = K * (tz * ax - tx * az) - K * (by - ty * tb);
  uz = K * (tx * ay - ty * ax) - K * (bz - tz * tb);
}

// Near leaf pairs, both fields: one CTA of NT threads per (target leaf, source
// split), TPT targets per thread, the source leaf's particles of both fields
// staged in shared memory.  Split y takes every gridDim.y-th source leaf and
// writes the velocity of its partial sums to out + y 3N.  float64: pair64 on
// absolute positions.  Mixed: the paired float32 pair (pair32x2, two sources
// per instruction) with the sources packed relative to their own grid leaf
// (gq particles) and, per source grid leaf, the target's
// offset from that leaf's centre formed in float64 and rounded once, so that
// d' = (c_sub - t) kPackScale + (s - c_sub) kPackScale carries the rounding
// of grid-leaf-sized terms rather than tree-leaf-sized ones (the divergence
// tendency differentiates the velocity twice and amplifies that rounding);
// float32 sums per source grid leaf (two interleaved halves) added into
// float64.
template <int NT, int TPT, bool GUARD, bool MIXED>
__global__ void __launch_bounds__(NT)
    k_bltc_swe_near(TreeGeom tg, StepGeom fg, const double* __restrict__ x, const double* __restrict__ y,
                    const double* __restrict__ z, const double4* __restrict__ psrc, const double4* __restrict__ psrc2,
                    const float4* __restrict__ psrcf, const float4* __restrict__ psrcf2, double* __restrict__ out,
                    const double* __restrict__ gcentre, int gq) {
  using Src = typename std::conditional<MIXED, float4, double4>::type;
  extern __shared__ __align__(16) unsigned char smem[];
  Src* t1 = reinterpret_cast<Src*>(smem);
  Src* t2 = t1 + tg.npl;
  const int f = blockIdx.x, split = blockIdx.y, nsplit = gridDim.y, npl = tg.npl;
  double* v = out + (long)split * 3 * tg.N;
  // float64: the targets' positions; mixed: their packed positions t k as
  // float pairs hi + lo (t k to within u^2), so that the offset from a grid
  // leaf's centre c, (c - t) k, forms in float32 as (C_hi - T_hi) + (C_lo -
  // T_lo) with the rounding of the offset itself (no float64 conversions in
  // the source loop, which would share the reciprocals' pipe)
  constexpr int TD = MIXED ? 1 : TPT, TF = MIXED ? TPT : 1;
  double tx[TD], ty[TD], tz[TD];
  float2 nt[3][TF];
  double ax[TPT], ay[TPT], az[TPT], bx[TPT], by[TPT], bz[TPT];
#pragma unroll
  for (int r = 0; r < TPT; r++) {
    const int k = threadIdx.x + r * NT;
    const long i = (long)f * npl + (k < npl ? k : 0);
    if constexpr (MIXED) {
      const double p[3] = {x[i] * kPackScale, y[i] * kPackScale, z[i] * kPackScale};
#pragma unroll
      for (int c = 0; c < 3; c++) {
        const float hi = (float)p[c], lo = (float)(p[c] - (double)hi);
        nt[c][r] = make_float2(-hi, -lo);
      }
    } else {
      tx[r] = x[i];
      ty[r] = y[i];
      tz[r] = z[i];
    }
    ax[r] = ay[r] = az[r] = bx[r] = by[r] = bz[r] = 0;
  }
  const float feps = (float)tg.eps;
  const int hq = (gq + 1) / 2, ngl = npl / gq, np2 = ngl * hq;
  for (int e = tg.near_start[f] + split; e < tg.near_start[f + 1]; e += nsplit) {
    const int sl = tg.near_src[e];
    const long sb = (long)sl * npl;
    __syncthreads();
    if constexpr (MIXED) {
      // both fields' sources two at a time, transposed so that every operand
      // of the pair arithmetic is a register pair (x0,x1,y0,y1),(z0,z1,w0,w1)
      // for the paired float32 instructions (pair32x2); each grid leaf takes
      // hq = ceil(gq/2) pairs, an odd gq closing on a source of zero strength
      // at the grid leaf's centre (which adds exactly zero); after them the
      // grid leaves' packed centres c k as (x_hi, x_lo, y_hi, y_lo),
      // (z_hi, z_lo, -, -)
      float4* tp = reinterpret_cast<float4*>(smem);
      const float4 none = make_float4(0.f, 0.f, 0.f, 0.f);
      for (int p = threadIdx.x; p < np2; p += NT) {
        const int gl = p / hq, j = p - gl * hq;
        const long s0 = sb + (long)gl * gq + 2 * j;
        const bool two = 2 * j + 1 < gq;
        const float4 a0 = psrcf[s0], a1 = two ? psrcf[s0 + 1] : none;
        const float4 c0 = psrcf2[s0], c1 = two ? psrcf2[s0 + 1] : none;
        tp[4 * p] = make_float4(a0.x, a1.x, a0.y, a1.y);
        tp[4 * p + 1] = make_float4(a0.z, a1.z, a0.w, a1.w);
        tp[4 * p + 2] = make_float4(c0.x, c1.x, c0.y, c1.y);
        tp[4 * p + 3] = make_float4(c0.z, c1.z, c0.w, c1.w);
      }
      for (int gl = threadIdx.x; gl < ngl; gl += NT) {
        const double* cs = gcentre + 4 * (sb / gq + gl);
        float hl[6];
#pragma unroll
        for (int c = 0; c < 3; c++) {
          const double pc = cs[c] * kPackScale;
          hl[2 * c] = (float)pc;
          hl[2 * c + 1] = (float)(pc - (double)hl[2 * c]);
        }
        tp[4 * np2 + 2 * gl] = make_float4(hl[0], hl[1], hl[2], hl[3]);
        tp[4 * np2 + 2 * gl + 1] = make_float4(hl[4], hl[5], 0.f, 0.f);
      }
    } else {
      for (int k = threadIdx.x; k < npl; k += NT) {
        t1[k] = psrc[sb + k];
        t2[k] = psrc2[sb + k];
      }
    }
    __syncthreads();
    if constexpr (MIXED) {
      const float4* tp = reinterpret_cast<const float4*>(smem);
      const float2 eps2 = make_float2(feps, feps);
      for (int gl = 0; gl < ngl; gl++) {
        const float4 C0 = tp[4 * np2 + 2 * gl], C1 = tp[4 * np2 + 2 * gl + 1];
        const float2 cc[3] = {make_float2(C0.x, C0.y), make_float2(C0.z, C0.w), make_float2(C1.x, C1.y)};
        float2 bq[3][TPT], fa[TPT][3], fb[TPT][3];
#pragma unroll
        for (int r = 0; r < TPT; r++) {
#pragma unroll
          for (int c = 0; c < 3; c++) {
            const float2 dd = __fadd2_rn(cc[c], nt[c][r]);
            const float bc = dd.x + dd.y;
            bq[c][r] = make_float2(bc, bc);
          }
          fa[r][0] = fa[r][1] = fa[r][2] = fb[r][0] = fb[r][1] = fb[r][2] = make_float2(0.f, 0.f);
        }
#pragma unroll 4
        for (int p = gl * hq; p < (gl + 1) * hq; p++) {
          const float4 A = tp[4 * p], B = tp[4 * p + 1], C = tp[4 * p + 2], D = tp[4 * p + 3];
#pragma unroll
          for (int r = 0; r < TPT; r++) {
            pair32x2<GUARD>(bq[0][r], bq[1][r], bq[2][r], make_float2(A.x, A.y), make_float2(A.z, A.w),
                            make_float2(B.x, B.y), make_float2(B.z, B.w), eps2, fa[r][0], fa[r][1], fa[r][2]);
            pair32x2<GUARD>(bq[0][r], bq[1][r], bq[2][r], make_float2(C.x, C.y), make_float2(C.z, C.w),
                            make_float2(D.x, D.y), make_float2(D.z, D.w), eps2, fb[r][0], fb[r][1], fb[r][2]);
          }
        }
#pragma unroll
        for (int r = 0; r < TPT; r++) {
          ax[r] += (double)(fa[r][0].x + fa[r][0].y);
          ay[r] += (double)(fa[r][1].x + fa[r][1].y);
          az[r] += (double)(fa[r][2].x + fa[r][2].y);
          bx[r] += (double)(fb[r][0].x + fb[r][0].y);
          by[r] += (double)(fb[r][1].x + fb[r][1].y);
          bz[r] += (double)(fb[r][2].x + fb[r][2].y);
        }
      }
    } else {
#pragma unroll 4
      for (int k = 0; k < npl; k++) {
        const double4 s1 = t1[k], s2 = t2[k];
#pragma unroll
        for (int r = 0; r < TPT; r++) {
          pair64<GUARD>(tx[r], ty[r], tz[r], s1, tg.eps, ax[r], ay[r], az[r]);
          pair64<GUARD>(tx[r], ty[r], tz[r], s2, tg.eps, bx[r], by[r], bz[r]);
        }
      }
    }
  }
  constexpr double K = MIXED ? kBiotSavartPacked : kBiotSavart;
#pragma unroll
  for (int r = 0; r < TPT; r++) {
    const int k = threadIdx.x + r * NT;
    if (k >= npl) continue;
    const long i = (long)f * npl + k;
    double ux, uy, uz;
    swe_tree_epilogue(K, x[i], y[i], z[i], ax[r], ay[r], az[r], bx[r], by[r], bz[r], ux, uy, uz);
    v[i] = ux;
    v[tg.N + i] = uy;
    v[2 * tg.N + i] = uz;
  }
}

// Well-separated pairs of both fields, mixed precision, over chunks of the
// interaction list: the BVE treecode's chunks of at most C consecutive
// entries of one target panel, S chunk slots of Q target proxies per block
// (thread k: target proxy k % Q of slot k / Q).  Per entry a slot stages the
// source panel's Q proxies of both fields as ceil(Q/2) source pairs (an odd
// Q closing on a zero-strength proxy at the panel's centre) and every thread
// runs them on the paired float32 instructions against its target proxy;
// each source panel's float32 sums are added into float64.  A slot writes
// its chunk's raw sums of both fields (6 rows of Q) to its own row of
// partial; k_swe_cc_reduce adds a target's chunks in list order and applies
// the SWE epilogue.  Against one warp per target panel (k_swe_interact, 81
// of 96 lanes busy at Q = 81) the slots keep the lanes busy and spread long
// lists over the GPU.
template <int Q, int S>
struct SweCcShape {
  static constexpr int NT = (S * Q + 31) / 32 * 32;
  static constexpr int Q2 = (Q + 1) / 2;
};

template <int Q, int S, bool GUARD>
__global__ void __launch_bounds__(SweCcShape<Q, S>::NT)
    k_swe_cc32(StepGeom g, const float4* __restrict__ srcf2, const int4* __restrict__ chunks, int nchunks,
               double* __restrict__ partial) {
  constexpr int Q2 = SweCcShape<Q, S>::Q2;
  __shared__ float4 tile[S][2][2 * Q2];  // per field (x0,x1,y0,y1),(z0,z1,w0,w1)
  const int h = threadIdx.x / Q, j = threadIdx.x - h * Q;
  const int c = blockIdx.x * S + h;
  const bool live = h < S && c < nchunks;
  int nmax = 0;  // the block's longest chunk: every thread passes the same barriers
  for (int k = 0; k < S && blockIdx.x * S + k < nchunks; k++) {
    const int4 ck = chunks[blockIdx.x * S + k];
    nmax = max(nmax, ck.z - ck.y);
  }
  const int4 ch = live ? chunks[c] : make_int4(0, 0, 0, 0);
  const int n = ch.z - ch.y;
  const long pn = (long)g.panels * Q;
  double cx = 0, cy = 0, cz = 0;
  float dtx = 0, dty = 0, dtz = 0;
  if (live) {
    const double* ct = g.pd_centre + 4 * (long)ch.x;
    cx = ct[0];
    cy = ct[1];
    cz = ct[2];
    const long o = (long)ch.x * Q + j;
    dtx = (float)((g.px[o] - cx) * kPackScale);
    dty = (float)((g.px[pn + o] - cy) * kPackScale);
    dtz = (float)((g.px[2 * pn + o] - cz) * kPackScale);
  }
  const float feps = (float)g.eps;
  const float2 eps2 = make_float2(feps, feps);
  double ax = 0, ay = 0, az = 0, bx = 0, by = 0, bz = 0;
  for (int e = 0; e < nmax; e++) {
    const bool act = live && e < n;
    const int sp = act ? __ldg(g.src_panel + ch.y + e) : 0;
    __syncthreads();
    if (act && j < Q2) {
      const long sb = (long)sp * Q + 2 * j;
      const bool two = 2 * j + 1 < Q;
      const float4 none = make_float4(0.f, 0.f, 0.f, 0.f);
      const float4 a0 = g.srcf[sb], a1 = two ? g.srcf[sb + 1] : none;
      const float4 c0 = srcf2[sb], c1 = two ? srcf2[sb + 1] : none;
      tile[h][0][2 * j] = make_float4(a0.x, a1.x, a0.y, a1.y);
      tile[h][0][2 * j + 1] = make_float4(a0.z, a1.z, a0.w, a1.w);
      tile[h][1][2 * j] = make_float4(c0.x, c1.x, c0.y, c1.y);
      tile[h][1][2 * j + 1] = make_float4(c0.z, c1.z, c0.w, c1.w);
    }
    __syncthreads();
    if (act) {
      const double* cs = g.pd_centre + 4 * (long)sp;
      const float b0 = (float)((cs[0] - cx) * kPackScale) - dtx, b1 = (float)((cs[1] - cy) * kPackScale) - dty,
                  b2 = (float)((cs[2] - cz) * kPackScale) - dtz;
      const float2 px2 = make_float2(b0, b0), py2 = make_float2(b1, b1), pz2 = make_float2(b2, b2);
      float2 fa[3], fb[3];
      fa[0] = fa[1] = fa[2] = fb[0] = fb[1] = fb[2] = make_float2(0.f, 0.f);
      const float4* t1 = tile[h][0];
      const float4* t2 = tile[h][1];
#pragma unroll 4
      for (int k2 = 0; k2 < Q2; k2++) {
        const float4 A = t1[2 * k2], B = t1[2 * k2 + 1], C = t2[2 * k2], D = t2[2 * k2 + 1];
        pair32x2<GUARD>(px2, py2, pz2, make_float2(A.x, A.y), make_float2(A.z, A.w), make_float2(B.x, B.y),
                        make_float2(B.z, B.w), eps2, fa[0], fa[1], fa[2]);
        pair32x2<GUARD>(px2, py2, pz2, make_float2(C.x, C.y), make_float2(C.z, C.w), make_float2(D.x, D.y),
                        make_float2(D.z, D.w), eps2, fb[0], fb[1], fb[2]);
      }
      ax += (double)(fa[0].x + fa[0].y);
      ay += (double)(fa[1].x + fa[1].y);
      az += (double)(fa[2].x + fa[2].y);
      bx += (double)(fb[0].x + fb[0].y);
      by += (double)(fb[1].x + fb[1].y);
      bz += (double)(fb[2].x + fb[2].y);
    }
  }
  if (live) {
    double* p = partial + (long)c * 6 * Q;
    p[j] = ax;
    p[Q + j] = ay;
    p[2 * Q + j] = az;
    p[3 * Q + j] = bx;
    p[4 * Q + j] = by;
    p[5 * Q + j] = bz;
  }
}

// Each target proxy's chunk sums in list order, then the SWE epilogue with
// the packed kernel constant (the sums are over packed differences).
__global__ void k_swe_cc_reduce(StepGeom g, const int* __restrict__ cstart, const double* __restrict__ partial,
                                double* __restrict__ out) {
  const int q = g.q;
  const long pn = (long)g.panels * q;
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= pn) return;
  const int t = (int)(i / q), j = (int)(i - (long)t * q);
  double a[6] = {0, 0, 0, 0, 0, 0};
  for (int c = cstart[t]; c < cstart[t + 1]; c++) {
    const double* p = partial + (long)c * 6 * q + j;
#pragma unroll
    for (int r = 0; r < 6; r++) a[r] += p[r * q];
  }
  double ux, uy, uz;
  swe_tree_epilogue(kBiotSavartPacked, g.px[i], g.px[pn + i], g.px[2 * pn + i], a[0], a[1], a[2], a[3], a[4], a[5],
                    ux, uy, uz);
  out[i] = ux;
  out[pn + i] = uy;
  out[2 * pn + i] = uz;
}

}  // namespace

void launch_bltc_swe_sources(const TreeGeom& tg, const StepGeom& fg, const BliTable& tab, int stage, double dtd,
                             double dts, const double* vprev, const double* tprev, const double* x, const double* y,
                             const double* z, const double* vors, const double* divs, const double* area,
                             const double* dispx, const double* dispy, const double* dispz, const double* wv,
                             const double* wd, double4* psrc, float4* psrcf,
                             double4* psrc2, float4* psrcf2, double4* proxy, double4* proxy2, bool mixed,
                             const double* gcentre, int gq, cudaStream_t st) {
  const int n1 = tg.n + 1, qx = n1 * n1, G = kThreads / qx > 0 ? kThreads / qx : 1;
  const size_t smem = sizeof(double) * ((size_t)tg.npl * n1 * 2 + 2 * (size_t)tg.npl + 2 * (size_t)G * qx);
  static std::atomic<unsigned long long> attr{0};
  raise_smem_once(attr, 200 * 1024, k_bltc_swe_sources);
  SB_LAUNCH(k_bltc_swe_sources, (unsigned)fg.leaves, kThreads, smem, st, tg, fg, tab, stage, dtd, dts, vprev, tprev,
            x, y, z, vors, divs, area, dispx, dispy, dispz, wv, wd, psrc, psrcf, psrc2, psrcf2, proxy, proxy2,
            mixed ? 1 : 0, gcentre, gq);
}

void launch_bltc_swe_near(const TreeGeom& tg, const StepGeom& fg, int precision, const double* x, const double* y,
                          const double* z, const double4* psrc, const double4* psrc2, const float4* psrcf,
                          const float4* psrcf2, double* near, int splits, const double* gcentre, int gq,
                          cudaStream_t st) {
  const dim3 grid((unsigned)fg.leaves, (unsigned)splits);
  const bool guard = !(tg.eps > 0), mixed = precision == SBSLPM_MIXED;
  constexpr int NT = 128;
  const int tpt = (tg.npl + NT - 1) / NT;
  // mixed: four float4 per source pair, ceil(gq/2) pairs per grid leaf, and
  // two float4 per grid leaf for its centre
  const size_t smem = mixed ? sizeof(float4) * (size_t)(tg.npl / gq) * (4 * ((gq + 1) / 2) + 2)
                            : sizeof(double4) * 2 * (size_t)tg.npl;
#define SB_SN(TPT)                                                                                                \
  do {                                                                                                            \
    if (mixed) {                                                                                                  \
      if (guard) SB_LAUNCH((k_bltc_swe_near<NT, TPT, true, true>), grid, NT, smem, st, tg, fg, x, y, z, psrc,     \
                           psrc2, psrcf, psrcf2, near, gcentre, gq);                                              \
      else SB_LAUNCH((k_bltc_swe_near<NT, TPT, false, true>), grid, NT, smem, st, tg, fg, x, y, z, psrc, psrc2,   \
                     psrcf, psrcf2, near, gcentre, gq);                                                           \
    } else {                                                                                                      \
      if (guard) SB_LAUNCH((k_bltc_swe_near<NT, TPT, true, false>), grid, NT, smem, st, tg, fg, x, y, z, psrc,    \
                           psrc2, psrcf, psrcf2, near, gcentre, gq);                                              \
      else SB_LAUNCH((k_bltc_swe_near<NT, TPT, false, false>), grid, NT, smem, st, tg, fg, x, y, z, psrc, psrc2,  \
                     psrcf, psrcf2, near, gcentre, gq);                                                           \
    }                                                                                                             \
  } while (0)
  // the shallow-water context refuses leaves of more than 256 particles, so
  // two targets per thread of 128 cover every leaf
  if (tpt <= 1) SB_SN(1);
  else SB_SN(2);
#undef SB_SN
}

bool swe_tree_cc_supported(int q) { return q == 36 || q == 49 || q == 64 || q == 81 || q == 100 || q == 121; }

// Slots per block for each proxy count: at most a few lanes of the block idle
// (36: 7 x 36 of 256, 49: 5 x 49 of 256, 64: 2 x 64 of 128, 81: 3 x 81 of
// 256, 100: 5 x 100 of 512, 121: 2 x 121 of 256).
void launch_swe_tree_cc(const StepGeom& fg, const float4* srcf2, const int4* chunks, int nchunks, const int* cstart,
                        double* partial, double* tgt, cudaStream_t st) {
  const bool guard = !(fg.eps > 0);
  if (nchunks > 0) {
#define SB_SCC(Q, S)                                                                                           \
  case Q:                                                                                                      \
    if (guard)                                                                                                 \
      SB_LAUNCH((k_swe_cc32<Q, S, true>), (unsigned)((nchunks + S - 1) / S), (SweCcShape<Q, S>::NT), 0, st, fg, \
                srcf2, chunks, nchunks, partial);                                                              \
    else                                                                                                       \
      SB_LAUNCH((k_swe_cc32<Q, S, false>), (unsigned)((nchunks + S - 1) / S), (SweCcShape<Q, S>::NT), 0, st,   \
                fg, srcf2, chunks, nchunks, partial);                                                          \
    break;
    switch (fg.q) {
      SB_SCC(36, 7)
      SB_SCC(49, 5)
      SB_SCC(64, 2)
      SB_SCC(81, 3)
      SB_SCC(100, 5)
      SB_SCC(121, 2)
      default:
        break;
    }
#undef SB_SCC
  }
  const long pn = (long)fg.panels * fg.q;
  SB_LAUNCH(k_swe_cc_reduce, blocks_for(pn, 256), 256, 0, st, fg, cstart, partial, tgt);
}

}  // namespace sbslpm
