// Treecode velocity with decoupled proxy degree (proxy_degree > 0), sm_100a.
//
// The particle grid is the reference's (levels, interp_degree); the treecode
// runs on the same cubed-sphere quadtree truncated at the level whose panels
// hold at most leaf_size particles.  Every treecode panel carries
// (n+1)^2 fixed Chebyshev proxy points of degree n.  Per velocity evaluation:
//
//   k_bltc_sources     one CTA per treecode leaf: displaced particle sources
//                      (as bve_disp_update, src/bve_time_step.cpp:69-105) and
//                      their anterpolation onto the leaf's proxies (BLI at the
//                      displaced positions, as base_pots_ll,
//                      src/fmm_funcs_impl.hpp:190-222, with displaced points)
//   upward pass        k_upward_subtree, mode 2, on the proxies
//   k_bltc_near        near leaf pairs, particle x particle
//   proxy interactions k_interact64/32 on every well-separated pair, proxy x
//                      proxy (cc of swe_vel_panel_interaction_ll,
//                      src/fmm_interactions/swe_vel_impl.hpp:149-288)
//   downward pass      k_downward_subtree on the proxies
//   k_bltc_to_particles leaf proxies -> particles (tensor-product BLI with the
//                      leaf-box basis of the particle grid, as
//                      child_panel_interp_3_ll, src/fmm_funcs_impl.hpp:312-364)
//
// Particles of one treecode leaf are contiguous in the [leaf panel][q]
// arrays (the leaf's descendants are consecutive panels), so the kernels
// read them as one block.
#include <cuda_runtime.h>

#include "../../include/sbslpm.h"
#include "bve_kernels.cuh"
#include "device_common.cuh"

namespace sbslpm {

namespace {

using namespace dev;

constexpr int kThreads = 256;

// Barycentric Lagrange basis of degree n on Chebyshev extrema of [lo, hi]
// without the reference's range check: displaced sources may sit slightly
// outside their leaf, where the interpolant extrapolates smoothly.  The
// second barycentric form multiplied through by prod_j (t - c_j):
// f_i = w_i P_i / sum_k w_k P_k with P_i = prod_{j != i} (t - c_j), one
// division instead of n + 2 (nodes within 1e-15 are hit exactly).
__device__ __forceinline__ void bli_1d_free(double t, double lo, double hi, int n, const double* cosv,
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

__device__ __forceinline__ void bltc_sources_body(const TreeGeom& tg, const StepGeom& fg, const BliTable& tab, int f,
                                                  int stage, double dt_s, const double* __restrict__ vprev,
                                                  const double* __restrict__ x, const double* __restrict__ y,
                                                  const double* __restrict__ z, const double* __restrict__ vors,
                                                  const double* __restrict__ area, double4* __restrict__ psrc,
                                                  float4* __restrict__ psrcf, double4* __restrict__ proxy,
                                                  int mixed) {
  extern __shared__ double sh[];
  const int n1 = tg.n + 1, npl = tg.npl;
  double* lx = sh;              // [npl][n1]
  double* ly = lx + npl * n1;   // [npl][n1]
  double* sw = ly + npl * n1;   // [npl]
  const int panel = fg.offset + f;
  const double* bd = tg.fbounds + 4 * panel;
  const int face = tg.fface[panel];
  const double* cc = fg.pd_centre + 4 * (long)panel;
  const long N = tg.N;
  for (int k = threadIdx.x; k < npl; k += blockDim.x) {
    const long i = (long)f * npl + k;
    double xx = x[i], yy = y[i], zz = z[i], w;
    if (stage == 0) {
      w = area[i] * (fg.force ? vors[i] + fg.force[i] : vors[i]);
    } else {
      const double vx = vprev[i], vy = vprev[N + i], vz = vprev[2 * N + i];
      xx += vx * dt_s;
      yy += vy * dt_s;
      zz += vz * dt_s;
      project_to_sphere(xx, yy, zz);
      const double dvor = vors[i] + 2 * tg.omega * z[i] - 2 * tg.omega * zz;
      w = area[i] * (fg.force ? dvor + fg.force[i] : dvor);
    }
    if (stage == 0) project_to_sphere(xx, yy, zz);
    psrc[i] = make_double4(xx, yy, zz, w);
    if (mixed)
      psrcf[i] = make_float4((float)((xx - cc[0]) * kPackScale), (float)((yy - cc[1]) * kPackScale),
                             (float)((zz - cc[2]) * kPackScale), (float)w);
    double xi, eta;
    xieta_from_xyz_face(xx, yy, zz, face, xi, eta);
    bli_1d_free(xi, bd[0], bd[1], tg.n, tab.cosv, tab.w, lx + k * n1);
    bli_1d_free(eta, bd[2], bd[3], tg.n, tab.cosv, tab.w, ly + k * n1);
    sw[k] = w;
  }
  __syncthreads();
  // proxy strengths S[a][b] = sum_k lx[k][a] ly[k][b] w_k: the particles are
  // cut into G contiguous groups (G = threads / q), one thread per (group,
  // proxy), and the G partial sums are added in group order
  const int qx = n1 * n1, G = blockDim.x / qx > 0 ? blockDim.x / qx : 1;
  double* part = sw + npl;  // [G][qx]
  const int per = (npl + G - 1) / G;
  for (int t = threadIdx.x; t < G * qx; t += blockDim.x) {
    const int gi = t / qx, m = t - gi * qx, a = m / n1, b = m % n1;
    const int k0 = gi * per, k1 = min(npl, k0 + per);
    double acc = 0;
    for (int k = k0; k < k1; k++) acc = fma(lx[k * n1 + a] * ly[k * n1 + b], sw[k], acc);
    part[t] = acc;
  }
  __syncthreads();
  for (int m = threadIdx.x; m < qx; m += blockDim.x) {
    double acc = part[m];
    for (int gi = 1; gi < G; gi++) acc += part[gi * qx + m];
    proxy[(long)panel * qx + m].w = acc;
  }
}

__global__ void __launch_bounds__(kThreads)
    k_bltc_sources(TreeGeom tg, StepGeom fg, BliTable tab, int stage, double dt_s, const double* __restrict__ vprev,
                   const double* __restrict__ x, const double* __restrict__ y, const double* __restrict__ z,
                   const double* __restrict__ vors, const double* __restrict__ area, double4* __restrict__ psrc,
                   float4* __restrict__ psrcf, double4* __restrict__ proxy, int mixed) {
  bltc_sources_body(tg, fg, tab, blockIdx.x, stage, dt_s, vprev, x, y, z, vors, area, psrc, psrcf, proxy, mixed);
}

// Batched members (member blockIdx.y) on one particle grid.
__global__ void __launch_bounds__(kThreads)
    k_bltc_sources_batch(const BatchMember* __restrict__ mem, int stage, double dt_s, const double* __restrict__ vprev,
                         const double* __restrict__ x, const double* __restrict__ y, const double* __restrict__ z,
                         const double* __restrict__ vors, const double* __restrict__ area,
                         double4* __restrict__ psrc, float4* __restrict__ psrcf, int mixed) {
  const BatchMember& m = mem[blockIdx.y];
  const TreeGeom tg = m.tg;
  const StepGeom fg = m.fg;
  const long N = tg.N, mo = (long)blockIdx.y;
  bltc_sources_body(tg, fg, m.tab, blockIdx.x, stage, dt_s, vprev ? vprev + mo * 3 * N : nullptr, x, y, z,
                    vors + mo * N, area, psrc + mo * N, psrcf ? psrcf + mo * N : nullptr, m.fsrc, mixed);
}

// Near leaf pairs: one CTA of NT threads per (target leaf, source split),
// TPT targets per thread (NT * TPT >= particles per leaf), the source leaf's
// particles staged in shared memory and read back as broadcasts.  Split y of
// gridDim.y takes every gridDim.y-th source leaf and writes its partial sums
// to out + y * 3N (the splits even out the work across SMs);
// k_bltc_to_particles adds them in split order.
template <int NT, int TPT, bool GUARD>
__device__ __forceinline__ void bltc_near64_body(const TreeGeom& tg, int f, int split, int nsplit,
                                                 const double* __restrict__ x, const double* __restrict__ y,
                                                 const double* __restrict__ z, const double4* __restrict__ psrc,
                                                 double* __restrict__ out) {
  double* v = out + (long)split * 3 * tg.N;  // partial sums of this source split
  extern __shared__ double4 tile[];
  const int npl = tg.npl;
  double tx[TPT], ty[TPT], tz[TPT], ax[TPT], ay[TPT], az[TPT];
#pragma unroll
  for (int r = 0; r < TPT; r++) {
    int k = threadIdx.x + r * NT;
    long i = (long)f * npl + (k < npl ? k : 0);
    tx[r] = x[i];
    ty[r] = y[i];
    tz[r] = z[i];
    ax[r] = ay[r] = az[r] = 0;
  }
  const double eps = tg.eps;
  for (int e = tg.near_start[f] + split; e < tg.near_start[f + 1]; e += nsplit) {
    const long sb = (long)tg.near_src[e] * npl;
    __syncthreads();
    for (int k = threadIdx.x; k < npl; k += NT) tile[k] = psrc[sb + k];
    __syncthreads();
#pragma unroll 8
    for (int k = 0; k < npl; k++) {
      const double4 s = tile[k];
#pragma unroll
      for (int r = 0; r < TPT; r++) {
        double dx = s.x - tx[r], dy = s.y - ty[r], dz = s.z - tz[r];
        double r2 = fma(dx, dx, fma(dy, dy, dz * dz));
        double g = s.w * recip_nr(fma(0.5, r2, eps));
        if (GUARD) g = r2 > 0.0 ? g : 0.0;
        ax[r] = fma(g, dx, ax[r]);
        ay[r] = fma(g, dy, ay[r]);
        az[r] = fma(g, dz, az[r]);
      }
    }
  }
#pragma unroll
  for (int r = 0; r < TPT; r++) {
    int k = threadIdx.x + r * NT;
    if (k >= npl) continue;
    long i = (long)f * npl + k;
    v[i] = kBiotSavart * (ty[r] * az[r] - tz[r] * ay[r]);
    v[tg.N + i] = kBiotSavart * (tz[r] * ax[r] - tx[r] * az[r]);
    v[2 * tg.N + i] = kBiotSavart * (tx[r] * ay[r] - ty[r] * ax[r]);
  }
}

// Batched members (member blockIdx.z): sources psrc + m N, partials out + m splits 3N.
template <int NT, int TPT, bool GUARD>
__global__ void __launch_bounds__(NT)
    k_bltc_near64_batch(const BatchMember* __restrict__ mem, const double* __restrict__ x,
                        const double* __restrict__ y, const double* __restrict__ z,
                        const double4* __restrict__ psrc, double* __restrict__ out) {
  const TreeGeom tg = mem[blockIdx.z].tg;
  const long mo = blockIdx.z;
  bltc_near64_body<NT, TPT, GUARD>(tg, tg.leaf0 + blockIdx.x, blockIdx.y, gridDim.y, x, y, z, psrc + mo * tg.N,
                                   out + mo * gridDim.y * 3 * tg.N);
}

// Mixed precision: target and source particles relative to their leaves'
// centres (scaled by kPackScale), float32 pairs, per-source-leaf float32
// sums added into float64.  Sources are staged two at a time, transposed as
// (x0,x1,y0,y1),(z0,z1,w0,w1), so that every operand of the pair arithmetic
// is a register pair and the paired FP32 instructions of sm_100
// (FADD2 / FFMA2 / FMUL2) evaluate two pairs per instruction; a missing
// partner of an odd source count has zero strength (pair32x2).  EXP: the
// expanded form (pair32x2_expanded), sources staged as four float4 per two.
template <int NT, int TPT, bool GUARD, bool EXP>
__device__ __forceinline__ void bltc_near32_body(const TreeGeom& tg, const StepGeom& fg, int f, int split,
                                                 int nsplit, const double* __restrict__ x,
                                                 const double* __restrict__ y, const double* __restrict__ z,
                                                 const float4* __restrict__ psrcf, double* __restrict__ out) {
  static_assert(!(GUARD && EXP), "the expanded form needs eps > 0");
  double* v = out + (long)split * 3 * tg.N;  // partial sums of this source split
  extern __shared__ float4 tilef[];  // [(npl+1)/2][EXP ? 4 : 2]
  const int npl = tg.npl, npl2 = (npl + 1) >> 1;
  const double* ct = fg.pd_centre + 4 * (long)(fg.offset + f);
  const double cx = ct[0], cy = ct[1], cz = ct[2];
  // target positions are re-read for the final cross product, so only their
  // packed offsets stay in registers
  double ax[TPT], ay[TPT], az[TPT];
  float dtx[TPT], dty[TPT], dtz[TPT];
#pragma unroll
  for (int r = 0; r < TPT; r++) {
    int k = threadIdx.x + r * NT;
    long i = (long)f * npl + (k < npl ? k : 0);
    dtx[r] = (float)((x[i] - cx) * kPackScale);
    dty[r] = (float)((y[i] - cy) * kPackScale);
    dtz[r] = (float)((z[i] - cz) * kPackScale);
    ax[r] = ay[r] = az[r] = 0;
  }
  const float feps = (float)tg.eps;
  const float2 eps2 = make_float2(feps, feps);
  for (int e = tg.near_start[f] + split; e < tg.near_start[f + 1]; e += nsplit) {
    const int sl = tg.near_src[e];
    const long sb = (long)sl * npl;
    const double* cs = fg.pd_centre + 4 * (long)(fg.offset + sl);
    const float bx0 = (float)((cs[0] - cx) * kPackScale), by0 = (float)((cs[1] - cy) * kPackScale),
                bz0 = (float)((cs[2] - cz) * kPackScale);
    __syncthreads();
    for (int k2 = threadIdx.x; k2 < npl2; k2 += NT) {
      if constexpr (EXP) {
        dev::stage_expanded(psrcf + sb, k2, npl, feps, tilef + 4 * k2);
      } else {
        const float4 s0 = psrcf[sb + 2 * k2];
        const float4 s1 = (2 * k2 + 1 < npl) ? psrcf[sb + 2 * k2 + 1] : make_float4(0.f, 0.f, 0.f, 0.f);
        tilef[2 * k2] = make_float4(s0.x, s1.x, s0.y, s1.y);
        tilef[2 * k2 + 1] = make_float4(s0.z, s1.z, s0.w, s1.w);
      }
    }
    __syncthreads();
    float2 fx[TPT], fy[TPT], fz[TPT], fw[TPT], bx[TPT], by[TPT], bz[TPT], bb[TPT];
#pragma unroll
    for (int r = 0; r < TPT; r++) {
      fx[r] = fy[r] = fz[r] = fw[r] = make_float2(0.f, 0.f);
      const float b0 = bx0 - dtx[r], b1 = by0 - dty[r], b2 = bz0 - dtz[r];
      if constexpr (EXP) {  // m = 2b (exact), |b|^2
        bx[r] = make_float2(2.f * b0, 2.f * b0);
        by[r] = make_float2(2.f * b1, 2.f * b1);
        bz[r] = make_float2(2.f * b2, 2.f * b2);
        const float q = fmaf(b0, b0, fmaf(b1, b1, b2 * b2));
        bb[r] = make_float2(q, q);
      } else {
        bx[r] = make_float2(b0, b0);
        by[r] = make_float2(b1, b1);
        bz[r] = make_float2(b2, b2);
      }
    }
    // unrolled 8 deep (measured: 2.4% faster than 4 for the 128 x 2 shape on the
    // 393,216-particle treecode, 16 no better, 2 slower), registers permitting
#pragma unroll 8
    for (int k2 = 0; k2 < npl2; k2++) {
      if constexpr (EXP) {
        const float4 A = tilef[4 * k2], B = tilef[4 * k2 + 1], C = tilef[4 * k2 + 2], D = tilef[4 * k2 + 3];
#pragma unroll
        for (int r = 0; r < TPT; r++)
          dev::pair32x2_expanded(bx[r], by[r], bz[r], bb[r], A, B, C, D, fx[r], fy[r], fz[r], fw[r]);
      } else {
        const float4 A = tilef[2 * k2], B = tilef[2 * k2 + 1];
        const float2 sx = make_float2(A.x, A.y), sy = make_float2(A.z, A.w), sz = make_float2(B.x, B.y),
                     sw = make_float2(B.z, B.w);
#pragma unroll
        for (int r = 0; r < TPT; r++)
          pair32x2<GUARD>(bx[r], by[r], bz[r], sx, sy, sz, sw, eps2, fx[r], fy[r], fz[r]);
      }
    }
#pragma unroll
    for (int r = 0; r < TPT; r++) {
      ax[r] += (double)fx[r].x + (double)fx[r].y;
      ay[r] += (double)fy[r].x + (double)fy[r].y;
      az[r] += (double)fz[r].x + (double)fz[r].y;
      if constexpr (EXP) {  // + b sum r w, b = m / 2 exactly
        const double sw = (double)fw[r].x + (double)fw[r].y;
        ax[r] = fma(0.5 * (double)bx[r].x, sw, ax[r]);
        ay[r] = fma(0.5 * (double)by[r].x, sw, ay[r]);
        az[r] = fma(0.5 * (double)bz[r].x, sw, az[r]);
      }
    }
  }
#pragma unroll
  for (int r = 0; r < TPT; r++) {
    int k = threadIdx.x + r * NT;
    if (k >= npl) continue;
    long i = (long)f * npl + k;
    const double tx = x[i], ty = y[i], tz = z[i];
    v[i] = kBiotSavartPacked * (ty * az[r] - tz * ay[r]);
    v[tg.N + i] = kBiotSavartPacked * (tz * ax[r] - tx * az[r]);
    v[2 * tg.N + i] = kBiotSavartPacked * (tx * ay[r] - ty * ax[r]);
  }
}

// 256-thread shapes are held to 64 registers (four blocks per SM): on the
// 393,216-particle treecode the (256 x 1) shape then ran 535 us per launch
// against 555 us uncapped; the smaller shapes of the difference form measured
// slower when capped, so they keep their registers.  The 128-thread shapes of
// the expanded form are held to 128 registers (four blocks per SM: 495.5 us
// per launch for 128 x 2 against 502.2 us at 138 registers).  The autotuner
// chooses among all of them.
template <int NT, int TPT, bool GUARD, bool EXP>
__global__ void __launch_bounds__(NT, NT >= 256 ? 4 : (EXP && NT == 128 ? 4 : 1))
    k_bltc_near32_batch(const BatchMember* __restrict__ mem, const double* __restrict__ x,
                        const double* __restrict__ y, const double* __restrict__ z,
                        const float4* __restrict__ psrcf, double* __restrict__ out) {
  const TreeGeom tg = mem[blockIdx.z].tg;
  const StepGeom fg = mem[blockIdx.z].fg;
  const long mo = blockIdx.z;
  bltc_near32_body<NT, TPT, GUARD, EXP>(tg, fg, tg.leaf0 + blockIdx.x, blockIdx.y, gridDim.y, x, y, z, psrcf + mo * tg.N,
                                   out + mo * gridDim.y * 3 * tg.N);
}

// The near field of the first RK stage for a group of MB members at once.
// At stage 0 every member's particles sit on the shared grid (only the
// strengths differ), so a leaf pair's differences, distances and
// reciprocals are member-independent: they are evaluated once and applied to
// the MB members' strengths with the paired float32 instructions across
// members (FMUL2 / FFMA2 over member pairs).  Members are grouped by sorted
// theta; a group walks the union of its members' near lists (entry = source
// leaf | member bits << 24), a member outside an entry's bits taking zero
// strength there.  Per member, per source leaf: float32 sums added into
// float64, partials per split as in the per-member kernel.
template <int NT, int MB, bool GUARD>
__global__ void __launch_bounds__(NT)
    k_bltc_near32_multi(const BatchMember* __restrict__ mem, const int* __restrict__ perm, int members,
                        const int* __restrict__ ustart, const int* __restrict__ uent, const double* __restrict__ x,
                        const double* __restrict__ y, const double* __restrict__ z, const float4* __restrict__ psrcf,
                        double* __restrict__ out) {
  extern __shared__ float4 tq[];  // [npl/2][2] paired positions, then [npl][MB] strengths
  const int f = blockIdx.x, split = blockIdx.y, nsplit = gridDim.y, grp = blockIdx.z;
  const int m0 = perm[grp * MB];
  const TreeGeom tg = mem[m0].tg;
  const StepGeom fg = mem[m0].fg;
  const int npl = tg.npl, npl2 = (npl + 1) >> 1, leaves = fg.leaves;
  const long N = tg.N;
  float* wt = reinterpret_cast<float*>(tq + 2 * npl2);
  int mid[MB];
#pragma unroll
  for (int j = 0; j < MB; j++) mid[j] = grp * MB + j < members ? perm[grp * MB + j] : -1;
  const int k = threadIdx.x;
  const bool tgt = k < npl;
  const double* ct = fg.pd_centre + 4 * (long)(fg.offset + f);
  const long ti = (long)f * npl + (tgt ? k : 0);
  const float dtx = (float)((x[ti] - ct[0]) * kPackScale), dty = (float)((y[ti] - ct[1]) * kPackScale),
              dtz = (float)((z[ti] - ct[2]) * kPackScale);
  double ax[MB], ay[MB], az[MB];
#pragma unroll
  for (int j = 0; j < MB; j++) ax[j] = ay[j] = az[j] = 0;
  const float feps = (float)tg.eps;
  const float2 eps2 = make_float2(feps, feps);
  const int* us = ustart + (long)grp * (leaves + 1);
  for (int e = us[f] + split; e < us[f + 1]; e += nsplit) {
    const unsigned ent = (unsigned)__ldg(uent + e);
    const int sl = (int)(ent & 0xffffffu), bits = (int)(ent >> 24);
    const double* cs = fg.pd_centre + 4 * (long)(fg.offset + sl);
    const float bx0 = (float)((cs[0] - ct[0]) * kPackScale), by0 = (float)((cs[1] - ct[1]) * kPackScale),
                bz0 = (float)((cs[2] - ct[2]) * kPackScale);
    const long sb = (long)sl * npl;
    __syncthreads();
    for (int kk = threadIdx.x; kk < npl2; kk += NT) {
      const float4 s0 = psrcf[(long)m0 * N + sb + 2 * kk];
      const float4 s1 = 2 * kk + 1 < npl ? psrcf[(long)m0 * N + sb + 2 * kk + 1] : make_float4(0.f, 0.f, 0.f, 0.f);
      tq[2 * kk] = make_float4(s0.x, s1.x, s0.y, s1.y);
      tq[2 * kk + 1] = make_float4(s0.z, s1.z, 0.f, 0.f);
    }
    for (int kk = threadIdx.x; kk < 2 * npl2; kk += NT) {
#pragma unroll
      for (int j = 0; j < MB; j++)
        wt[kk * MB + j] = (kk < npl && mid[j] >= 0 && ((bits >> j) & 1)) ? psrcf[(long)mid[j] * N + sb + kk].w : 0.f;
    }
    __syncthreads();
    if (tgt) {
      const float b0 = bx0 - dtx, b1 = by0 - dty, b2 = bz0 - dtz;
      const float2 bx = make_float2(b0, b0), by = make_float2(b1, b1), bz = make_float2(b2, b2);
      float2 fx[MB / 2], fy[MB / 2], fz[MB / 2];
#pragma unroll
      for (int p = 0; p < MB / 2; p++) fx[p] = fy[p] = fz[p] = make_float2(0.f, 0.f);
#pragma unroll 4
      for (int k2 = 0; k2 < npl2; k2++) {
        const float4 A = tq[2 * k2], B = tq[2 * k2 + 1];
        const float2 dx = __fadd2_rn(bx, make_float2(A.x, A.y)), dy = __fadd2_rn(by, make_float2(A.z, A.w)),
                     dz = __fadd2_rn(bz, make_float2(B.x, B.y));
        const float2 den = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __ffma2_rn(dz, dz, eps2)));
        float r0 = recip_f32(den.x), r1 = recip_f32(den.y);
        if (GUARD) {
          r0 = den.x > 0.0f ? r0 : 0.0f;
          r1 = den.y > 0.0f ? r1 : 0.0f;
        }
        const float2* w0 = reinterpret_cast<const float2*>(wt + (2 * k2) * MB);
        const float2* w1 = reinterpret_cast<const float2*>(wt + (2 * k2 + 1) * MB);
#pragma unroll
        for (int p = 0; p < MB / 2; p++) {
          const float2 g0 = __fmul2_rn(w0[p], make_float2(r0, r0)), g1 = __fmul2_rn(w1[p], make_float2(r1, r1));
          fx[p] = __ffma2_rn(g0, make_float2(dx.x, dx.x), fx[p]);
          fy[p] = __ffma2_rn(g0, make_float2(dy.x, dy.x), fy[p]);
          fz[p] = __ffma2_rn(g0, make_float2(dz.x, dz.x), fz[p]);
          fx[p] = __ffma2_rn(g1, make_float2(dx.y, dx.y), fx[p]);
          fy[p] = __ffma2_rn(g1, make_float2(dy.y, dy.y), fy[p]);
          fz[p] = __ffma2_rn(g1, make_float2(dz.y, dz.y), fz[p]);
        }
      }
#pragma unroll
      for (int p = 0; p < MB / 2; p++) {
        ax[2 * p] += (double)fx[p].x;
        ay[2 * p] += (double)fy[p].x;
        az[2 * p] += (double)fz[p].x;
        ax[2 * p + 1] += (double)fx[p].y;
        ay[2 * p + 1] += (double)fy[p].y;
        az[2 * p + 1] += (double)fz[p].y;
      }
    }
  }
  if (!tgt) return;
  const double tx = x[ti], ty = y[ti], tz = z[ti];
#pragma unroll
  for (int j = 0; j < MB; j++) {
    if (mid[j] < 0) continue;
    double* v = out + (long)mid[j] * nsplit * 3 * N + (long)split * 3 * N;
    v[ti] = kBiotSavartPacked * (ty * az[j] - tz * ay[j]);
    v[N + ti] = kBiotSavartPacked * (tz * ax[j] - tx * az[j]);
    v[2 * N + ti] = kBiotSavartPacked * (tx * ay[j] - ty * ax[j]);
  }
}

// The first stage's near field with each leaf pair evaluated once for both
// directions.  At stage 0 the sources sit on the grid (psrcf holds the
// particles themselves, packed relative to their leaf's centre), so for
// particle i of leaf T and j of leaf S the differences are opposite, d_ji =
// -d_ij, and the distance and reciprocal are shared: one evaluation gives
// w_j r d to i and -w_i r d to j -- 7 paired float32 operations per pair
// instead of 10, and one reciprocal instead of two.  One CTA of 256 threads
// per unit (T, S, eT, eS) of 256-particle leaves: warp w takes S's particles
// 32w..32w+31 (shared memory), lane l T's particles 8l..8l+7 (registers, in
// pairs for FFMA2).  In step r lane l meets source 32w + (l + r) mod 32, so
// the 32 lanes of a warp update 32 different source accumulators (shared
// memory) and each source sees the lanes in a fixed order; after 32 steps the
// warps' target partials are added in warp order.  The float32 sums of the
// unit go to slot eT (what T's particles receive from S, [3][256]) and, for
// eS >= 0, slot eS (what S's receive from T); units with eS < 0 -- the
// diagonal pairs (T, T) and pairs whose mirror is not in the list -- evaluate
// T's side only.  k_near_slot_sum adds a leaf's slots in list order.
template <bool GUARD>
__global__ void __launch_bounds__(256, 2)
    k_bltc_near32_mutual(StepGeom fg, const int4* __restrict__ units, const float4* __restrict__ psrcf, float eps,
                         float* __restrict__ slot) {
  constexpr int L = kMutualLeaf;
  __shared__ float4 src[L];        // S's particles: packed position, strength
  __shared__ float4 sacc[L];       // what S's particles receive from T
  __shared__ float red[8][3][L];   // the warps' target partials
  const int4 u = units[blockIdx.x];
  const int T = u.x, S = u.y, eT = u.z, eS = u.w;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const bool both = eS >= 0;
  src[tid] = psrcf[(long)S * L + tid];
  sacc[tid] = make_float4(0.f, 0.f, 0.f, 0.f);
  const double* ct = fg.pd_centre + 4 * (long)(fg.offset + T);
  const double* cs = fg.pd_centre + 4 * (long)(fg.offset + S);
  const float bx0 = (float)((cs[0] - ct[0]) * kPackScale), by0 = (float)((cs[1] - ct[1]) * kPackScale),
              bz0 = (float)((cs[2] - ct[2]) * kPackScale);
  float2 bx[4], by[4], bz[4], wt[4], ax[4], ay[4], az[4];
#pragma unroll
  for (int p = 0; p < 4; p++) {
    const float4 t0 = psrcf[(long)T * L + 8 * lane + 2 * p], t1 = psrcf[(long)T * L + 8 * lane + 2 * p + 1];
    bx[p] = make_float2(bx0 - t0.x, bx0 - t1.x);
    by[p] = make_float2(by0 - t0.y, by0 - t1.y);
    bz[p] = make_float2(bz0 - t0.z, bz0 - t1.z);
    wt[p] = make_float2(t0.w, t1.w);
    ax[p] = ay[p] = az[p] = make_float2(0.f, 0.f);
  }
  const float2 eps2 = make_float2(eps, eps);
  __syncthreads();
#pragma unroll 2
  for (int r = 0; r < 32; r++) {
    const int j = 32 * warp + ((lane + r) & 31);
    const float4 sj = src[j];
    const float2 sx = make_float2(sj.x, sj.x), sy = make_float2(sj.y, sj.y), sz = make_float2(sj.z, sj.z),
                 sw = make_float2(sj.w, sj.w);
    float2 gx = make_float2(0.f, 0.f), gy = gx, gz = gx;
#pragma unroll
    for (int p = 0; p < 4; p++) {
      const float2 dx = __fadd2_rn(bx[p], sx), dy = __fadd2_rn(by[p], sy), dz = __fadd2_rn(bz[p], sz);
      const float2 den = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __ffma2_rn(dz, dz, eps2)));
      float r0 = recip_f32(den.x), r1 = recip_f32(den.y);
      if (GUARD) {
        r0 = den.x > 0.0f ? r0 : 0.0f;
        r1 = den.y > 0.0f ? r1 : 0.0f;
      }
      const float2 rr = make_float2(r0, r1);
      const float2 g = __fmul2_rn(sw, rr);
      ax[p] = __ffma2_rn(g, dx, ax[p]);
      ay[p] = __ffma2_rn(g, dy, ay[p]);
      az[p] = __ffma2_rn(g, dz, az[p]);
      if (both) {
        const float2 h = __fmul2_rn(wt[p], rr);
        gx = __ffma2_rn(h, dx, gx);
        gy = __ffma2_rn(h, dy, gy);
        gz = __ffma2_rn(h, dz, gz);
      }
    }
    if (both) {  // source j receives -(sum of h d): the difference points the other way
      float4 a = sacc[j];
      a.x -= gx.x + gx.y;
      a.y -= gy.x + gy.y;
      a.z -= gz.x + gz.y;
      sacc[j] = a;
    }
    __syncwarp();
  }
#pragma unroll
  for (int p = 0; p < 4; p++) {
    const int k = 8 * lane + 2 * p;
    red[warp][0][k] = ax[p].x;
    red[warp][0][k + 1] = ax[p].y;
    red[warp][1][k] = ay[p].x;
    red[warp][1][k + 1] = ay[p].y;
    red[warp][2][k] = az[p].x;
    red[warp][2][k + 1] = az[p].y;
  }
  __syncthreads();
  float* o = slot + (long)eT * 3 * L;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    float a = red[0][c][tid];
#pragma unroll
    for (int w = 1; w < 8; w++) a += red[w][c][tid];
    o[c * L + tid] = a;
  }
  if (both) {
    float* q = slot + (long)eS * 3 * L;
    const float4 a = sacc[tid];
    q[tid] = a.x;
    q[L + tid] = a.y;
    q[2 * L + tid] = a.z;
  }
}

// Near-field sums of every particle from the unit slots: leaf T's slots in
// its near-list order (float32 sums added in float64), then u = cb t x a as
// the per-leaf-pair kernel's epilogue; written as split 0 of the near buffer.
__global__ void k_near_slot_sum(TreeGeom tg, const float* __restrict__ slot, const double* __restrict__ x,
                                const double* __restrict__ y, const double* __restrict__ z, double* __restrict__ near) {
  constexpr int L = kMutualLeaf;
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= tg.N) return;
  const int T = (int)(i / L), k = (int)(i - (long)T * L);
  double a0 = 0, a1 = 0, a2 = 0;
  for (int e = tg.near_start[T]; e < tg.near_start[T + 1]; e++) {
    const float* p = slot + (long)e * 3 * L;
    a0 += (double)p[k];
    a1 += (double)p[L + k];
    a2 += (double)p[2 * L + k];
  }
  const double tx = x[i], ty = y[i], tz = z[i];
  near[i] = kBiotSavartPacked * (ty * a2 - tz * a1);
  near[tg.N + i] = kBiotSavartPacked * (tz * a0 - tx * a2);
  near[2 * tg.N + i] = kBiotSavartPacked * (tx * a1 - ty * a0);
}

// Leaf proxy targets -> particles: v_i = (near-field splits summed in order)
// + sum_a lx[k][a] sum_b ly[k][b] T[a][b], with the leaf-box basis of
// particle k of the (uniform) leaf.
__device__ __forceinline__ void bltc_to_particles_body(const TreeGeom& tg, const StepGeom& fg, int f,
                                                       const double* __restrict__ tgt,
                                                       const double* __restrict__ near, int splits,
                                                       double* __restrict__ v) {
  extern __shared__ double tsh[];  // 3 x qx
  const int n1 = tg.n + 1, qx = n1 * n1, npl = tg.npl;
  const long pn = (long)fg.panels * qx;
  const long base = (long)(fg.offset + f) * qx;
  for (int m = threadIdx.x; m < qx; m += blockDim.x) {
    tsh[m] = tgt[base + m];
    tsh[qx + m] = tgt[pn + base + m];
    tsh[2 * qx + m] = tgt[2 * pn + base + m];
  }
  __syncthreads();
  for (int k = threadIdx.x; k < npl; k += blockDim.x) {
    const double* lxk = tg.lx + k * n1;
    const double* lyk = tg.ly + k * n1;
    // the particle's eta basis in registers (n1 <= kMaxDegree + 1), read once
    double lb[kMaxDegree + 1];
#pragma unroll
    for (int b = 0; b <= kMaxDegree; b++) lb[b] = b < n1 ? __ldg(lyk + b) : 0.0;
    double u0 = 0, u1 = 0, u2 = 0;
    for (int a = 0; a < n1; a++) {
      double s0 = 0, s1 = 0, s2 = 0;
#pragma unroll
      for (int b = 0; b <= kMaxDegree; b++) {
        if (b < n1) {
          s0 = fma(lb[b], tsh[a * n1 + b], s0);
          s1 = fma(lb[b], tsh[qx + a * n1 + b], s1);
          s2 = fma(lb[b], tsh[2 * qx + a * n1 + b], s2);
        }
      }
      double la = __ldg(lxk + a);
      u0 = fma(la, s0, u0);
      u1 = fma(la, s1, u1);
      u2 = fma(la, s2, u2);
    }
    const long i = (long)f * npl + k;
    double n0 = 0, n1s = 0, n2 = 0;
    for (int y = 0; y < splits; y++) {
      const double* p = near + (long)y * 3 * tg.N;
      n0 += p[i];
      n1s += p[tg.N + i];
      n2 += p[2 * tg.N + i];
    }
    v[i] = n0 + u0;
    v[tg.N + i] = n1s + u1;
    v[2 * tg.N + i] = n2 + u2;
  }
}

__global__ void __launch_bounds__(kThreads)
    k_bltc_to_particles(TreeGeom tg, StepGeom fg, const double* __restrict__ tgt, const double* __restrict__ near,
                        int splits, double* __restrict__ v) {
  bltc_to_particles_body(tg, fg, tg.leaf0 + blockIdx.x, tgt, near, splits, v);
}

__global__ void __launch_bounds__(kThreads)
    k_bltc_to_particles_batch(const BatchMember* __restrict__ mem, const double* __restrict__ near, int splits,
                              double* __restrict__ v) {
  const BatchMember& m = mem[blockIdx.y];
  const TreeGeom tg = m.tg;
  const StepGeom fg = m.fg;
  const long mo = blockIdx.y;
  bltc_to_particles_body(tg, fg, blockIdx.x, m.ftgt, near + mo * splits * 3 * tg.N, splits, v + mo * 3 * tg.N);
}

}  // namespace

using dev::blocks_for;

void launch_bltc_sources(const TreeGeom& tg, const StepGeom& fg, const BliTable& tab, int stage, double dt_s,
                         const double* vprev, const double* x, const double* y, const double* z, const double* vors,
                         const double* area, double4* psrc, float4* psrcf, double4* proxy, bool mixed,
                         cudaStream_t st) {
  size_t smem = sizeof(double) * ((size_t)tg.npl * (tg.n + 1) * 2 + tg.npl + kThreads);
  static std::atomic<unsigned long long> attr{0};
  raise_smem_once(attr, 200 * 1024, k_bltc_sources);
  SB_LAUNCH(k_bltc_sources, (unsigned)fg.leaves, kThreads, smem, st, tg, fg, tab, stage, dt_s, vprev, x, y, z, vors,
            area, psrc, psrcf, proxy, mixed ? 1 : 0);
}

void launch_bltc_sources_batch(const BatchMember* mem, int members, int leaves, int npl, int nmax, int stage,
                               double dt_s, const double* vprev, const double* x, const double* y, const double* z,
                               const double* vors, const double* area, double4* psrc, float4* psrcf, bool mixed,
                               cudaStream_t st) {
  size_t smem = sizeof(double) * ((size_t)npl * (nmax + 1) * 2 + npl + kThreads);
  static std::atomic<unsigned long long> attr{0};
  raise_smem_once(attr, 200 * 1024, k_bltc_sources_batch);
  SB_LAUNCH(k_bltc_sources_batch, dim3((unsigned)leaves, (unsigned)members), kThreads, smem, st, mem, stage, dt_s,
            vprev, x, y, z, vors, area, psrc, mixed ? psrcf : nullptr, mixed ? 1 : 0);
}

void launch_bltc_near_batch(const BatchMember* mem, int members, int leaves, int npl, double eps, int precision,
                            const double* x, const double* y, const double* z, const double4* psrc,
                            const float4* psrcf, double* near, int splits, int nt, int tpt, bool expanded,
                            cudaStream_t st) {
  const bool guard = !(eps > 0);
  const dim3 grid((unsigned)leaves, (unsigned)splits, (unsigned)members);
#define SB_NEARB(NT, TPT)                                                                                         \
  do {                                                                                                            \
    if (precision == SBSLPM_MIXED) {                                                                              \
      const size_t sm32 = sizeof(float4) * (expanded && !guard ? 4 : 2) * ((npl + 1) / 2);                       \
      if (guard)                                                                                                  \
        SB_LAUNCH((k_bltc_near32_batch<NT, TPT, true, false>), grid, NT, sm32, st, mem, x, y, z, psrcf, near);    \
      else if (expanded)                                                                                          \
        SB_LAUNCH((k_bltc_near32_batch<NT, TPT, false, true>), grid, NT, sm32, st, mem, x, y, z, psrcf, near);    \
      else                                                                                                        \
        SB_LAUNCH((k_bltc_near32_batch<NT, TPT, false, false>), grid, NT, sm32, st, mem, x, y, z, psrcf, near);   \
    } else {                                                                                                      \
      const size_t sm64 = sizeof(double4) * npl;                                                                 \
      if (guard) SB_LAUNCH((k_bltc_near64_batch<NT, TPT, true>), grid, NT, sm64, st, mem, x, y, z, psrc, near);   \
      else SB_LAUNCH((k_bltc_near64_batch<NT, TPT, false>), grid, NT, sm64, st, mem, x, y, z, psrc, near);        \
    }                                                                                                             \
  } while (0)
  // tile shapes the autotuner chooses from (NT threads x TPT targets per thread >= npl)
  if (nt == 64 && tpt == 4) SB_NEARB(64, 4);
  else if (nt == 128 && tpt == 2) SB_NEARB(128, 2);
  else if (nt == 256 && tpt == 1) SB_NEARB(256, 1);
  else if (nt == 64 && tpt == 2) SB_NEARB(64, 2);
  else if (nt == 64 && tpt == 1) SB_NEARB(64, 1);
  else if (nt == 256 && tpt == 2) SB_NEARB(256, 2);
  else if (nt == 128 && tpt == 1) SB_NEARB(128, 1);
#undef SB_NEARB
}

void launch_bltc_near_multi(const BatchMember* mem, const int* perm, int members, int groups, int leaves, int npl,
                            double eps, const int* ustart, const int* uent, const double* x, const double* y,
                            const double* z, const float4* psrcf, double* near, int splits, cudaStream_t st) {
  constexpr int MB = kNearGroup;
  const bool guard = !(eps > 0);
  const dim3 grid((unsigned)leaves, (unsigned)splits, (unsigned)groups);
  const size_t smem = sizeof(float4) * 2 * ((npl + 1) / 2) + sizeof(float) * MB * 2 * ((npl + 1) / 2);
  if (npl <= 64) {
    if (guard) SB_LAUNCH((k_bltc_near32_multi<64, MB, true>), grid, 64, smem, st, mem, perm, members, ustart, uent, x, y, z, psrcf, near);
    else SB_LAUNCH((k_bltc_near32_multi<64, MB, false>), grid, 64, smem, st, mem, perm, members, ustart, uent, x, y, z, psrcf, near);
  } else {
    if (guard) SB_LAUNCH((k_bltc_near32_multi<256, MB, true>), grid, 256, smem, st, mem, perm, members, ustart, uent, x, y, z, psrcf, near);
    else SB_LAUNCH((k_bltc_near32_multi<256, MB, false>), grid, 256, smem, st, mem, perm, members, ustart, uent, x, y, z, psrcf, near);
  }
}

void launch_bltc_near_mutual(const TreeGeom& tg, const StepGeom& fg, const int4* units, int nunits,
                             const float4* psrcf, float* slot, const double* x, const double* y, const double* z,
                             double* near, cudaStream_t st) {
  if (nunits > 0) {
    if (!(tg.eps > 0)) SB_LAUNCH(k_bltc_near32_mutual<true>, (unsigned)nunits, 256, 0, st, fg, units, psrcf,
                                 (float)tg.eps, slot);
    else SB_LAUNCH(k_bltc_near32_mutual<false>, (unsigned)nunits, 256, 0, st, fg, units, psrcf, (float)tg.eps, slot);
  }
  SB_LAUNCH(k_near_slot_sum, blocks_for(tg.N, 256), 256, 0, st, tg, slot, x, y, z, near);
}

void launch_bltc_to_particles_batch(const BatchMember* mem, int members, int leaves, int nmax, const double* near,
                                    int splits, double* v, cudaStream_t st) {
  const int qx = (nmax + 1) * (nmax + 1);
  SB_LAUNCH(k_bltc_to_particles_batch, dim3((unsigned)leaves, (unsigned)members), kThreads,
            sizeof(double) * 3 * qx, st, mem, near, splits, v);
}

void launch_bltc_to_particles(const TreeGeom& tg, const StepGeom& fg, const double* tgt, const double* near,
                              int splits, double* v, cudaStream_t st) {
  int qx = (tg.n + 1) * (tg.n + 1);
  SB_LAUNCH(k_bltc_to_particles, (unsigned)(tg.owned > 0 ? tg.owned : fg.leaves), kThreads, sizeof(double) * 3 * qx,
            st, tg, fg, tgt, near, splits, v);
}

}  // namespace sbslpm
