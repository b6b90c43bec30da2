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
// absolute positions.  Mixed: pair32 with the sources packed relative to
// their own grid leaf (gq particles) and, per source grid leaf, the target's
// offset from that leaf's centre formed in float64 and rounded once, so that
// d' = (c_sub - t) kPackScale + (s - c_sub) kPackScale carries the rounding
// of grid-leaf-sized terms rather than tree-leaf-sized ones (the divergence
// tendency differentiates the velocity twice and amplifies that rounding);
// float32 sums per source grid leaf added into float64.
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
  double tx[TPT], ty[TPT], tz[TPT], ax[TPT], ay[TPT], az[TPT], bx[TPT], by[TPT], bz[TPT];
#pragma unroll
  for (int r = 0; r < TPT; r++) {
    const int k = threadIdx.x + r * NT;
    const long i = (long)f * npl + (k < npl ? k : 0);
    tx[r] = x[i];
    ty[r] = y[i];
    tz[r] = z[i];
    ax[r] = ay[r] = az[r] = bx[r] = by[r] = bz[r] = 0;
  }
  const float feps = (float)tg.eps;
  for (int e = tg.near_start[f] + split; e < tg.near_start[f + 1]; e += nsplit) {
    const int sl = tg.near_src[e];
    const long sb = (long)sl * npl;
    __syncthreads();
    for (int k = threadIdx.x; k < npl; k += NT) {
      if constexpr (MIXED) {
        t1[k] = psrcf[sb + k];
        t2[k] = psrcf2[sb + k];
      } else {
        t1[k] = psrc[sb + k];
        t2[k] = psrc2[sb + k];
      }
    }
    __syncthreads();
    if constexpr (MIXED) {
      for (int k0 = 0; k0 < npl; k0 += gq) {
        const double* cs = gcentre + 4 * ((sb + k0) / gq);
        float b0[TPT], b1[TPT], b2[TPT], fa[TPT][3], fb[TPT][3];
#pragma unroll
        for (int r = 0; r < TPT; r++) {
          b0[r] = (float)((cs[0] - tx[r]) * kPackScale);
          b1[r] = (float)((cs[1] - ty[r]) * kPackScale);
          b2[r] = (float)((cs[2] - tz[r]) * kPackScale);
          fa[r][0] = fa[r][1] = fa[r][2] = fb[r][0] = fb[r][1] = fb[r][2] = 0.f;
        }
#pragma unroll 4
        for (int k = k0; k < k0 + gq; k++) {
          const float4 s1 = t1[k], s2 = t2[k];
#pragma unroll
          for (int r = 0; r < TPT; r++) {
            pair32<GUARD>(b0[r], b1[r], b2[r], s1, feps, fa[r][0], fa[r][1], fa[r][2]);
            pair32<GUARD>(b0[r], b1[r], b2[r], s2, feps, fb[r][0], fb[r][1], fb[r][2]);
          }
        }
#pragma unroll
        for (int r = 0; r < TPT; r++) {
          ax[r] += fa[r][0];
          ay[r] += fa[r][1];
          az[r] += fa[r][2];
          bx[r] += fb[r][0];
          by[r] += fb[r][1];
          bz[r] += fb[r][2];
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
    swe_tree_epilogue(K, tx[r], ty[r], tz[r], ax[r], ay[r], az[r], bx[r], by[r], bz[r], ux, uy, uz);
    v[i] = ux;
    v[tg.N + i] = uy;
    v[2 * tg.N + i] = uz;
  }
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
  const size_t smem = (mixed ? sizeof(float4) : sizeof(double4)) * 2 * (size_t)tg.npl;
#define SB_SN(TPT)                                                                                                \
  do {                                                                                                            \
    if (mixed) {                                                                                                  \
      if (guard) SB_LAUNCH((k_bltc_swe_near<NT, TPT, true, true>), grid, NT, smem, st, tg, fg, x, y, z, psrc,     \
                           psrc2, psrcf, psrcf2, near, gcentre, gq);                                                           \
      else SB_LAUNCH((k_bltc_swe_near<NT, TPT, false, true>), grid, NT, smem, st, tg, fg, x, y, z, psrc, psrc2,   \
                     psrcf, psrcf2, near, gcentre, gq);                                                                        \
    } else {                                                                                                      \
      if (guard) SB_LAUNCH((k_bltc_swe_near<NT, TPT, true, false>), grid, NT, smem, st, tg, fg, x, y, z, psrc,    \
                           psrc2, psrcf, psrcf2, near, gcentre, gq);                                                           \
      else SB_LAUNCH((k_bltc_swe_near<NT, TPT, false, false>), grid, NT, smem, st, tg, fg, x, y, z, psrc, psrc2,  \
                     psrcf, psrcf2, near, gcentre, gq);                                                                        \
    }                                                                                                             \
  } while (0)
  if (tpt <= 1) SB_SN(1);
  else if (tpt == 2) SB_SN(2);
  else if (tpt <= 4) SB_SN(4);
  else SB_SN(8);
#undef SB_SN
}

}  // namespace sbslpm
