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

namespace sbslpm {

long& launch_counter();

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ double recip_nr(double d) {
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(d));
  double e = fma(-d, r, 1.0);
  r = fma(r, e, r);
  e = fma(-d, r, 1.0);
  return fma(r, e, r);
}

__device__ __forceinline__ float recip_f32(float d) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(d));
  return r;
}

// Barycentric Lagrange basis of degree n on Chebyshev extrema of [lo, hi]
// without the reference's range check: displaced sources may sit slightly
// outside their leaf, where the interpolant extrapolates smoothly.
__device__ __forceinline__ void bli_1d_free(double t, double lo, double hi, int n, const double* cosv,
                                            const double* w, double* f) {
  if (n == 0) {
    f[0] = 1;
    return;
  }
  double range = 0.5 * (hi - lo), offset = 0.5 * (hi + lo);
  int hit = -1;
  for (int i = 0; i <= n; i++)
    if (hit < 0 && fabs(t - (cosv[i] * range + offset)) < 1e-15) hit = i;
  if (hit >= 0) {
    for (int i = 0; i <= n; i++) f[i] = (i == hit) ? 1.0 : 0.0;
    return;
  }
  double den = 0;
  for (int i = 0; i <= n; i++) {
    double v = w[i] / (t - (cosv[i] * range + offset));
    f[i] = v;
    den += v;
  }
  double inv = 1.0 / den;
  for (int i = 0; i <= n; i++) f[i] *= inv;
}

__global__ void __launch_bounds__(kThreads)
    k_bltc_sources(TreeGeom tg, StepGeom fg, BliTable tab, int stage, double dt_s, const double* __restrict__ vprev,
                   const double* __restrict__ x, const double* __restrict__ y, const double* __restrict__ z,
                   const double* __restrict__ vors, const double* __restrict__ area, double4* __restrict__ psrc,
                   float4* __restrict__ psrcf, double4* __restrict__ proxy, int mixed) {
  extern __shared__ double sh[];
  const int n1 = tg.n + 1, npl = tg.npl, f = blockIdx.x;
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
      w = area[i] * vors[i];
    } else {
      const double vx = vprev[i], vy = vprev[N + i], vz = vprev[2 * N + i];
      xx += vx * dt_s;
      yy += vy * dt_s;
      zz += vz * dt_s;
      project_to_sphere(xx, yy, zz);
      w = area[i] * (vors[i] + 2 * tg.omega * z[i] - 2 * tg.omega * zz);
    }
    if (stage == 0) project_to_sphere(xx, yy, zz);
    psrc[i] = make_double4(xx, yy, zz, w);
    if (mixed) psrcf[i] = make_float4((float)(xx - cc[0]), (float)(yy - cc[1]), (float)(zz - cc[2]), (float)w);
    double xi, eta;
    xieta_from_xyz_face(xx, yy, zz, face, xi, eta);
    bli_1d_free(xi, bd[0], bd[1], tg.n, tab.cosv, tab.w, lx + k * n1);
    bli_1d_free(eta, bd[2], bd[3], tg.n, tab.cosv, tab.w, ly + k * n1);
    sw[k] = w;
  }
  __syncthreads();
  const int qx = n1 * n1;
  for (int m = threadIdx.x; m < qx; m += blockDim.x) {
    const int a = m / n1, b = m % n1;
    double acc = 0;
    for (int k = 0; k < npl; k++) acc = fma(lx[k * n1 + a] * ly[k * n1 + b], sw[k], acc);
    proxy[(long)panel * qx + m].w = acc;
  }
}

// Near leaf pairs: one CTA per target leaf, TPT targets per thread, the
// source leaf's particles staged in shared memory.
template <int TPT, bool GUARD>
__global__ void __launch_bounds__(kThreads)
    k_bltc_near64(TreeGeom tg, const double* __restrict__ x, const double* __restrict__ y,
                  const double* __restrict__ z, const double4* __restrict__ psrc, double* __restrict__ v) {
  extern __shared__ double4 tile[];
  const int npl = tg.npl, f = blockIdx.x;
  double tx[TPT], ty[TPT], tz[TPT], ax[TPT], ay[TPT], az[TPT];
#pragma unroll
  for (int r = 0; r < TPT; r++) {
    int k = threadIdx.x + r * kThreads;
    long i = (long)f * npl + (k < npl ? k : 0);
    tx[r] = x[i];
    ty[r] = y[i];
    tz[r] = z[i];
    ax[r] = ay[r] = az[r] = 0;
  }
  const double eps = tg.eps;
  for (int e = tg.near_start[f]; e < tg.near_start[f + 1]; e++) {
    const long sb = (long)tg.near_src[e] * npl;
    __syncthreads();
    for (int k = threadIdx.x; k < npl; k += kThreads) tile[k] = psrc[sb + k];
    __syncthreads();
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
    int k = threadIdx.x + r * kThreads;
    if (k >= npl) continue;
    long i = (long)f * npl + k;
    v[i] = kBiotSavart * (ty[r] * az[r] - tz[r] * ay[r]);
    v[tg.N + i] = kBiotSavart * (tz[r] * ax[r] - tx[r] * az[r]);
    v[2 * tg.N + i] = kBiotSavart * (tx[r] * ay[r] - ty[r] * ax[r]);
  }
}

// Mixed precision: target and source particles relative to their leaves'
// centres, float32 pairs, per-source-leaf float32 sums added into float64.
template <int TPT, bool GUARD>
__global__ void __launch_bounds__(kThreads)
    k_bltc_near32(TreeGeom tg, StepGeom fg, const double* __restrict__ x, const double* __restrict__ y,
                  const double* __restrict__ z, const float4* __restrict__ psrcf, double* __restrict__ v) {
  extern __shared__ float4 tilef[];
  const int npl = tg.npl, f = blockIdx.x;
  const double* ct = fg.pd_centre + 4 * (long)(fg.offset + f);
  const double cx = ct[0], cy = ct[1], cz = ct[2];
  double tx[TPT], ty[TPT], tz[TPT], ax[TPT], ay[TPT], az[TPT];
  float dtx[TPT], dty[TPT], dtz[TPT];
#pragma unroll
  for (int r = 0; r < TPT; r++) {
    int k = threadIdx.x + r * kThreads;
    long i = (long)f * npl + (k < npl ? k : 0);
    tx[r] = x[i];
    ty[r] = y[i];
    tz[r] = z[i];
    dtx[r] = (float)(tx[r] - cx);
    dty[r] = (float)(ty[r] - cy);
    dtz[r] = (float)(tz[r] - cz);
    ax[r] = ay[r] = az[r] = 0;
  }
  const float eps = (float)tg.eps;
  for (int e = tg.near_start[f]; e < tg.near_start[f + 1]; e++) {
    const int sl = tg.near_src[e];
    const long sb = (long)sl * npl;
    const double* cs = fg.pd_centre + 4 * (long)(fg.offset + sl);
    const float bx0 = (float)(cs[0] - cx), by0 = (float)(cs[1] - cy), bz0 = (float)(cs[2] - cz);
    __syncthreads();
    for (int k = threadIdx.x; k < npl; k += kThreads) tilef[k] = psrcf[sb + k];
    __syncthreads();
    float fx[TPT], fy[TPT], fz[TPT], bx[TPT], by[TPT], bz[TPT];
#pragma unroll
    for (int r = 0; r < TPT; r++) {
      fx[r] = fy[r] = fz[r] = 0.f;
      bx[r] = bx0 - dtx[r];
      by[r] = by0 - dty[r];
      bz[r] = bz0 - dtz[r];
    }
    for (int k = 0; k < npl; k++) {
      const float4 s = tilef[k];
#pragma unroll
      for (int r = 0; r < TPT; r++) {
        float dx = bx[r] + s.x, dy = by[r] + s.y, dz = bz[r] + s.z;
        float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
        float g = s.w * recip_f32(fmaf(0.5f, r2, eps));
        if (GUARD) g = r2 > 0.0f ? g : 0.0f;
        fx[r] = fmaf(g, dx, fx[r]);
        fy[r] = fmaf(g, dy, fy[r]);
        fz[r] = fmaf(g, dz, fz[r]);
      }
    }
#pragma unroll
    for (int r = 0; r < TPT; r++) {
      ax[r] += fx[r];
      ay[r] += fy[r];
      az[r] += fz[r];
    }
  }
#pragma unroll
  for (int r = 0; r < TPT; r++) {
    int k = threadIdx.x + r * kThreads;
    if (k >= npl) continue;
    long i = (long)f * npl + k;
    v[i] = kBiotSavart * (ty[r] * az[r] - tz[r] * ay[r]);
    v[tg.N + i] = kBiotSavart * (tz[r] * ax[r] - tx[r] * az[r]);
    v[2 * tg.N + i] = kBiotSavart * (tx[r] * ay[r] - ty[r] * ax[r]);
  }
}

// Leaf proxy targets -> particles: v_i += sum_a lx[k][a] sum_b ly[k][b] T[a][b]
// with the leaf-box basis of particle k of the (uniform) leaf.
__global__ void __launch_bounds__(kThreads)
    k_bltc_to_particles(TreeGeom tg, StepGeom fg, const double* __restrict__ tgt, double* __restrict__ v) {
  extern __shared__ double tsh[];  // 3 x qx
  const int n1 = tg.n + 1, qx = n1 * n1, npl = tg.npl, f = blockIdx.x;
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
    double u0 = 0, u1 = 0, u2 = 0;
    for (int a = 0; a < n1; a++) {
      double s0 = 0, s1 = 0, s2 = 0;
      for (int b = 0; b < n1; b++) {
        double lb = __ldg(lyk + b);
        s0 = fma(lb, tsh[a * n1 + b], s0);
        s1 = fma(lb, tsh[qx + a * n1 + b], s1);
        s2 = fma(lb, tsh[2 * qx + a * n1 + b], s2);
      }
      double la = __ldg(lxk + a);
      u0 = fma(la, s0, u0);
      u1 = fma(la, s1, u1);
      u2 = fma(la, s2, u2);
    }
    const long i = (long)f * npl + k;
    v[i] += u0;
    v[tg.N + i] += u1;
    v[2 * tg.N + i] += u2;
  }
}

inline unsigned blocks_for(long n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

#define SB_LAUNCH(kernel, grid, block, shmem, st, ...)      \
  do {                                                     \
    kernel<<<grid, block, shmem, st>>>(__VA_ARGS__);       \
    launch_counter()++;                                    \
  } while (0)

void launch_bltc_sources(const TreeGeom& tg, const StepGeom& fg, const BliTable& tab, int stage, double dt_s,
                         const double* vprev, const double* x, const double* y, const double* z, const double* vors,
                         const double* area, double4* psrc, float4* psrcf, double4* proxy, bool mixed,
                         cudaStream_t st) {
  size_t smem = sizeof(double) * ((size_t)tg.npl * (tg.n + 1) * 2 + tg.npl);
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_bltc_sources, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    attr = true;
  }
  SB_LAUNCH(k_bltc_sources, (unsigned)fg.leaves, kThreads, smem, st, tg, fg, tab, stage, dt_s, vprev, x, y, z, vors,
            area, psrc, psrcf, proxy, mixed ? 1 : 0);
}

void launch_bltc_near(const TreeGeom& tg, const StepGeom& fg, int precision, const double* x, const double* y,
                      const double* z, const double4* psrc, const float4* psrcf, double* v, cudaStream_t st) {
  const bool guard = !(tg.eps > 0);
  const unsigned grid = (unsigned)fg.leaves;
  if (precision == SBSLPM_MIXED) {
    size_t smem = sizeof(float4) * tg.npl;
    if (tg.npl <= kThreads) {
      if (guard) SB_LAUNCH((k_bltc_near32<1, true>), grid, kThreads, smem, st, tg, fg, x, y, z, psrcf, v);
      else SB_LAUNCH((k_bltc_near32<1, false>), grid, kThreads, smem, st, tg, fg, x, y, z, psrcf, v);
    } else {
      if (guard) SB_LAUNCH((k_bltc_near32<2, true>), grid, kThreads, smem, st, tg, fg, x, y, z, psrcf, v);
      else SB_LAUNCH((k_bltc_near32<2, false>), grid, kThreads, smem, st, tg, fg, x, y, z, psrcf, v);
    }
  } else {
    size_t smem = sizeof(double4) * tg.npl;
    if (tg.npl <= kThreads) {
      if (guard) SB_LAUNCH((k_bltc_near64<1, true>), grid, kThreads, smem, st, tg, x, y, z, psrc, v);
      else SB_LAUNCH((k_bltc_near64<1, false>), grid, kThreads, smem, st, tg, x, y, z, psrc, v);
    } else {
      if (guard) SB_LAUNCH((k_bltc_near64<2, true>), grid, kThreads, smem, st, tg, x, y, z, psrc, v);
      else SB_LAUNCH((k_bltc_near64<2, false>), grid, kThreads, smem, st, tg, x, y, z, psrc, v);
    }
  }
}

void launch_bltc_to_particles(const TreeGeom& tg, const StepGeom& fg, const double* tgt, double* v,
                              cudaStream_t st) {
  int qx = (tg.n + 1) * (tg.n + 1);
  SB_LAUNCH(k_bltc_to_particles, (unsigned)fg.leaves, kThreads, sizeof(double) * 3 * qx, st, tg, fg, tgt, v);
}

}  // namespace sbslpm
