// Device helpers shared by the kernel files: the reciprocal used by every
// pair kernel, the Biot-Savart pair in float64 / float32 / paired float32,
// the device error word, and the launch macro that counts launches.
#pragma once

#include <cuda_runtime.h>

#include <atomic>

#include "bve_kernels.cuh"

namespace sbslpm {
namespace dev {

__device__ __forceinline__ void flag(unsigned* err, unsigned bits) {
  if (bits) atomicOr(err, bits);
}

// 1/d from the hardware approximation refined by two Newton-Raphson steps
// r <- r + r (1 - d r); each step squares the relative error.  d > 0.
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

// One Biot-Savart pair in float64.  With d = y - x and |x| = |y| = 1,
// 1 - x.y = |d|^2 / 2, and x cross y = x cross d, so the accumulated
// a = sum g d gives u = -1/(4 pi) x cross a.  Coincident points add nothing:
// with eps > 0 because d = 0; with eps = 0 (GUARD) because g is zeroed.
template <bool GUARD>
__device__ __forceinline__ void pair64(double tx, double ty, double tz, const double4 s, double eps, double& ax,
                                       double& ay, double& az) {
  double dx = s.x - tx, dy = s.y - ty, dz = s.z - tz;
  double r2 = fma(dx, dx, fma(dy, dy, dz * dz));
  double g = s.w * recip_nr(fma(0.5, r2, eps));
  if (GUARD) g = r2 > 0.0 ? g : 0.0;
  ax = fma(g, dx, ax);
  ay = fma(g, dy, ay);
  az = fma(g, dz, az);
}

// The same pair in float32 on panel-relative coordinates scaled by 1/sqrt(2)
// (kPackScale): d' = base + s.xyz with base = (c_S - c_T)/sqrt(2) - delta_t,
// and |d'|^2 + eps = |d|^2/2 + eps in one FMA chain.
template <bool GUARD>
__device__ __forceinline__ void pair32(float bx, float by, float bz, const float4 s, float eps, float& ax, float& ay,
                                       float& az) {
  float dx = bx + s.x, dy = by + s.y, dz = bz + s.z;
  float den = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, eps)));
  float g = s.w * recip_f32(den);
  if (GUARD) g = den > 0.0f ? g : 0.0f;
  ax = fmaf(g, dx, ax);
  ay = fmaf(g, dy, ay);
  az = fmaf(g, dz, az);
}

// Two pairs at once with the paired FP32 instructions of sm_100 (FADD2 /
// FFMA2 / FMUL2): one target (b broadcast in both halves) against two
// sources given as register pairs (x0,x1), (y0,y1), (z0,z1), (w0,w1).
template <bool GUARD>
__device__ __forceinline__ void pair32x2(const float2 bx, const float2 by, const float2 bz, const float2 sx,
                                         const float2 sy, const float2 sz, const float2 sw, const float2 eps2,
                                         float2& ax, float2& ay, float2& az) {
  const float2 dx = __fadd2_rn(bx, sx), dy = __fadd2_rn(by, sy), dz = __fadd2_rn(bz, sz);
  const float2 den = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __ffma2_rn(dz, dz, eps2)));
  float2 g = __fmul2_rn(sw, make_float2(recip_f32(den.x), recip_f32(den.y)));
  if (GUARD) {
    g.x = den.x > 0.0f ? g.x : 0.0f;
    g.y = den.y > 0.0f ? g.y : 0.0f;
  }
  ax = __ffma2_rn(g, dx, ax);
  ay = __ffma2_rn(g, dy, ay);
  az = __ffma2_rn(g, dz, az);
}

// Two pairs in the expanded form: with b = base (target side, as above) and
// s the source's packed offset, |b + s|^2 + eps = (|s|^2 + eps) + |b|^2 +
// 2 b.s, and sum g (b + s) = sum r (w s) + b sum r w with r = 1/den.  The
// source side is staged as (x0,x1,y0,y1) (z0,z1,q0,q1) (w0x0,w1x1,w0y0,w1y1)
// (w0z0,w1z1,w0,w1) with q = |s|^2 + eps, the target side as m = 2b and
// bb = |b|^2: 4 paired operations for the denominator and 4 for the sums, 8
// per two pairs against 10 in pair32x2.  The expansion rounds the
// denominator to u (|b| + |s|)^2 instead of u |b + s| (|b| + |s|), so it is
// used only where eps dominates that (a coincident pair still adds nothing:
// its s = -b cancels in the final b sum r w + sum r w s up to rounding of
// w s / eps).  fx, fy, fz accumulate sum r w s; fw accumulates sum r w.
__device__ __forceinline__ void pair32x2_expanded(const float2 mx, const float2 my, const float2 mz, const float2 bb,
                                                  const float4 A, const float4 B, const float4 C, const float4 D,
                                                  float2& fx, float2& fy, float2& fz, float2& fw) {
  float2 den = __fadd2_rn(make_float2(B.z, B.w), bb);
  den = __ffma2_rn(mz, make_float2(B.x, B.y), den);
  den = __ffma2_rn(my, make_float2(A.z, A.w), den);
  den = __ffma2_rn(mx, make_float2(A.x, A.y), den);
  const float2 r = make_float2(recip_f32(den.x), recip_f32(den.y));
  fx = __ffma2_rn(r, make_float2(C.x, C.y), fx);
  fy = __ffma2_rn(r, make_float2(C.z, C.w), fy);
  fz = __ffma2_rn(r, make_float2(D.x, D.y), fz);
  fw = __ffma2_rn(r, make_float2(D.z, D.w), fw);
}

// Stages the sources 2k, 2k+1 of a packed float4 array (x, y, z, w) in the
// expanded form's four float4 (a missing partner past n has zero strength).
__device__ __forceinline__ void stage_expanded(const float4* __restrict__ src, int k2, int n, float eps,
                                               float4* __restrict__ out) {
  const float4 s0 = src[2 * k2];
  const float4 s1 = (2 * k2 + 1 < n) ? src[2 * k2 + 1] : make_float4(0.f, 0.f, 0.f, 0.f);
  const float q0 = fmaf(s0.x, s0.x, fmaf(s0.y, s0.y, fmaf(s0.z, s0.z, eps)));
  const float q1 = fmaf(s1.x, s1.x, fmaf(s1.y, s1.y, fmaf(s1.z, s1.z, eps)));
  out[0] = make_float4(s0.x, s1.x, s0.y, s1.y);
  out[1] = make_float4(s0.z, s1.z, q0, q1);
  out[2] = make_float4(s0.w * s0.x, s1.w * s1.x, s0.w * s0.y, s1.w * s1.y);
  out[3] = make_float4(s0.w * s0.z, s1.w * s1.z, s0.w, s1.w);
}

// First panel id of the k-th level below the subtree root (level, root_rel).
__device__ __forceinline__ int subtree_first(int level, int root_rel, int k) {
  return level_start(level + k) + (root_rel << (2 * k));
}

__device__ __forceinline__ void nonleaf_position(const StepGeom& g, long i, int stage, double dt_s,
                                                 const double* __restrict__ vprev, double& px, double& py,
                                                 double& pz) {
  const long pn = (long)g.panels * g.q, ln = (long)g.leaves * g.q;
  px = g.px[i];
  py = g.px[pn + i];
  pz = g.px[2 * pn + i];
  if (stage > 0) {
    const long np = (long)g.offset * g.q;
    const long row = (long)g.il_row[i] * g.q;
    double ax = 0, ay = 0, az = 0;
    for (int m = 0; m < g.q; m++) {
      double bm = g.il_basis[m * np + i];
      ax += (dt_s * vprev[row + m]) * bm;
      ay += (dt_s * vprev[ln + row + m]) * bm;
      az += (dt_s * vprev[2 * ln + row + m]) * bm;
    }
    px += ax;
    py += ay;
    pz += az;
  }
  project_to_sphere(px, py, pz);
}


// Point location + tensor-product BLI basis at a point (point_locate_panel
// and interp_vals_bli, src/interp_funcs_impl.hpp:11-142), and gathers of a
// [leaf][q] field with it.
template <int D>
struct Basis {
  double fx[D + 1], fe[D + 1];
  long row;  // (leaf - offset) * q
};

template <int D>
__device__ __forceinline__ void locate_basis(const StepGeom& g, const BliTable& tab, double x, double y, double z,
                                             Basis<D>& b, unsigned& err) {
  double xi, eta;
  Bounds bd;
  int leaf = locate_leaf(x, y, z, g.levels, xi, eta, bd, err);
  bli_1d(xi, kPi / 4.0 * bd.min_xi, kPi / 4.0 * bd.max_xi, D, tab.cosv, tab.w, b.fx, err);
  bli_1d(eta, kPi / 4.0 * bd.min_eta, kPi / 4.0 * bd.max_eta, D, tab.cosv, tab.w, b.fe, err);
  b.row = (long)(leaf - g.offset) * g.q;
}

// The same basis with fewer float64 divisions, for the departure / remap
// kernel (one thread per particle, four locations each): the projection and
// the face coordinates multiply by one reciprocal, and the barycentric basis
// uses the common-denominator form f_i = w_i P_i / sum_k w_k P_k with
// P_i = prod_{j != i} (t - c_j) -- the second barycentric form multiplied
// through by prod_j (t - c_j): one division per direction instead of 2(D+1).
// Nodes within 1e-15 are hit exactly as in bli_1d; results differ from
// locate_basis by rounding only.
template <int D>
__device__ __forceinline__ void bli_1d_common(double t, double lo, double hi, const BliTable& tab, double* f,
                                              unsigned& err) {
  const double range = 0.5 * (hi - lo), offset = 0.5 * (hi + lo);
  if (t < lo - 1e-15 || t > hi + 1e-15) err |= kErrOutOfPanel;
  if (D == 0) {
    f[0] = 1;
    return;
  }
  double dl[D + 1];
  int hit = -1;
#pragma unroll
  for (int i = 0; i <= D; i++) {
    dl[i] = t - (tab.cosv[i] * range + offset);
    if (hit < 0 && fabs(dl[i]) < 1e-15) hit = i;
  }
  if (hit >= 0) {
#pragma unroll
    for (int i = 0; i <= D; i++) f[i] = (i == hit) ? 1.0 : 0.0;
    return;
  }
  double pre[D + 1], suf = 1.0, den = 0.0;
  pre[0] = 1.0;
#pragma unroll
  for (int i = 1; i <= D; i++) pre[i] = pre[i - 1] * dl[i - 1];
#pragma unroll
  for (int i = D; i >= 0; i--) {
    f[i] = tab.w[i] * (pre[i] * suf);
    den += f[i];
    suf *= dl[i];
  }
  const double inv = 1.0 / den;
#pragma unroll
  for (int i = 0; i <= D; i++) f[i] *= inv;
}

__device__ __forceinline__ void project_to_sphere_rcp(double& x, double& y, double& z) {
  const double inv = 1.0 / sqrt(x * x + y * y + z * z);
  x *= inv;
  y *= inv;
  z *= inv;
}

template <int D>
__device__ __forceinline__ void locate_basis_rcp(const StepGeom& g, const BliTable& tab, double x, double y, double z,
                                                 Basis<D>& b, unsigned& err) {
  const int face = face_from_xyz(x, y, z);
  double xi, eta;
  switch (face) {  // xieta_from_xyz_face with one reciprocal of the face's axis coordinate
    case 0: { const double r = 1.0 / x; xi = atan(y * r); eta = atan(z * r); break; }
    case 1: { const double r = 1.0 / y; xi = atan(-x * r); eta = atan(z * r); break; }
    case 2: { const double r = 1.0 / x; xi = atan(y * r); eta = atan(-z * r); break; }
    case 3: { const double r = 1.0 / y; xi = atan(-x * r); eta = atan(-z * r); break; }
    case 4: { const double r = 1.0 / z; xi = atan(y * r); eta = atan(-x * r); break; }
    default: { const double r = 1.0 / z; xi = atan(-y * r); eta = atan(-x * r); break; }
  }
  // tree descent of locate_leaf from the face's coordinates
  Bounds bd{-1, 1, -1, 1};
  int id = face;
  for (int lev = 0; lev < g.levels - 1; lev++) {
    const double mid_xi = 0.5 * kPi / 4.0 * (bd.max_xi + bd.min_xi);
    const double mid_eta = 0.5 * kPi / 4.0 * (bd.max_eta + bd.min_eta);
    const double ux = 0.5 * (bd.max_xi + bd.min_xi), ue = 0.5 * (bd.max_eta + bd.min_eta);
    int c;
    if ((xi >= mid_xi) && (eta >= mid_eta)) {
      c = 0;
      bd.min_xi = ux;
      bd.min_eta = ue;
    } else if ((xi <= mid_xi) && (eta >= mid_eta)) {
      c = 1;
      bd.max_xi = ux;
      bd.min_eta = ue;
    } else if ((xi <= mid_xi) && (eta <= mid_eta)) {
      c = 2;
      bd.max_xi = ux;
      bd.max_eta = ue;
    } else if ((xi >= mid_xi) && (eta <= mid_eta)) {
      c = 3;
      bd.min_xi = ux;
      bd.max_eta = ue;
    } else {
      err |= kErrNonFinite;  // NaN coordinates
      c = 0;
      bd.min_xi = ux;
      bd.min_eta = ue;
    }
    id = level_start(lev + 1) + 4 * (id - level_start(lev)) + c;
  }
  bli_1d_common<D>(xi, kPi / 4.0 * bd.min_xi, kPi / 4.0 * bd.max_xi, tab, b.fx, err);
  bli_1d_common<D>(eta, kPi / 4.0 * bd.min_eta, kPi / 4.0 * bd.max_eta, tab, b.fe, err);
  b.row = (long)(id - g.offset) * g.q;
}

// sum_m field[row + m] * fx[i] fe[j] with m = i (D+1) + j, in m order.
template <int D>
__device__ __forceinline__ double gather(const Basis<D>& b, const double* __restrict__ f, long stride = 1,
                                         long base = 0) {
  double acc = 0;
  int m = 0;
#pragma unroll
  for (int i = 0; i <= D; i++)
#pragma unroll
    for (int j = 0; j <= D; j++, m++) acc += f[(b.row + m) * stride + base] * (b.fx[i] * b.fe[j]);
  return acc;
}

template <int D>
__device__ __forceinline__ void gather3(const Basis<D>& b, const double* __restrict__ v, long n, double& a,
                                        double& c, double& e) {
  a = 0;
  c = 0;
  e = 0;
  int m = 0;
#pragma unroll
  for (int i = 0; i <= D; i++)
#pragma unroll
    for (int j = 0; j <= D; j++, m++) {
      double bm = b.fx[i] * b.fe[j];
      a += v[b.row + m] * bm;
      c += v[n + b.row + m] * bm;
      e += v[2 * n + b.row + m] * bm;
    }
}

inline unsigned blocks_for(long n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace dev

// Kernel launches made by the library (a process-wide diagnostic count).
std::atomic<long>& launch_counter();

// Raises kernels' dynamic shared-memory limit on the current device, once per
// device (the attribute is per device: a process that drives several GPUs
// must set it on each).  done: the caller's static record of the devices set
// (device ordinals >= 64 are set on every call).
template <typename... K>
inline void raise_smem_once(std::atomic<unsigned long long>& done, int bytes, K... kernels) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return;
  const unsigned long long bit = dev < 64 ? 1ull << dev : 0ull;
  if (bit && (done.load(std::memory_order_acquire) & bit)) return;
  (cudaFuncSetAttribute(kernels, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes), ...);
  if (bit) done.fetch_or(bit, std::memory_order_acq_rel);
}

}  // namespace sbslpm

#define SB_LAUNCH(kernel, grid, block, shmem, st, ...)      \
  do {                                                     \
    kernel<<<grid, block, shmem, st>>>(__VA_ARGS__);       \
    ::sbslpm::launch_counter()++;                          \
  } while (0)
