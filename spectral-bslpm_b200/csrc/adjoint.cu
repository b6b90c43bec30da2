// Hand-written adjoint (vector-Jacobian products) of the BVE step, sm_100a:
// the Biot-Savart sum with respect to source positions and strengths, the
// source displacement and planetary-vorticity terms, the backward RK4
// departure search and the BLI remap (bve_back_rk4_step,
// src/bve_time_step.cpp:311-419, differentiated in reverse order).
//
// Forward pieces and their adjoints (K = -1/(4 pi), d = y - x, D = |d|^2/2 + eps):
//   u_i = K x_i x sum_j q_j d_ij / D_ij
//     qbar_j  = K sum_i g c_i.d            (c_i = ubar_i x x_i, g = 1/D)
//     ybar_j  = K q_j sum_i [g c_i - g^2 (c_i.d) d]
//   y = proj(p) = p/|p|:   pbar = (ybar - yhat (yhat.ybar)) / |p|
//   BLI f(P) = sum_m f_m Lx_a(xi(P)) Ly_b(eta(P)):
//     fbar_m += abar Lx_a Ly_b (scattered with atomics),
//     Pbar = abar [ (sum f_m Lx_a' Ly_b) grad xi + (sum f_m Lx_a Ly_b') grad eta ]
// with the barycentric derivative L_a' = L_a (T/S - 1/(t - t_a)) off the nodes
// (r_k = w_k/(t - t_k), S = sum r_k, T = sum r_k/(t - t_k)) and the
// differentiation-matrix entries at a node.
#include <cuda_runtime.h>

#include "../../include/sbslpm.h"
#include "adjoint.cuh"
#include "adjoint_pair32.cuh"
#include "device_common.cuh"

namespace sbslpm {
namespace {

using namespace dev;

constexpr int kAdjThreads = 128;

// ---------------------------------------------------------------------------
// Biot-Savart sum: vector-Jacobian product with respect to the sources.
// One thread per source; target tiles (x_i, c_i = ubar_i x x_i) staged in
// shared memory; gridDim.y groups of targets write partials [group][4][ns]
// (qbar, ybar x, y, z) that k_sum_groups adds in group order.
template <bool GUARD>
__global__ void __launch_bounds__(kAdjThreads)
    k_bs_vjp64(long nt, const double* __restrict__ tx, const double* __restrict__ ty, const double* __restrict__ tz,
               const double* __restrict__ ux, const double* __restrict__ uy, const double* __restrict__ uz, long ns,
               const double4* __restrict__ src, double eps, double* __restrict__ partial) {
  __shared__ double sx[kAdjThreads], sy[kAdjThreads], sz[kAdjThreads], scx[kAdjThreads], scy[kAdjThreads],
      scz[kAdjThreads];
  const long j = blockIdx.x * (long)kAdjThreads + threadIdx.x;
  const long per = (nt + gridDim.y - 1) / gridDim.y;
  const long t0 = blockIdx.y * per, t1 = min(nt, t0 + per);
  double4 s = j < ns ? src[j] : make_double4(0, 0, 0, 0);
  double qb = 0, bx = 0, by = 0, bz = 0;
  for (long base = t0; base < t1; base += kAdjThreads) {
    const long i = base + threadIdx.x;
    __syncthreads();
    if (i < t1) {
      const double x = tx[i], y = ty[i], z = tz[i], a = ux[i], b = uy[i], c = uz[i];
      sx[threadIdx.x] = x;
      sy[threadIdx.x] = y;
      sz[threadIdx.x] = z;
      scx[threadIdx.x] = b * z - c * y;  // ubar x x
      scy[threadIdx.x] = c * x - a * z;
      scz[threadIdx.x] = a * y - b * x;
    }
    __syncthreads();
    const int cnt = (int)min((long)kAdjThreads, t1 - base);
    for (int k = 0; k < cnt; k++) {
      const double dx = s.x - sx[k], dy = s.y - sy[k], dz = s.z - sz[k];
      const double r2 = fma(dx, dx, fma(dy, dy, dz * dz));
      double g = recip_nr(fma(0.5, r2, eps));
      if (GUARD) g = r2 > 0.0 ? g : 0.0;
      const double cx = scx[k], cy = scy[k], cz = scz[k];
      const double sd = fma(cx, dx, fma(cy, dy, cz * dz));
      qb = fma(g, sd, qb);
      const double t = g * g * sd;
      bx = fma(g, cx, fma(-t, dx, bx));
      by = fma(g, cy, fma(-t, dy, by));
      bz = fma(g, cz, fma(-t, dz, bz));
    }
  }
  if (j < ns) {
    double* p = partial + (long)blockIdx.y * 4 * ns;
    p[j] = kBiotSavart * qb;
    p[ns + j] = kBiotSavart * s.w * bx;
    p[2 * ns + j] = kBiotSavart * s.w * by;
    p[3 * ns + j] = kBiotSavart * s.w * bz;
  }
}

// The same VJP in mixed precision for the step's own particles (targets and
// sources both [leaf][q]; leaf centres g.pd_centre): one thread per source,
// packed relative to its leaf's centre; target tiles of whole leaves staged
// as pairs (adj_stage), the offset between the two leaves' centres rounded
// to float32 once per (source, target leaf), the float32 sums of a target
// leaf added into float64 -- the arithmetic of the forward's mixed leaf-pair
// kernels.  gridDim.y groups of target leaves write partials [group][4][ns].
template <bool GUARD>
__global__ void __launch_bounds__(kAdjThreads)
    k_bs_vjp32_leaves(StepGeom g, const double* __restrict__ tx, const double* __restrict__ ty,
                      const double* __restrict__ tz, const double* __restrict__ ux, const double* __restrict__ uy,
                      const double* __restrict__ uz, const double4* __restrict__ src, double* __restrict__ partial) {
  __shared__ float4 tile[3 * (kAdjThreads / 2)];  // TL leaves x qh target pairs x 3
  const int q = g.q, qh = (q + 1) >> 1, TL = max(1, kAdjThreads / (2 * qh));
  const long ns = (long)g.leaves * q;
  const long j = blockIdx.x * (long)kAdjThreads + threadIdx.x;
  const int per = (g.leaves + gridDim.y - 1) / gridDim.y;
  const int l0 = blockIdx.y * per, l1 = min(g.leaves, l0 + per);
  const double4 s = src[j < ns ? j : 0];
  const double* cs = g.pd_centre + 4 * (long)(g.offset + (j < ns ? j / q : 0));
  const float sx = (float)((s.x - cs[0]) * kPackScale), sy = (float)((s.y - cs[1]) * kPackScale),
              sz = (float)((s.z - cs[2]) * kPackScale);
  const float feps = (float)g.eps;
  const float2 eps2 = make_float2(feps, feps);
  double qb = 0, bx = 0, by = 0, bz = 0;
  for (int L = l0; L < l1; L += TL) {
    const int nl = min(TL, l1 - L);
    __syncthreads();
    for (int k = threadIdx.x; k < nl * 2 * qh; k += blockDim.x) {
      const int ll = k / (2 * qh), idx = k - ll * 2 * qh;
      float4* lt = tile + 3 * qh * ll;
      if (idx < q) {
        const long i = (long)(L + ll) * q + idx;
        adj_stage(lt, idx, tx[i], ty[i], tz[i], ux[i], uy[i], uz[i], g.pd_centre + 4 * (long)(g.offset + L + ll));
      } else {
        adj_stage_zero(lt, idx);
      }
    }
    __syncthreads();
    for (int ll = 0; ll < nl; ll++) {
      const double* ct = g.pd_centre + 4 * (long)(g.offset + L + ll);
      const float a0 = sx + (float)((cs[0] - ct[0]) * kPackScale), a1 = sy + (float)((cs[1] - ct[1]) * kPackScale),
                  a2 = sz + (float)((cs[2] - ct[2]) * kPackScale);
      const float2 ax = make_float2(a0, a0), ay = make_float2(a1, a1), az = make_float2(a2, a2);
      float2 qq = make_float2(0.f, 0.f), cx = qq, cy = qq, cz = qq, dx = qq, dy = qq, dz = qq;
      const float4* lt = tile + 3 * qh * ll;
      for (int k2 = 0; k2 < qh; k2++)
        adj_pair32x2<GUARD>(ax, ay, az, lt[3 * k2], lt[3 * k2 + 1], lt[3 * k2 + 2], eps2, qq, cx, cy, cz, dx, dy, dz);
      qb += (double)qq.x + (double)qq.y;
      bx += ((double)cx.x + (double)cx.y) - 2.0 * ((double)dx.x + (double)dx.y);
      by += ((double)cy.x + (double)cy.y) - 2.0 * ((double)dy.x + (double)dy.y);
      bz += ((double)cz.x + (double)cz.y) - 2.0 * ((double)dz.x + (double)dz.y);
    }
  }
  if (j < ns) {
    double* p = partial + (long)blockIdx.y * 4 * ns;
    p[j] = kBiotSavart / kPackScale * qb;
    p[ns + j] = kBiotSavart * s.w * bx;
    p[2 * ns + j] = kBiotSavart * s.w * by;
    p[3 * ns + j] = kBiotSavart * s.w * bz;
  }
}

__global__ void k_sum_groups(const double* __restrict__ partial, int groups, long n, long gstride,
                             double* __restrict__ out) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double a = 0;
  for (int k = 0; k < groups; k++) a += partial[(long)k * gstride + i];
  out[i] = a;
}

__global__ void k_pack_sources(long n, const double* __restrict__ x, const double* __restrict__ y,
                               const double* __restrict__ z, const double* __restrict__ q, double4* __restrict__ s) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  s[i] = make_double4(x[i], y[i], z[i], q[i]);
}

// ---------------------------------------------------------------------------
// Sources of a stage (k_leaf_sources): adjoint.  q_j = a_j (w_j + 2 Omega z_j
// - 2 Omega y_z), y_j = proj(x_j + h v_prev,j).  Adds a_j qbar_j to wbar and
// h J(p)^T ybar' to vbar_prev, ybar' = ybar - 2 Omega a_j qbar_j e_z.
__global__ void k_src_adjoint(long n, int stage, double h, double omega, const double* __restrict__ vprev,
                              const double* __restrict__ x, const double* __restrict__ y, const double* __restrict__ z,
                              const double* __restrict__ area, const double* __restrict__ qbar,
                              const double* __restrict__ ybar, double* __restrict__ wbar,
                              double* __restrict__ vbar_prev) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double aq = area[i] * qbar[i];
  wbar[i] += aq;
  if (stage == 0) return;
  const double px = x[i] + h * vprev[i], py = y[i] + h * vprev[n + i], pz = z[i] + h * vprev[2 * n + i];
  const double r = sqrt(px * px + py * py + pz * pz), ir = 1.0 / r;
  const double hx = px * ir, hy = py * ir, hz = pz * ir;
  const double gx = ybar[i], gy = ybar[n + i], gz = ybar[2 * n + i] - 2.0 * omega * aq;
  const double dd = hx * gx + hy * gy + hz * gz;
  vbar_prev[i] += h * (gx - hx * dd) * ir;
  vbar_prev[n + i] += h * (gy - hy * dd) * ir;
  vbar_prev[2 * n + i] += h * (gz - hz * dd) * ir;
}

// ---------------------------------------------------------------------------
// Departure search + remap: adjoint.

// 1-D barycentric basis and its derivative in t (the BLI of
// interp_vals_bli, src/interp_funcs_impl.hpp:11-42, on Chebyshev extrema).
template <int D>
__device__ __forceinline__ void bli_1d_deriv(double t, double lo, double hi, const BliTable& tab, double* f,
                                             double* df, unsigned& err) {
  const double range = 0.5 * (hi - lo), offset = 0.5 * (hi + lo);
  if (t < lo - 1e-15 || t > hi + 1e-15) err |= kErrOutOfPanel;
  double node[D + 1];
  int hit = -1;
#pragma unroll
  for (int i = 0; i <= D; i++) {
    node[i] = tab.cosv[i] * range + offset;
    if (hit < 0 && fabs(t - node[i]) < 1e-15) hit = i;
  }
  if (hit >= 0) {
    double sum = 0;
#pragma unroll
    for (int a = 0; a <= D; a++) {
      f[a] = a == hit ? 1.0 : 0.0;
      df[a] = a == hit ? 0.0 : (tab.w[a] / tab.w[hit]) / (node[hit] - node[a]);
      sum += df[a];
    }
    df[hit] = -sum;
    return;
  }
  double S = 0, T = 0;
#pragma unroll
  for (int k = 0; k <= D; k++) {
    const double r = tab.w[k] / (t - node[k]);
    f[k] = r;
    S += r;
    T += r / (t - node[k]);
  }
  const double iS = 1.0 / S, TS = T * iS;
#pragma unroll
  for (int a = 0; a <= D; a++) {
    f[a] *= iS;
    df[a] = f[a] * (TS - 1.0 / (t - node[a]));
  }
}

template <int D>
struct BasisD {
  double fx[D + 1], fe[D + 1], dfx[D + 1], dfe[D + 1];
  double gxi[3], geta[3];  // gradients of xi and eta with respect to the point
  long row;
};

// xi = atan(u/w) on the located face: grad xi = (w grad u - u grad w)/(u^2 + w^2)
// with u, w signed coordinates (xieta_from_xyz, src/cubed_sphere_transforms_impl.hpp:68-98).
__device__ __forceinline__ void atan_grad(double u, int iu, double su, double w, int iw, double sw, double* gr) {
  const double den = 1.0 / (u * u + w * w);
  gr[0] = gr[1] = gr[2] = 0;
  gr[iu] += w * su * den;
  gr[iw] -= u * sw * den;
}

template <int D>
__device__ __forceinline__ void locate_basis_d(const StepGeom& g, const BliTable& tab, double x, double y, double z,
                                               BasisD<D>& b, unsigned& err) {
  double xi, eta;
  Bounds bd;
  const int leaf = locate_leaf(x, y, z, g.levels, xi, eta, bd, err);
  bli_1d_deriv<D>(xi, kPi / 4.0 * bd.min_xi, kPi / 4.0 * bd.max_xi, tab, b.fx, b.dfx, err);
  bli_1d_deriv<D>(eta, kPi / 4.0 * bd.min_eta, kPi / 4.0 * bd.max_eta, tab, b.fe, b.dfe, err);
  b.row = (long)(leaf - g.offset) * g.q;
  switch (face_from_xyz(x, y, z)) {  // (u, w) of xi and eta per face, with signs
    case 0: atan_grad(y, 1, 1, x, 0, 1, b.gxi); atan_grad(z, 2, 1, x, 0, 1, b.geta); break;
    case 1: atan_grad(-x, 0, -1, y, 1, 1, b.gxi); atan_grad(z, 2, 1, y, 1, 1, b.geta); break;
    case 2: atan_grad(y, 1, 1, x, 0, 1, b.gxi); atan_grad(-z, 2, -1, x, 0, 1, b.geta); break;
    case 3: atan_grad(-x, 0, -1, y, 1, 1, b.gxi); atan_grad(-z, 2, -1, y, 1, 1, b.geta); break;
    case 4: atan_grad(y, 1, 1, z, 2, 1, b.gxi); atan_grad(-x, 0, -1, z, 2, 1, b.geta); break;
    default: atan_grad(-y, 1, -1, z, 2, 1, b.gxi); atan_grad(-x, 0, -1, z, 2, 1, b.geta); break;
  }
}

// a (3 components at stride n) interpolated at the located point, into k.
template <int D>
__device__ __forceinline__ void interp3(const BasisD<D>& b, const double* __restrict__ v, long n, double* k) {
  k[0] = k[1] = k[2] = 0;
  int m = 0;
#pragma unroll
  for (int i = 0; i <= D; i++)
#pragma unroll
    for (int j = 0; j <= D; j++, m++) {
      const double bm = b.fx[i] * b.fe[j];
      k[0] += v[b.row + m] * bm;
      k[1] += v[n + b.row + m] * bm;
      k[2] += v[2 * n + b.row + m] * bm;
    }
}

// Adjoint of k = interp3(v)(P): vbar += kbar b_m (atomics), returns Pbar.
template <int D>
__device__ __forceinline__ void interp3_adjoint(const BasisD<D>& b, const double* __restrict__ v, long n,
                                                const double* kbar, double* __restrict__ vbar, double* Pbar) {
  double dxi = 0, deta = 0;
  int m = 0;
#pragma unroll
  for (int i = 0; i <= D; i++)
#pragma unroll
    for (int j = 0; j <= D; j++, m++) {
      const double bm = b.fx[i] * b.fe[j];
      const long o = b.row + m;
      const double s = kbar[0] * v[o] + kbar[1] * v[n + o] + kbar[2] * v[2 * n + o];
      dxi += s * (b.dfx[i] * b.fe[j]);
      deta += s * (b.fx[i] * b.dfe[j]);
      atomicAdd(vbar + o, kbar[0] * bm);
      atomicAdd(vbar + n + o, kbar[1] * bm);
      atomicAdd(vbar + 2 * n + o, kbar[2] * bm);
    }
  for (int c = 0; c < 3; c++) Pbar[c] = dxi * b.gxi[c] + deta * b.geta[c];
}

__device__ __forceinline__ void proj_t(const double* p, const double* a, double* out) {
  const double r = sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]), ir = 1.0 / r;
  const double h0 = p[0] * ir, h1 = p[1] * ir, h2 = p[2] * ir;
  const double dd = h0 * a[0] + h1 * a[1] + h2 * a[2];
  out[0] = (a[0] - h0 * dd) * ir;
  out[1] = (a[1] - h1 * dd) * ir;
  out[2] = (a[2] - h2 * dd) * ir;
}

__device__ __forceinline__ void proj3(const double* p, double* y) {
  double a = p[0], b = p[1], c = p[2];
  project_to_sphere(a, b, c);
  y[0] = a;
  y[1] = b;
  y[2] = c;
}

// One particle: recompute the departure chain of bve_find_departure_points
// (src/bve_time_step.cpp:172-309) and the remap of bve_departure_to_target
// (:15-67), then run them backwards from wbar_new.
template <int D>
__global__ void k_depart_remap_adjoint(StepGeom g, BliTable tab, const double* __restrict__ x,
                                       const double* __restrict__ y, const double* __restrict__ z,
                                       const double* __restrict__ v0, const double* __restrict__ v1,
                                       const double* __restrict__ v2, const double* __restrict__ v3, double dt,
                                       const double* __restrict__ w, const double* __restrict__ wbar_new,
                                       double* __restrict__ wbar, double* __restrict__ vb0, double* __restrict__ vb1,
                                       double* __restrict__ vb2, double* __restrict__ vb3) {
  const long n = (long)g.leaves * g.q;
  const long o = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (o >= n) return;
  unsigned err = 0;
  const double x0[3] = {x[o], y[o], z[o]};
  const double k1[3] = {v3[o], v3[n + o], v3[2 * n + o]};
  double q2[3], P2[3], k2[3], q3[3], P3[3], k3[3], q4[3], P4[3], k4[3];
  BasisD<D> B2, B3, B4, Bd;
  for (int c = 0; c < 3; c++) q2[c] = x0[c] - 0.5 * dt * k1[c];
  proj3(q2, P2);
  locate_basis_d<D>(g, tab, P2[0], P2[1], P2[2], B2, err);
  interp3<D>(B2, v2, n, k2);
  for (int c = 0; c < 3; c++) q3[c] = x0[c] - 0.5 * dt * k2[c];
  proj3(q3, P3);
  locate_basis_d<D>(g, tab, P3[0], P3[1], P3[2], B3, err);
  interp3<D>(B3, v1, n, k3);
  for (int c = 0; c < 3; c++) q4[c] = x0[c] - dt * k3[c];
  proj3(q4, P4);
  locate_basis_d<D>(g, tab, P4[0], P4[1], P4[2], B4, err);
  interp3<D>(B4, v0, n, k4);
  double p1[3], D1[3], p2[3], D2[3], p3[3], D3[3], p4[3], dep[3];
  for (int c = 0; c < 3; c++) p1[c] = x0[c] - 1.0 / 6.0 * dt * k1[c];
  proj3(p1, D1);
  for (int c = 0; c < 3; c++) p2[c] = D1[c] + 1.0 / 3.0 * dt * k2[c];
  proj3(p2, D2);
  for (int c = 0; c < 3; c++) p3[c] = D2[c] + 1.0 / 3.0 * dt * k3[c];
  proj3(p3, D3);
  for (int c = 0; c < 3; c++) p4[c] = D3[c] + 1.0 / 6.0 * dt * k4[c];
  proj3(p4, dep);
  locate_basis_d<D>(g, tab, dep[0], dep[1], dep[2], Bd, err);

  // remap: w_new = BLI(w)(dep) + 2 Omega dep_z - 2 Omega z
  const double a = wbar_new[o];
  double dxi = 0, deta = 0;
  {
    int m = 0;
#pragma unroll
    for (int i = 0; i <= D; i++)
#pragma unroll
      for (int j = 0; j <= D; j++, m++) {
        const long r = Bd.row + m;
        dxi += w[r] * (Bd.dfx[i] * Bd.fe[j]);
        deta += w[r] * (Bd.fx[i] * Bd.dfe[j]);
        atomicAdd(wbar + r, a * (Bd.fx[i] * Bd.fe[j]));
      }
  }
  double dbar[3];
  for (int c = 0; c < 3; c++) dbar[c] = a * (dxi * Bd.gxi[c] + deta * Bd.geta[c]);
  dbar[2] += a * 2.0 * g.omega;

  // combination, backwards
  double t4[3], t3[3], t2[3], t1[3], kb1[3], kb2[3], kb3[3], kb4[3];
  proj_t(p4, dbar, t4);
  for (int c = 0; c < 3; c++) kb4[c] = 1.0 / 6.0 * dt * t4[c];
  proj_t(p3, t4, t3);
  for (int c = 0; c < 3; c++) kb3[c] = 1.0 / 3.0 * dt * t3[c];
  proj_t(p2, t3, t2);
  for (int c = 0; c < 3; c++) kb2[c] = 1.0 / 3.0 * dt * t2[c];
  proj_t(p1, t2, t1);
  for (int c = 0; c < 3; c++) kb1[c] = -1.0 / 6.0 * dt * t1[c];
  // k4 = v0 at P4 = proj(x - dt k3)
  double Pb[3], qb[3];
  interp3_adjoint<D>(B4, v0, n, kb4, vb0, Pb);
  proj_t(q4, Pb, qb);
  for (int c = 0; c < 3; c++) kb3[c] += -dt * qb[c];
  // k3 = v1 at P3 = proj(x - dt/2 k2)
  interp3_adjoint<D>(B3, v1, n, kb3, vb1, Pb);
  proj_t(q3, Pb, qb);
  for (int c = 0; c < 3; c++) kb2[c] += -0.5 * dt * qb[c];
  // k2 = v2 at P2 = proj(x - dt/2 k1)
  interp3_adjoint<D>(B2, v2, n, kb2, vb2, Pb);
  proj_t(q2, Pb, qb);
  for (int c = 0; c < 3; c++) kb1[c] += -0.5 * dt * qb[c];
  // k1 = v3 at the particle
  vb3[o] = kb1[0];
  vb3[n + o] = kb1[1];
  vb3[2 * n + o] = kb1[2];
  flag(g.err, err);
}

int vjp_groups(long nt, long ns) {
  const long sblocks = (ns + kAdjThreads - 1) / kAdjThreads;
  long want = (4L * 148 * 8 + sblocks - 1) / sblocks;
  const long maxg = (nt + 1023) / 1024;
  long gsel = want < maxg ? want : maxg;
  return (int)(gsel < 1 ? 1 : (gsel > 64 ? 64 : gsel));
}

}  // namespace

int adjoint_groups(long nt, long ns) { return vjp_groups(nt, ns); }

void launch_bs_vjp(long nt, const double* tx, const double* ty, const double* tz, const double* ux,
                   const double* uy, const double* uz, long ns, const double4* src, double eps, double* partial,
                   int groups, double* qbar, double* ybar, cudaStream_t st) {
  const dim3 grid(blocks_for(ns, kAdjThreads), (unsigned)groups);
  if (eps > 0)
    SB_LAUNCH(k_bs_vjp64<false>, grid, kAdjThreads, 0, st, nt, tx, ty, tz, ux, uy, uz, ns, src, eps, partial);
  else
    SB_LAUNCH(k_bs_vjp64<true>, grid, kAdjThreads, 0, st, nt, tx, ty, tz, ux, uy, uz, ns, src, eps, partial);
  // partial: [group][4][ns] -> qbar [ns], ybar [3][ns]
  SB_LAUNCH(k_sum_groups, blocks_for(ns, 256), 256, 0, st, partial, groups, ns, 4 * ns, qbar);
  for (int c = 0; c < 3; c++)
    SB_LAUNCH(k_sum_groups, blocks_for(ns, 256), 256, 0, st, partial + (long)(c + 1) * ns, groups, ns, 4 * ns,
              ybar + (long)c * ns);
}

void launch_bs_vjp_leaves32(const StepGeom& g, const double* tx, const double* ty, const double* tz,
                            const double* ux, const double* uy, const double* uz, const double4* src, double* partial,
                            int groups, double* qbar, double* ybar, cudaStream_t st) {
  const long ns = (long)g.leaves * g.q;
  const int gl = groups < g.leaves ? groups : g.leaves;
  const dim3 grid(blocks_for(ns, kAdjThreads), (unsigned)gl);
  if (g.eps > 0)
    SB_LAUNCH(k_bs_vjp32_leaves<false>, grid, kAdjThreads, 0, st, g, tx, ty, tz, ux, uy, uz, src, partial);
  else
    SB_LAUNCH(k_bs_vjp32_leaves<true>, grid, kAdjThreads, 0, st, g, tx, ty, tz, ux, uy, uz, src, partial);
  SB_LAUNCH(k_sum_groups, blocks_for(ns, 256), 256, 0, st, partial, gl, ns, 4 * ns, qbar);
  for (int c = 0; c < 3; c++)
    SB_LAUNCH(k_sum_groups, blocks_for(ns, 256), 256, 0, st, partial + (long)(c + 1) * ns, gl, ns, 4 * ns,
              ybar + (long)c * ns);
}

void launch_pack_sources(long n, const double* x, const double* y, const double* z, const double* q, double4* s,
                         cudaStream_t st) {
  SB_LAUNCH(k_pack_sources, blocks_for(n, 256), 256, 0, st, n, x, y, z, q, s);
}

void launch_src_adjoint(long n, int stage, double h, double omega, const double* vprev, const double* x,
                        const double* y, const double* z, const double* area, const double* qbar, const double* ybar,
                        double* wbar, double* vbar_prev, cudaStream_t st) {
  SB_LAUNCH(k_src_adjoint, blocks_for(n, 256), 256, 0, st, n, stage, h, omega, vprev, x, y, z, area, qbar, ybar,
            wbar, vbar_prev);
}

void launch_depart_remap_adjoint(const StepGeom& g, const BliTable& tab, const double* x, const double* y,
                                 const double* z, const double* v0, const double* v1, const double* v2,
                                 const double* v3, double dt, const double* w, const double* wbar_new, double* wbar,
                                 double* vb0, double* vb1, double* vb2, double* vb3, cudaStream_t st) {
  const long n = (long)g.leaves * g.q;
#define SB_DRA(D)                                                                                                 \
  case D:                                                                                                         \
    SB_LAUNCH(k_depart_remap_adjoint<D>, blocks_for(n, 128), 128, 0, st, g, tab, x, y, z, v0, v1, v2, v3, dt, w,  \
              wbar_new, wbar, vb0, vb1, vb2, vb3);                                                                \
    break;
  switch (g.degree) {
    SB_DRA(1) SB_DRA(2) SB_DRA(3) SB_DRA(4) SB_DRA(5) SB_DRA(6) SB_DRA(7) SB_DRA(8) SB_DRA(9) SB_DRA(10)
  }
#undef SB_DRA
}

}  // namespace sbslpm
