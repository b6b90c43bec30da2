// Adjoint of the decoupled-degree treecode velocity (float64): the reverse
// of k_bltc_sources -> upward pass -> well-separated proxy interactions ->
// downward pass -> leaf interpolation + near field.  Every forward piece is
// linear in the strengths; the source positions enter the near field and the
// anterpolation onto the leaf proxies (the proxies themselves are fixed):
//
//   v_i      = near_i + sum_k B_k(x_i) T_leaf(i),k          B: leaf-box BLI basis (fixed)
//   T        = D (cc(Q))                                    D: downward pass
//   cc(Q)_t  = K x_t x sum_s sum_k g (y_k - x_t) Q_s,k       fixed proxies x_t, y_k
//   Q        = U (A(y) q)                                   U: upward pass, A: anterpolation
//   near_i   = K x_i x sum_j g (y_j - x_i) q_j              near leaf pairs
//
// Reverse: Tbar_leaf = B^T vbar; Tbar = D^T Tbar (an upward accumulation of
// three fields); Qbar_s = cc^T(Tbar) (a source-owned sum over the transposed
// well-separated list); Qbar = U^T Qbar (a downward accumulation); then per
// particle qbar_j = [A^T Qbar]_j + near^T, ybar_j = q_j grad_y(A^T Qbar) +
// near^T, with near^T the source-owned sum over the transposed near list.
//
// The reference's own spectral FMM (proxies = the panels' interp_degree
// points, displaced and re-projected at every stage; bve_vel_impl.hpp:85-122,
// bve_time_step.cpp:69-170) reverses the same way on the panel quadtree, with
// two differences: the interactions' sources move, so their transpose also
// gives position adjoints, and a non-leaf proxy's displacement is the BLI
// interpolation of its containing leaf's (bve_disp_interp), whose transpose
// scatters back onto the leaf velocities.
#include <cuda_runtime.h>

#include "adjoint_pair32.cuh"
#include "adjoint_tree.cuh"
#include "device_common.cuh"

namespace sbslpm {
namespace {

using namespace dev;

constexpr int kT = 128;

// Tbar_leaf[c][k] = sum_i B_k(x_i) vbar_c,i over the leaf's particles.
__global__ void k_tree_to_particles_T(TreeGeom tg, StepGeom fg, const double* __restrict__ vbar,
                                      double* __restrict__ tbar) {
  extern __shared__ double sv[];  // 3 x npl
  const int f = blockIdx.x, npl = tg.npl, n1 = tg.n + 1, qx = n1 * n1;
  const long N = tg.N, pn = (long)fg.panels * qx;
  for (int i = threadIdx.x; i < npl; i += blockDim.x)
    for (int c = 0; c < 3; c++) sv[c * npl + i] = vbar[c * N + (long)f * npl + i];
  __syncthreads();
  const long base = (long)(fg.offset + f) * qx;
  for (int m = threadIdx.x; m < 3 * qx; m += blockDim.x) {
    const int c = m / qx, k = m % qx, a = k / n1, b = k % n1;
    double acc = 0;
    for (int i = 0; i < npl; i++) acc = fma(__ldg(tg.lx + i * n1 + a) * __ldg(tg.ly + i * n1 + b), sv[c * npl + i], acc);
    tbar[c * pn + base + k] = acc;
  }
}

// One level of the transpose of the downward pass: parents at `level` add
// the anterpolation of their children's three fields (child_to_parent form).
__global__ void k_tree_up3(StepGeom fg, int level, double* __restrict__ t) {
  const int n1 = fg.degree + 1, q = fg.q;
  const long pn = (long)fg.panels * q;
  const long np = 6L << (2 * level);
  const long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (idx >= np * q * 3) return;
  const int c3 = (int)(idx / (np * q));
  const long r = idx % (np * q);
  const long p = level_start(level) + r / q;
  const int k = (int)(r % q), a = k / n1, b = k % n1;
  double acc = 0;
  for (int c = 0; c < 4; c++) {
    const long ch = level_start(level + 1) + 4 * (p - level_start(level)) + c;
    const double* lx = fg.child_1d + ((c == 1 || c == 2) ? n1 * n1 : 0);
    const double* ly = fg.child_1d + (c >= 2 ? n1 * n1 : 0);
    const double* tc = t + c3 * pn + ch * q;
    for (int i = 0; i < n1; i++) {
      double s = 0;
      for (int j = 0; j < n1; j++) s = fma(__ldg(ly + j * n1 + b), tc[i * n1 + j], s);
      acc = fma(__ldg(lx + i * n1 + a), s, acc);
    }
  }
  t[c3 * pn + p * q + k] += acc;
}

// One level of the transpose of the upward pass: children of `level` add the
// interpolation of their parent's (final) adjoint strengths.
__global__ void k_tree_down1(StepGeom fg, int level, double* __restrict__ qb) {
  const int n1 = fg.degree + 1, q = fg.q;
  const long nc = 6L << (2 * (level + 1));
  const long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (idx >= nc * q) return;
  const long ch = level_start(level + 1) + idx / q;
  const int k = (int)(idx % q), i = k / n1, j = k % n1;
  const long rel = ch - level_start(level + 1);
  const long p = level_start(level) + rel / 4;
  const int c = (int)(rel % 4);
  const double* lx = fg.child_1d + ((c == 1 || c == 2) ? n1 * n1 : 0) + i * n1;
  const double* ly = fg.child_1d + (c >= 2 ? n1 * n1 : 0) + j * n1;
  double acc = 0;
  for (int a = 0; a < n1; a++) {
    double s = 0;
    for (int b = 0; b < n1; b++) s = fma(__ldg(ly + b), qb[p * q + a * n1 + b], s);
    acc = fma(__ldg(lx + a), s, acc);
  }
  qb[ch * q + k] += acc;
}

// Transposed well-separated interactions: source panel s (blockIdx.x) sums
// over the target panels t whose list holds s: Qbar_s,k = K sum_t sum_i g c.d,
// c = Tbar_t,i x x_i, d = y_k - x_i.
template <bool GUARD>
__global__ void __launch_bounds__(kT) k_tree_cc_T(StepGeom fg, const int* __restrict__ tstart,
                                                 const int* __restrict__ ttgt, const double* __restrict__ tbar,
                                                 double* __restrict__ qbar) {
  __shared__ double sx[kT], sy[kT], sz[kT], cx[kT], cy[kT], cz[kT];
  const int s = blockIdx.x, q = fg.q;
  const long pn = (long)fg.panels * q;
  const int k = threadIdx.x;
  double yx = 0, yy = 0, yz = 0;
  if (k < q) {
    yx = fg.px[(long)s * q + k];
    yy = fg.px[pn + (long)s * q + k];
    yz = fg.px[2 * pn + (long)s * q + k];
  }
  double acc = 0;
  for (int e = tstart[s]; e < tstart[s + 1]; e++) {
    const long tb = (long)ttgt[e] * q;
    __syncthreads();
    if (k < q) {
      const double x = fg.px[tb + k], y = fg.px[pn + tb + k], z = fg.px[2 * pn + tb + k];
      const double a = tbar[tb + k], b = tbar[pn + tb + k], c = tbar[2 * pn + tb + k];
      sx[k] = x;
      sy[k] = y;
      sz[k] = z;
      cx[k] = b * z - c * y;
      cy[k] = c * x - a * z;
      cz[k] = a * y - b * x;
    }
    __syncthreads();
    if (k < q)
      for (int i = 0; i < q; i++) {
        const double dx = yx - sx[i], dy = yy - sy[i], dz = yz - sz[i];
        const double r2 = fma(dx, dx, fma(dy, dy, dz * dz));
        double g = recip_nr(fma(0.5, r2, fg.eps));
        if (GUARD) g = r2 > 0.0 ? g : 0.0;
        acc = fma(g, fma(cx[i], dx, fma(cy[i], dy, cz[i] * dz)), acc);
      }
  }
  if (k < q) qbar[(long)s * q + k] = kBiotSavart * acc;
}

// Transposed near field: source leaf sl (blockIdx.x), one thread per source
// particle, over the target leaves whose near list holds sl.  Writes qbar_j
// and ybar_j (3 components) of the leaf's particles.
template <bool GUARD>
__global__ void __launch_bounds__(512) k_tree_near_T(TreeGeom tg, const int* __restrict__ tstart,
                                                   const int* __restrict__ ttgt, const double* __restrict__ x,
                                                   const double* __restrict__ y, const double* __restrict__ z,
                                                   const double* __restrict__ vbar, const double4* __restrict__ psrc,
                                                   double* __restrict__ qbar, double* __restrict__ ybar) {
  extern __shared__ double tile[];  // 6 x npl: target positions, c = vbar x x
  const int sl = blockIdx.x, npl = tg.npl;
  const long N = tg.N;
  double* tx = tile;
  double* ty = tx + npl;
  double* tz = ty + npl;
  double* cx = tz + npl;
  double* cy = cx + npl;
  double* cz = cy + npl;
  const int j = threadIdx.x;
  const long oj = (long)sl * npl + j;
  const double4 s = j < npl ? psrc[oj] : make_double4(0, 0, 0, 0);
  double qb = 0, bx = 0, by = 0, bz = 0;
  for (int e = tstart[sl]; e < tstart[sl + 1]; e++) {
    const long tb = (long)ttgt[e] * npl;
    __syncthreads();
    for (int i = threadIdx.x; i < npl; i += blockDim.x) {
      const double a = vbar[tb + i], b = vbar[N + tb + i], c = vbar[2 * N + tb + i];
      const double px = x[tb + i], py = y[tb + i], pz = z[tb + i];
      tx[i] = px;
      ty[i] = py;
      tz[i] = pz;
      cx[i] = b * pz - c * py;
      cy[i] = c * px - a * pz;
      cz[i] = a * py - b * px;
    }
    __syncthreads();
    if (j < npl)
      for (int i = 0; i < npl; i++) {
        const double dx = s.x - tx[i], dy = s.y - ty[i], dz = s.z - tz[i];
        const double r2 = fma(dx, dx, fma(dy, dy, dz * dz));
        double g = recip_nr(fma(0.5, r2, tg.eps));
        if (GUARD) g = r2 > 0.0 ? g : 0.0;
        const double sd = fma(cx[i], dx, fma(cy[i], dy, cz[i] * dz));
        qb = fma(g, sd, qb);
        const double t = g * g * sd;
        bx = fma(g, cx[i], fma(-t, dx, bx));
        by = fma(g, cy[i], fma(-t, dy, by));
        bz = fma(g, cz[i], fma(-t, dz, bz));
      }
  }
  if (j < npl) {
    qbar[oj] = kBiotSavart * qb;
    ybar[oj] = kBiotSavart * s.w * bx;
    ybar[N + oj] = kBiotSavart * s.w * by;
    ybar[2 * N + oj] = kBiotSavart * s.w * bz;
  }
}

// Mixed-precision transposed near field: source leaf sl (blockIdx.x), one
// thread per source particle; per target leaf of the transposed list the
// float32 sums are added into float64.
template <bool GUARD>
__global__ void __launch_bounds__(512) k_tree_near_T32(TreeGeom tg, StepGeom fg, const int* __restrict__ tstart,
                                                     const int* __restrict__ ttgt, const double* __restrict__ x,
                                                     const double* __restrict__ y, const double* __restrict__ z,
                                                     const double* __restrict__ vbar,
                                                     const double4* __restrict__ psrc, double* __restrict__ qbar,
                                                     double* __restrict__ ybar) {
  extern __shared__ float4 tile32[];  // [(npl+1)/2][3]
  const int sl = blockIdx.x, npl = tg.npl, np2 = (npl + 1) >> 1;
  const long N = tg.N;
  const int j = threadIdx.x;
  const long oj = (long)sl * npl + (j < npl ? j : 0);
  const double4 s = psrc[oj];
  const double* cs = fg.pd_centre + 4 * (long)(fg.offset + sl);
  const float sx = (float)((s.x - cs[0]) * kPackScale), sy = (float)((s.y - cs[1]) * kPackScale),
              sz = (float)((s.z - cs[2]) * kPackScale);
  const float feps = (float)tg.eps;
  const float2 eps2 = make_float2(feps, feps);
  double qb = 0, bx = 0, by = 0, bz = 0;
  for (int e = tstart[sl]; e < tstart[sl + 1]; e++) {
    const int tl = ttgt[e];
    const long tb = (long)tl * npl;
    const double* ct = fg.pd_centre + 4 * (long)(fg.offset + tl);
    __syncthreads();
    for (int i = threadIdx.x; i < 2 * np2; i += blockDim.x) {
      if (i < npl)
        adj_stage(tile32, i, x[tb + i], y[tb + i], z[tb + i], vbar[tb + i], vbar[N + tb + i], vbar[2 * N + tb + i],
                  ct);
      else
        adj_stage_zero(tile32, i);
    }
    __syncthreads();
    const float a0 = sx + (float)((cs[0] - ct[0]) * kPackScale), a1 = sy + (float)((cs[1] - ct[1]) * kPackScale),
                a2 = sz + (float)((cs[2] - ct[2]) * kPackScale);
    const float2 ax = make_float2(a0, a0), ay = make_float2(a1, a1), az = make_float2(a2, a2);
    float2 q = make_float2(0.f, 0.f), cx = q, cy = q, cz = q, dx = q, dy = q, dz = q;
#pragma unroll 4
    for (int k2 = 0; k2 < np2; k2++)
      adj_pair32x2<GUARD>(ax, ay, az, tile32[3 * k2], tile32[3 * k2 + 1], tile32[3 * k2 + 2], eps2, q, cx, cy, cz,
                          dx, dy, dz);
    qb += (double)q.x + (double)q.y;
    bx += ((double)cx.x + (double)cx.y) - 2.0 * ((double)dx.x + (double)dx.y);
    by += ((double)cy.x + (double)cy.y) - 2.0 * ((double)dy.x + (double)dy.y);
    bz += ((double)cz.x + (double)cz.y) - 2.0 * ((double)dz.x + (double)dz.y);
  }
  if (j < npl) {
    qbar[oj] = kBiotSavart / kPackScale * qb;
    ybar[oj] = kBiotSavart * s.w * bx;
    ybar[N + oj] = kBiotSavart * s.w * by;
    ybar[2 * N + oj] = kBiotSavart * s.w * bz;
  }
}

// Mixed-precision transposed well-separated interactions: source panel s
// (blockIdx.x), one thread per source proxy, target panels' proxies and
// c = Tbar x x staged as pairs.
template <bool GUARD>
__global__ void __launch_bounds__(kT) k_tree_cc_T32(StepGeom fg, const int* __restrict__ tstart,
                                                   const int* __restrict__ ttgt, const double* __restrict__ tbar,
                                                   double* __restrict__ qbar) {
  __shared__ float4 tile[3 * ((kT + 1) / 2)];
  const int s = blockIdx.x, q = fg.q, q2 = (q + 1) >> 1;
  const long pn = (long)fg.panels * q;
  const int k = threadIdx.x;
  const long ok = (long)s * q + (k < q ? k : 0);
  const double* cs = fg.pd_centre + 4 * (long)s;
  const float sx = (float)((fg.px[ok] - cs[0]) * kPackScale), sy = (float)((fg.px[pn + ok] - cs[1]) * kPackScale),
              sz = (float)((fg.px[2 * pn + ok] - cs[2]) * kPackScale);
  const float feps = (float)fg.eps;
  const float2 eps2 = make_float2(feps, feps);
  double acc = 0;
  for (int e = tstart[s]; e < tstart[s + 1]; e++) {
    const int t = ttgt[e];
    const long tb = (long)t * q;
    const double* ct = fg.pd_centre + 4 * (long)t;
    __syncthreads();
    for (int i = threadIdx.x; i < 2 * q2; i += blockDim.x) {
      if (i < q)
        adj_stage(tile, i, fg.px[tb + i], fg.px[pn + tb + i], fg.px[2 * pn + tb + i], tbar[tb + i], tbar[pn + tb + i],
                  tbar[2 * pn + tb + i], ct);
      else
        adj_stage_zero(tile, i);
    }
    __syncthreads();
    const float a0 = sx + (float)((cs[0] - ct[0]) * kPackScale), a1 = sy + (float)((cs[1] - ct[1]) * kPackScale),
                a2 = sz + (float)((cs[2] - ct[2]) * kPackScale);
    const float2 ax = make_float2(a0, a0), ay = make_float2(a1, a1), az = make_float2(a2, a2);
    float2 qq = make_float2(0.f, 0.f), cx = qq, cy = qq, cz = qq, dx = qq, dy = qq, dz = qq;
#pragma unroll 4
    for (int k2 = 0; k2 < q2; k2++)
      adj_pair32x2<GUARD>(ax, ay, az, tile[3 * k2], tile[3 * k2 + 1], tile[3 * k2 + 2], eps2, qq, cx, cy, cz, dx, dy,
                          dz);
    acc += (double)qq.x + (double)qq.y;
  }
  if (k < q) qbar[(long)s * q + k] = kBiotSavart / kPackScale * acc;
}

// 1-D barycentric basis on the leaf's Chebyshev proxies and its derivative,
// without a range check (displaced particles may leave their leaf).
__device__ __forceinline__ void bli_free_deriv(double t, double lo, double hi, int n, const BliTable& tab, double* f,
                                               double* df) {
  const double range = 0.5 * (hi - lo), offset = 0.5 * (hi + lo);
  int hit = -1;
  for (int i = 0; i <= n; i++)
    if (hit < 0 && fabs(t - (tab.cosv[i] * range + offset)) < 1e-15) hit = i;
  if (hit >= 0) {
    const double th = tab.cosv[hit] * range + offset;
    double sum = 0;
    for (int a = 0; a <= n; a++) {
      f[a] = a == hit ? 1.0 : 0.0;
      df[a] = a == hit ? 0.0 : (tab.w[a] / tab.w[hit]) / (th - (tab.cosv[a] * range + offset));
      sum += df[a];
    }
    df[hit] = -sum;
    return;
  }
  double S = 0, T = 0;
  for (int k = 0; k <= n; k++) {
    const double dk = t - (tab.cosv[k] * range + offset);
    const double r = tab.w[k] / dk;
    f[k] = r;
    S += r;
    T += r / dk;
  }
  const double iS = 1.0 / S, TS = T * iS;
  for (int a = 0; a <= n; a++) {
    f[a] *= iS;
    df[a] = f[a] * (TS - 1.0 / (t - (tab.cosv[a] * range + offset)));
  }
}

__device__ __forceinline__ void atan_grad2(double u, int iu, double su, double w, int iw, double sw, double* gr) {
  const double den = 1.0 / (u * u + w * w);
  gr[0] = gr[1] = gr[2] = 0;
  gr[iu] += w * su * den;
  gr[iw] -= u * sw * den;
}

// Anterpolation adjoint: particle j of tree leaf f (blockIdx.x) adds
// sum_k B_k(y_j) Qbar_k to qbar_j and q_j sum_k grad B_k(y_j) Qbar_k to ybar_j,
// B_k = Lx_a(xi(y)) Ly_b(eta(y)) on the leaf's face.
__global__ void k_tree_sources_T(TreeGeom tg, StepGeom fg, BliTable tab, const double4* __restrict__ psrc,
                                 const double* __restrict__ qbl, double* __restrict__ qbar,
                                 double* __restrict__ ybar) {
  extern __shared__ double sq[];  // the leaf's adjoint proxy strengths, qx
  const int f = blockIdx.x, npl = tg.npl, n = tg.n, n1 = n + 1, qx = n1 * n1;
  const long N = tg.N;
  const int panel = fg.offset + f;
  for (int k = threadIdx.x; k < qx; k += blockDim.x) sq[k] = qbl[(long)panel * qx + k];
  __syncthreads();
  const double* bd = tg.fbounds + 4 * panel;
  const int face = tg.fface[panel];
  for (int jj = threadIdx.x; jj < npl; jj += blockDim.x) {
    const long o = (long)f * npl + jj;
    const double4 s = psrc[o];
    double xi, eta;
    xieta_from_xyz_face(s.x, s.y, s.z, face, xi, eta);
    double fx[kMaxDegree + 1], dfx[kMaxDegree + 1], fe[kMaxDegree + 1], dfe[kMaxDegree + 1];
    bli_free_deriv(xi, bd[0], bd[1], n, tab, fx, dfx);
    bli_free_deriv(eta, bd[2], bd[3], n, tab, fe, dfe);
    double val = 0, dxi = 0, deta = 0;
    for (int a = 0; a <= n; a++)
      for (int b = 0; b <= n; b++) {
        const double qk = sq[a * n1 + b];
        val = fma(fx[a] * fe[b], qk, val);
        dxi = fma(dfx[a] * fe[b], qk, dxi);
        deta = fma(fx[a] * dfe[b], qk, deta);
      }
    double gxi[3], geta[3];
    const double X = s.x, Y = s.y, Z = s.z;
    switch (face) {
      case 0: atan_grad2(Y, 1, 1, X, 0, 1, gxi); atan_grad2(Z, 2, 1, X, 0, 1, geta); break;
      case 1: atan_grad2(-X, 0, -1, Y, 1, 1, gxi); atan_grad2(Z, 2, 1, Y, 1, 1, geta); break;
      case 2: atan_grad2(Y, 1, 1, X, 0, 1, gxi); atan_grad2(-Z, 2, -1, X, 0, 1, geta); break;
      case 3: atan_grad2(-X, 0, -1, Y, 1, 1, gxi); atan_grad2(-Z, 2, -1, Y, 1, 1, geta); break;
      case 4: atan_grad2(Y, 1, 1, Z, 2, 1, gxi); atan_grad2(-X, 0, -1, Z, 2, 1, geta); break;
      default: atan_grad2(-Y, 1, -1, Z, 2, 1, gxi); atan_grad2(-X, 0, -1, Z, 2, 1, geta); break;
    }
    qbar[o] += val;
    for (int c = 0; c < 3; c++) ybar[c * N + o] += s.w * (dxi * gxi[c] + deta * geta[c]);
  }
}

// Transposed spectral-FMM interactions: one group of G lanes per source panel
// s (kT / G groups per block; G = q rounded up to a power of two for q <= 32,
// the whole block above), lane k its proxy k, over the target panels whose
// list holds s: Qbar_s,k = K sum g c.d and ybar_s,k = K S_s,k sum [g c -
// g^2 (c.d) d], c = Tbar_t,i x x_t,i, d = y_s,k - x_t,i (y: the stage's
// displaced proxy).  Float64, or mixed: d' = d kPackScale from coordinates
// packed relative to the two panels' centres (their offset rounded once per
// entry), one source against two targets per paired FP32 instruction
// (adj_pair32x2), per-entry float32 sums added into float64.  Writes qbar
// [panels*q]; position adjoints of leaf proxies to ybar_leaf [3][leaves*q],
// of non-leaf proxies to ybar_nl [3][offset*q].
template <int G, bool GUARD, bool MIXED>
__global__ void __launch_bounds__(kT) k_spec_interact_T(StepGeom g, const int* __restrict__ tstart,
                                                       const int* __restrict__ ttgt, const double* __restrict__ tbar,
                                                       const double4* __restrict__ src, double* __restrict__ qbar,
                                                       double* __restrict__ ybar_leaf, double* __restrict__ ybar_nl) {
  constexpr int S = kT / G;
  __shared__ double sd64[6][kT];                  // float64: x, y, z, c of each group's target panel
  __shared__ float4 sd32[S][3 * ((G + 1) / 2)];  // mixed: pairs of packed targets and c
  const int gi = threadIdx.x / G, k = threadIdx.x % G, base = gi * G;
  const int s = blockIdx.x * S + gi, q = g.q, qh = (q + 1) >> 1;
  const long pn = (long)g.panels * q;
  const bool panel = s < g.panels;
  const bool act = panel && k < q;
  const unsigned lanes = G >= 32 ? 0xffffffffu : (((1u << G) - 1u) << (threadIdx.x & 31 & ~(G - 1)));
  auto sync = [&] {
    if (G > 32) __syncthreads();
    else __syncwarp(lanes);
  };
  const double4 y = src[panel ? (long)s * q + (k < q ? k : 0) : 0];
  const double* cs = g.pd_centre + 4 * (long)(panel ? s : 0);
  const float ysx = (float)((y.x - cs[0]) * kPackScale), ysy = (float)((y.y - cs[1]) * kPackScale),
              ysz = (float)((y.z - cs[2]) * kPackScale);
  const float feps = (float)g.eps;
  const float2 eps2 = make_float2(feps, feps);
  double qb = 0, bx = 0, by = 0, bz = 0;
  const int e0 = panel ? tstart[s] : 0, e1 = panel ? tstart[s + 1] : 0;
  for (int e = e0; e < e1; e++) {
    const long tb = (long)ttgt[e] * q;
    sync();
    if constexpr (MIXED) {
      const double* ct = g.pd_centre + 4 * (long)ttgt[e];
      for (int i = k; i < 2 * qh; i += G) {
        if (i < q)
          adj_stage(sd32[gi], i, g.px[tb + i], g.px[pn + tb + i], g.px[2 * pn + tb + i], tbar[tb + i],
                    tbar[pn + tb + i], tbar[2 * pn + tb + i], ct);
        else
          adj_stage_zero(sd32[gi], i);
      }
      sync();
      if (act) {
        const float a0 = ysx + (float)((cs[0] - ct[0]) * kPackScale), a1 = ysy + (float)((cs[1] - ct[1]) * kPackScale),
                    a2 = ysz + (float)((cs[2] - ct[2]) * kPackScale);
        const float2 ax = make_float2(a0, a0), ay = make_float2(a1, a1), az = make_float2(a2, a2);
        float2 qq = make_float2(0.f, 0.f), cx = qq, cy = qq, cz = qq, dx = qq, dy = qq, dz = qq;
        for (int k2 = 0; k2 < qh; k2++)
          adj_pair32x2<GUARD>(ax, ay, az, sd32[gi][3 * k2], sd32[gi][3 * k2 + 1], sd32[gi][3 * k2 + 2], eps2, qq, cx,
                              cy, cz, dx, dy, dz);
        qb += (double)qq.x + (double)qq.y;
        bx += ((double)cx.x + (double)cx.y) - 2.0 * ((double)dx.x + (double)dx.y);
        by += ((double)cy.x + (double)cy.y) - 2.0 * ((double)dy.x + (double)dy.y);
        bz += ((double)cz.x + (double)cz.y) - 2.0 * ((double)dz.x + (double)dz.y);
      }
    } else {
      for (int i = k; i < q; i += G) {
        const double x = g.px[tb + i], yy = g.px[pn + tb + i], z = g.px[2 * pn + tb + i];
        const double a = tbar[tb + i], b = tbar[pn + tb + i], c = tbar[2 * pn + tb + i];
        sd64[0][base + i] = x;
        sd64[1][base + i] = yy;
        sd64[2][base + i] = z;
        sd64[3][base + i] = b * z - c * yy;
        sd64[4][base + i] = c * x - a * z;
        sd64[5][base + i] = a * yy - b * x;
      }
      sync();
      if (act)
        for (int i = 0; i < q; i++) {
          const double dx = y.x - sd64[0][base + i], dy = y.y - sd64[1][base + i], dz = y.z - sd64[2][base + i];
          const double cx = sd64[3][base + i], cy = sd64[4][base + i], cz = sd64[5][base + i];
          const double r2 = fma(dx, dx, fma(dy, dy, dz * dz));
          double gg = recip_nr(fma(0.5, r2, g.eps));
          if (GUARD) gg = r2 > 0.0 ? gg : 0.0;
          const double sdot = fma(cx, dx, fma(cy, dy, cz * dz));
          qb = fma(gg, sdot, qb);
          const double t = gg * gg * sdot;
          bx = fma(gg, cx, fma(-t, dx, bx));
          by = fma(gg, cy, fma(-t, dy, by));
          bz = fma(gg, cz, fma(-t, dz, bz));
        }
    }
  }
  if (!act) return;
  const long o = (long)s * q + k;
  qbar[o] = (MIXED ? kBiotSavart / kPackScale : kBiotSavart) * qb;
  if (s >= g.offset) {
    const long ln = (long)g.leaves * q, l = o - (long)g.offset * q;
    ybar_leaf[l] = kBiotSavart * y.w * bx;
    ybar_leaf[ln + l] = kBiotSavart * y.w * by;
    ybar_leaf[2 * ln + l] = kBiotSavart * y.w * bz;
  } else {
    const long nn = (long)g.offset * q;
    ybar_nl[o] = kBiotSavart * y.w * bx;
    ybar_nl[nn + o] = kBiotSavart * y.w * by;
    ybar_nl[2 * nn + o] = kBiotSavart * y.w * bz;
  }
}

template <int G>
void launch_spec_interact_T_g(const StepGeom& g, bool mixed, const int* tstart, const int* ttgt, const double* tbar,
                              const double4* src, double* qbar, double* ybar_leaf, double* ybar_nl, cudaStream_t st) {
  const unsigned blocks = (unsigned)((g.panels + kT / G - 1) / (kT / G));
  const bool guard = !(g.eps > 0);
  if (mixed) {
    if (guard) SB_LAUNCH((k_spec_interact_T<G, true, true>), blocks, kT, 0, st, g, tstart, ttgt, tbar, src, qbar, ybar_leaf, ybar_nl);
    else SB_LAUNCH((k_spec_interact_T<G, false, true>), blocks, kT, 0, st, g, tstart, ttgt, tbar, src, qbar, ybar_leaf, ybar_nl);
  } else {
    if (guard) SB_LAUNCH((k_spec_interact_T<G, true, false>), blocks, kT, 0, st, g, tstart, ttgt, tbar, src, qbar, ybar_leaf, ybar_nl);
    else SB_LAUNCH((k_spec_interact_T<G, false, false>), blocks, kT, 0, st, g, tstart, ttgt, tbar, src, qbar, ybar_leaf, ybar_nl);
  }
}

// Non-leaf proxy positions, reversed: y_i = proj(p_i + h sum_m B_mi v[row_i + m])
// (k_nonleaf_positions); vbar[c][row_i + m] += h B_mi J(p)^T ybar_i with
// J(p)^T ybar = (ybar - yhat (yhat.ybar)) / |p|.  Proxies of one leaf row add
// into the same velocity entries: double atomics.
__global__ void k_nonleaf_positions_T(StepGeom g, double h, const double* __restrict__ vprev,
                                      const double* __restrict__ ybar_nl, double* __restrict__ vbar) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const int q = g.q;
  const long np = (long)g.offset * q;
  if (i >= np) return;
  const long pn = (long)g.panels * q, ln = (long)g.leaves * q;
  const long row = (long)g.il_row[i] * q;
  double px = g.px[i], py = g.px[pn + i], pz = g.px[2 * pn + i];
  for (int m = 0; m < q; m++) {
    const double bm = g.il_basis[m * np + i];
    px += (h * vprev[row + m]) * bm;
    py += (h * vprev[ln + row + m]) * bm;
    pz += (h * vprev[2 * ln + row + m]) * bm;
  }
  const double r = sqrt(px * px + py * py + pz * pz), ir = 1.0 / r;
  const double hx = px * ir, hy = py * ir, hz = pz * ir;
  const double gx = ybar_nl[i], gy = ybar_nl[np + i], gz = ybar_nl[2 * np + i];
  const double dd = hx * gx + hy * gy + hz * gz;
  const double ax = h * (gx - hx * dd) * ir, ay = h * (gy - hy * dd) * ir, az = h * (gz - hz * dd) * ir;
  for (int m = 0; m < q; m++) {
    const double bm = g.il_basis[m * np + i];
    atomicAdd(vbar + row + m, ax * bm);
    atomicAdd(vbar + ln + row + m, ay * bm);
    atomicAdd(vbar + 2 * ln + row + m, az * bm);
  }
}

}  // namespace

void launch_spectral_velocity_adjoint(const StepGeom& g, const int* tstart, const int* ttgt, const double* vbar,
                                      const double4* src, double* tbar, double* qbar, double* ybar_leaf,
                                      double* ybar_nl, bool mixed, cudaStream_t st) {
  const int q = g.q;
  const long pn = (long)g.panels * q, ln = (long)g.leaves * q, off = (long)g.offset * q;
  // the leaf targets' adjoint is vbar itself (leaf proxies = particles); the
  // downward pass transposed accumulates it up the tree
  cudaMemsetAsync(tbar, 0, sizeof(double) * 3 * pn, st);
  for (int c = 0; c < 3; c++)
    cudaMemcpyAsync(tbar + c * pn + off, vbar + c * ln, sizeof(double) * ln, cudaMemcpyDeviceToDevice, st);
  for (int lev = g.levels - 2; lev >= 0; lev--) {
    const long work = (6L << (2 * lev)) * q * 3;
    SB_LAUNCH(k_tree_up3, blocks_for(work, 256), 256, 0, st, g, lev, tbar);
  }
  if (q <= 4) launch_spec_interact_T_g<4>(g, mixed, tstart, ttgt, tbar, src, qbar, ybar_leaf, ybar_nl, st);
  else if (q <= 16) launch_spec_interact_T_g<16>(g, mixed, tstart, ttgt, tbar, src, qbar, ybar_leaf, ybar_nl, st);
  else if (q <= 32) launch_spec_interact_T_g<32>(g, mixed, tstart, ttgt, tbar, src, qbar, ybar_leaf, ybar_nl, st);
  else launch_spec_interact_T_g<kT>(g, mixed, tstart, ttgt, tbar, src, qbar, ybar_leaf, ybar_nl, st);
  // the strengths' upward pass transposed: interpolate their adjoints down
  for (int lev = 0; lev < g.levels - 1; lev++) {
    const long work = (6L << (2 * (lev + 1))) * q;
    SB_LAUNCH(k_tree_down1, blocks_for(work, 256), 256, 0, st, g, lev, qbar);
  }
}

void launch_nonleaf_positions_adjoint(const StepGeom& g, double h, const double* vprev, const double* ybar_nl,
                                      double* vbar, cudaStream_t st) {
  const long np = (long)g.offset * g.q;
  if (np > 0) SB_LAUNCH(k_nonleaf_positions_T, blocks_for(np, 256), 256, 0, st, g, h, vprev, ybar_nl, vbar);
}

void launch_tree_velocity_adjoint(const TreeGeom& tg, const StepGeom& fg, const BliTable& ftab,
                                  const TreeAdjointLists& tl, const double* x, const double* y, const double* z,
                                  const double* vbar, const double4* psrc, double* tbar, double* qbl, double* qbar,
                                  double* ybar, bool mixed, cudaStream_t st) {
  const int qx = fg.q, Pf = fg.panels;
  const long pn = (long)Pf * qx;
  // leaf interpolation, transposed; non-leaf rows start at zero
  cudaMemsetAsync(tbar, 0, sizeof(double) * 3 * pn, st);
  SB_LAUNCH(k_tree_to_particles_T, (unsigned)fg.leaves, kT, sizeof(double) * 3 * tg.npl, st, tg, fg, vbar, tbar);
  // downward pass, transposed: accumulate up the tree
  for (int lev = fg.levels - 2; lev >= 0; lev--) {
    const long work = (6L << (2 * lev)) * qx * 3;
    SB_LAUNCH(k_tree_up3, blocks_for(work, 256), 256, 0, st, fg, lev, tbar);
  }
  // well-separated interactions, transposed
  if (mixed) {
    if (fg.eps > 0) SB_LAUNCH(k_tree_cc_T32<false>, (unsigned)Pf, kT, 0, st, fg, tl.cc_tstart, tl.cc_ttgt, tbar, qbl);
    else SB_LAUNCH(k_tree_cc_T32<true>, (unsigned)Pf, kT, 0, st, fg, tl.cc_tstart, tl.cc_ttgt, tbar, qbl);
  } else if (fg.eps > 0) {
    SB_LAUNCH(k_tree_cc_T<false>, (unsigned)Pf, kT, 0, st, fg, tl.cc_tstart, tl.cc_ttgt, tbar, qbl);
  } else {
    SB_LAUNCH(k_tree_cc_T<true>, (unsigned)Pf, kT, 0, st, fg, tl.cc_tstart, tl.cc_ttgt, tbar, qbl);
  }
  // upward pass, transposed: interpolate down the tree
  for (int lev = 0; lev < fg.levels - 1; lev++) {
    const long work = (6L << (2 * (lev + 1))) * qx;
    SB_LAUNCH(k_tree_down1, blocks_for(work, 256), 256, 0, st, fg, lev, qbl);
  }
  // near field, transposed (writes qbar, ybar), then the anterpolation adjoint (adds)
  const size_t sm = sizeof(double) * 6 * tg.npl;
  static std::atomic<unsigned long long> attr{0};
  raise_smem_once(attr, 64 * 1024, k_tree_near_T<false>, k_tree_near_T<true>);
  const int nth = tg.npl <= 256 ? 256 : 512;
  if (mixed) {
    const size_t sm32 = sizeof(float4) * 3 * ((tg.npl + 1) / 2);
    if (tg.eps > 0)
      SB_LAUNCH(k_tree_near_T32<false>, (unsigned)fg.leaves, nth, sm32, st, tg, fg, tl.near_tstart, tl.near_ttgt, x, y,
                z, vbar, psrc, qbar, ybar);
    else
      SB_LAUNCH(k_tree_near_T32<true>, (unsigned)fg.leaves, nth, sm32, st, tg, fg, tl.near_tstart, tl.near_ttgt, x, y,
                z, vbar, psrc, qbar, ybar);
  } else if (tg.eps > 0)
    SB_LAUNCH(k_tree_near_T<false>, (unsigned)fg.leaves, nth, sm, st, tg, tl.near_tstart, tl.near_ttgt, x, y, z, vbar,
              psrc, qbar, ybar);
  else
    SB_LAUNCH(k_tree_near_T<true>, (unsigned)fg.leaves, nth, sm, st, tg, tl.near_tstart, tl.near_ttgt, x, y, z, vbar,
              psrc, qbar, ybar);
  SB_LAUNCH(k_tree_sources_T, (unsigned)fg.leaves, kT, sizeof(double) * qx, st, tg, fg, ftab, psrc, qbl, qbar, ybar);
}

}  // namespace sbslpm
