// Shallow-water (SWE v2) finite-difference tendencies, edge unification and
// arrival values, sm_100a.
//
// This file is compiled with -fmad=false: every multiply and add is rounded
// separately and evaluated in the reference's operand order, so that with
// the host-precomputed node tables (tan, pow, finite-difference weights,
// computed with the reference's own expressions and libm) these kernels
// reproduce the reference's arithmetic.  The one-sided and centred
// finite-difference stencils divide by node spacings of O(panel width), so
// rounding differences would otherwise be amplified by 1/h per derivative.
//
// k_swe_tendency: one thread per grid point, PPB leaf panels per block, the
// panel's fields and derivatives in shared memory (19 arrays of q doubles per
// panel).  swe_tendency_computation_2 (src/swe_time_step_2_impl.hpp:10-128):
//   per point:   xietavec_from_xyzvec (src/cubed_sphere_transforms_impl.hpp:242-276),
//                zeta_f = vor + 2 Omega z, h v, |v|^2/2
//   per panel:   single_panel_curl_rad_comp_fd, single_panel_lap_fd (x2),
//                single_panel_div_fd (src/deriv_funcs_impl.hpp:94-185,
//                391-441, 510-543, 591-618, 661-698)
//   per point:   vorticity, divergence and height tendencies, zeroed within
//                1e-5 of the poles; then modify_tendencies
//                (src/swe_time_step_2.cpp:768-783) when base tendencies are given.
#include <cuda_runtime.h>

#include "../../include/sbslpm.h"
#include "device_common.cuh"
#include "swe_kernels.cuh"

namespace sbslpm {
namespace {

using dev::blocks_for;

constexpr double kFilterCoeff = 0.0005;  // spatial_filter_vals, src/deriv_funcs_impl.hpp:393

// Derivative at node (i, j) along xi (dir 0: stride n1 over i) or eta (dir 1:
// stride 1 over j) of f (fd_deriv_xi / fd_deriv_eta).  W: [n1][4] weights of
// this panel and direction.
__device__ __forceinline__ double fd1(const double* f, const double* W, int n1, int idx, int p, int stride) {
  const int d = n1 - 1;
  if (p == 0) {
    const double* w = W;
    return (w[0] * f[idx] + w[1] * f[idx + stride] + w[2] * f[idx + 2 * stride]) / w[3];
  }
  if (p == d) {
    const double* w = W;
    return -(w[0] * f[idx] + w[1] * f[idx - stride] + w[2] * f[idx - 2 * stride]) / w[3];
  }
  const double* w = W + 4 * p;
  return (w[0] * f[idx - stride] + w[1] * f[idx] + w[2] * f[idx + stride]) / w[3];
}

// spatial_filter_vals at node (i, j): FW [n1][2] neighbour weights.
__device__ __forceinline__ double filter_at(const double* f, const double* FW, int n1, int i, int j) {
  const int d = n1 - 1, idx = i * n1 + j;
  double out = (1.0 - kFilterCoeff) * f[idx];
  int i1, i2, j1, j2;
  if (i == 0) {
    i1 = i + 1;
    i2 = i + 2;
  } else if (i == d) {
    i1 = i - 1;
    i2 = i - 2;
  } else {
    i1 = i - 1;
    i2 = i + 1;
  }
  if (j == 0) {
    j1 = j + 1;
    j2 = j + 2;
  } else if (j == d) {
    j1 = j - 1;
    j2 = j - 2;
  } else {
    j1 = j - 1;
    j2 = j + 1;
  }
  out += FW[2 * i] * f[i2 * n1 + j];
  out += FW[2 * i + 1] * f[i1 * n1 + j];
  out += FW[2 * j] * f[i * n1 + j2];
  out += FW[2 * j + 1] * f[i * n1 + j1];
  return out;
}

enum {
  kXV, kEV, kDX, kDY, kSU, kDP,                       // point values
  kXVx, kEVx, kXVe, kEVe, kSUx, kSUe, kDPx, kDPe, kDXx, kDYe,  // first derivatives
  kCURL, kLAPS, kLAPD,                                // pre-filter curl and Laplacians
  kArrays
};

__global__ void k_swe_tendency(StepGeom g, SweGeom s, const double* __restrict__ x, const double* __restrict__ y,
                               const double* __restrict__ z, const double* __restrict__ vel,
                               const double* __restrict__ vors, const double* __restrict__ divs,
                               const double* __restrict__ height, const double* __restrict__ surface, double dts,
                               const double* __restrict__ tprev, const double* __restrict__ base_div,
                               const double* __restrict__ base_h, double* __restrict__ tend, int ppb) {
  extern __shared__ double sh[];
  const int q = g.q, n1 = g.degree + 1;
  const long ln = (long)g.leaves * q;
  const int lp = threadIdx.x / q, j = threadIdx.x % q;
  const int panel = blockIdx.x * ppb + lp;  // leaf panel, relative
  const bool live = lp < ppb && panel < g.leaves;
  double* a = sh + (long)lp * kArrays * q;
  auto A = [&](int k) { return a + k * q; };
  const long o = (long)panel * q + j;
  const int ii = j / n1, jj = j % n1;
  const double* W = s.fd + (long)panel * 2 * n1 * 4;
  const double* Wx = W;
  const double* We = W + n1 * 4;
  const double Xn = live ? s.ntan[(long)panel * 2 * n1 + ii] : 0.0;
  const double Yn = live ? s.ntan[(long)panel * 2 * n1 + n1 + jj] : 0.0;

  double vx = 0, vy = 0, vz = 0, zz = 0, vor = 0, div = 0;
  if (live) {
    const double xx = x[o], yy = y[o];
    zz = z[o];
    vx = vel[o];
    vy = vel[ln + o];
    vz = vel[2 * ln + o];
    vor = vors[o];
    div = divs[o];
    double H = height[o];
    double S = surface ? surface[o] : H;
    if (tprev) {
      H = H + dts * tprev[2 * ln + o];
      if (!surface) S = H;
    }
    // xietavec_from_xyzvec at the grid point (its own xi/eta tangents precomputed)
    double xi_c, eta_c;
    if (fabs(zz) < 1 - 1e-16) {
      const double X = s.ptan[2 * o], Y = s.ptan[2 * o + 1];
      const int face = s.pface[o];
      const double lon_comp = (-yy * vx + xx * vy) / sqrt(xx * xx + yy * yy);
      const double colat_comp = ((xx * vx + yy * vy) * zz - (xx * xx + yy * yy) * vz) / sqrt(xx * xx + yy * yy);
      const double X2 = X * X, Y2 = Y * Y;
      const double C = sqrt(1 + X2), D = sqrt(1 + Y2), delta = 1 + X2 + Y2;
      if (face <= 3) {
        xi_c = C * D / sqrt(delta) * lon_comp;
        eta_c = -1.0 * colat_comp + X * Y / sqrt(delta) * lon_comp;
      } else if (face == 4) {
        xi_c = 1.0 / sqrt(X2 + Y2) * (D * X * colat_comp - D * Y / sqrt(delta) * lon_comp);
        eta_c = 1.0 / sqrt(X2 + Y2) * (C * Y * colat_comp + C * X / sqrt(delta) * lon_comp);
      } else {
        xi_c = -1.0 / sqrt(X2 + Y2) * (D * X * colat_comp - D * Y / sqrt(delta) * lon_comp);
        eta_c = -1.0 / sqrt(X2 + Y2) * (C * Y * colat_comp + C * X / sqrt(delta) * lon_comp);
      }
    } else {
      xi_c = vx;
      eta_c = vy;
    }
    const double zetaf = vor + 2 * g.omega * zz;
    // div_fd scales its inputs by 1/sqrt(delta) at the panel nodes before differentiating
    const double dn = 1 + Xn * Xn + Yn * Yn;
    A(kDX)[j] = (H * xi_c) / sqrt(dn);
    A(kDY)[j] = (H * eta_c) / sqrt(dn);
    A(kXV)[j] = xi_c * zetaf;
    A(kEV)[j] = eta_c * zetaf;
    A(kSU)[j] = S;
    A(kDP)[j] = 0.5 * (vx * vx + vy * vy + vz * vz);
  }
  __syncthreads();
  if (live) {
    const int sx = n1, se = 1;
    A(kXVx)[j] = fd1(A(kXV), Wx, n1, j, ii, sx);
    A(kEVx)[j] = fd1(A(kEV), Wx, n1, j, ii, sx);
    A(kXVe)[j] = fd1(A(kXV), We, n1, j, jj, se);
    A(kEVe)[j] = fd1(A(kEV), We, n1, j, jj, se);
    A(kSUx)[j] = fd1(A(kSU), Wx, n1, j, ii, sx);
    A(kSUe)[j] = fd1(A(kSU), We, n1, j, jj, se);
    A(kDPx)[j] = fd1(A(kDP), Wx, n1, j, ii, sx);
    A(kDPe)[j] = fd1(A(kDP), We, n1, j, jj, se);
    A(kDXx)[j] = fd1(A(kDX), Wx, n1, j, ii, sx);
    A(kDYe)[j] = fd1(A(kDY), We, n1, j, jj, se);
  }
  __syncthreads();
  double hdiv = 0;
  if (live) {
    const int sx = n1, se = 1;
    const double C2 = 1 + Xn * Xn, D2 = 1 + Yn * Yn, delta = 1 + Xn * Xn + Yn * Yn;
    // single_panel_lap_fd of the surface and of |v|^2/2
    {
      const double xixi = fd1(A(kSUx), Wx, n1, j, ii, sx), etaeta = fd1(A(kSUe), We, n1, j, jj, se);
      const double xieta = fd1(A(kSUx), We, n1, j, jj, se), etaxi = fd1(A(kSUe), Wx, n1, j, ii, sx);
      const double mix = 0.5 * (xieta + etaxi);
      A(kLAPS)[j] = delta * (xixi / C2 + etaeta / D2 + 2.0 * Xn * Yn / (C2 * D2) * mix);
    }
    {
      const double xixi = fd1(A(kDPx), Wx, n1, j, ii, sx), etaeta = fd1(A(kDPe), We, n1, j, jj, se);
      const double xieta = fd1(A(kDPx), We, n1, j, jj, se), etaxi = fd1(A(kDPe), Wx, n1, j, ii, sx);
      const double mix = 0.5 * (xieta + etaxi);
      A(kLAPD)[j] = delta * (xixi / C2 + etaeta / D2 + 2.0 * Xn * Yn / (C2 * D2) * mix);
    }
    // single_panel_curl_rad_comp_fd
    {
      const double C = sqrt(1 + Xn * Xn), D = sqrt(1 + Yn * Yn);
      const double xdx = A(kXVx)[j], xde = A(kEVx)[j], edx = A(kXVe)[j], ede = A(kEVe)[j];
      A(kCURL)[j] = -sqrt(delta) * (Xn * Yn / (C * D) * (ede / D - xdx / C) - edx / D + xde / C);
      // single_panel_div_fd (no filter)
      hdiv = s.pow15[o] / (C * D) * (A(kDXx)[j] / C + A(kDYe)[j] / D);
    }
  }
  __syncthreads();
  if (!live) return;
  const double curl = filter_at(A(kCURL), s.filt, n1, ii, jj);
  double hlap = filter_at(A(kLAPS), s.filt, n1, ii, jj);
  const double dlap = filter_at(A(kLAPD), s.filt, n1, ii, jj);
  const double abs_vor = vor + 2.0 * g.omega * zz;
  const double vt = -div * abs_vor - 2.0 * g.omega * vz;
  hlap *= s.g_over_a;
  double dtn = curl - hlap - dlap;
  double htn = hdiv;
  if (1.0 - fabs(zz) < 1e-5) {
    dtn = 0.0;
    htn = 0.0;
  }
  if (base_div) dtn -= base_div[o];
  if (base_h) htn -= base_h[o];
  tend[o] = vt;
  tend[ln + o] = dtn;
  tend[2 * ln + o] = htn;
}

// unify_boundary_vals (src/initialize_cubed_sphere.cpp:328-370): the points of
// one position are summed in [leaf][q] order, starting from zero, and every
// copy gets the sum divided by their count; rounds > 1 applies it that many
// times in a row (after the first round the copies are equal, but a sum of
// three or four equal values divided by their count can differ from the
// value in the last bit, so repeated calls are not exactly idempotent).
__global__ void k_unify(SweGeom s, double* __restrict__ f0, double* __restrict__ f1, double* __restrict__ f2,
                        int rounds) {
  const long u = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (u >= s.unique) return;
  const int b = s.ustart[u], e = s.ustart[u + 1];
  const double cnt = (double)(e - b);
  double* f[3] = {f0, f1, f2};
#pragma unroll
  for (int k = 0; k < 3; k++) {
    if (!f[k]) continue;
    double sum = 0;
    for (int m = b; m < e; m++) sum += f[k][s.umem[m]];
    double v = sum / cnt;
    for (int r = 1; r < rounds; r++) {
      sum = 0;
      for (int m = b; m < e; m++) sum += v;
      v = sum / cnt;
    }
    for (int m = b; m < e; m++) f[k][s.umem[m]] = v;
  }
}

// swe_compute_arrival_values_2 (src/swe_time_step_2.cpp:498-627): only the
// forward-Euler update with the first-stage tendencies reaches the result.
__global__ void k_swe_arrival(long n, const double* __restrict__ tend1, double dt, const double* __restrict__ vors,
                              double* __restrict__ divs, double* __restrict__ height, double* __restrict__ avor) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  avor[i] = vors[i] + dt * tend1[i];
  divs[i] = divs[i] + dt * tend1[n + i];
  height[i] = height[i] + dt * tend1[2 * n + i];
}

}  // namespace

void launch_swe_tendency(const StepGeom& g, const SweGeom& s, const double* x, const double* y, const double* z,
                         const double* vel, const double* vors, const double* divs, const double* height,
                         const double* surface, double dts, const double* tprev, const double* base_div,
                         const double* base_h, double* tend, cudaStream_t st) {
  const int q = g.q;
  int ppb = 128 / q;
  if (ppb < 1) ppb = 1;
  const int threads = ((ppb * q + 31) / 32) * 32;
  const size_t smem = (size_t)ppb * kArrays * q * sizeof(double);
  SB_LAUNCH(k_swe_tendency, blocks_for(g.leaves, ppb), threads, smem, st, g, s, x, y, z, vel, vors, divs, height,
            surface, dts, tprev, base_div, base_h, tend, ppb);
}

void launch_unify(const SweGeom& s, double* f0, double* f1, double* f2, int rounds, cudaStream_t st) {
  SB_LAUNCH(k_unify, blocks_for(s.unique, 256), 256, 0, st, s, f0, f1, f2, rounds);
}

void launch_swe_arrival(const StepGeom& g, const double* tend1, double dt, const double* vors, double* divs,
                        double* height, double* avor, cudaStream_t st) {
  const long n = (long)g.leaves * g.q;
  SB_LAUNCH(k_swe_arrival, blocks_for(n, 256), 256, 0, st, n, tend1, dt, vors, divs, height, avor);
}

}  // namespace sbslpm
