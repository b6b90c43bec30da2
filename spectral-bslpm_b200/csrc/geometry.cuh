// Cubed-sphere geometry shared by host setup code and device kernels.
//
// Each function restates the reference's arithmetic with the same operand
// order, so host (glibc) results match the reference bit for bit and device
// results differ only by the last-bit differences of CUDA's tan/atan and of
// fused multiply-adds.
#pragma once

#include <math.h>

#ifdef __CUDACC__
#define SB_HD __host__ __device__ __forceinline__
#else
#define SB_HD inline
#endif

namespace sbslpm {

constexpr double kPi = 3.14159265358979323846;
constexpr int kMaxDegree = 10;
constexpr int kMaxQ = (kMaxDegree + 1) * (kMaxDegree + 1);
// -1/(4 pi), the Biot-Savart constant (src/fmm_interactions/bve_vel_impl.hpp:115)
constexpr double kBiotSavart = -0.07957747154594767;

// Error bits reported by device code through the context's error word.
enum : unsigned { kErrOutOfPanel = 1u, kErrNonFinite = 2u, kErrBadFace = 4u, kErrTimeout = 8u };

SB_HD int level_start(int level) { return 2 * ((1 << (2 * level)) - 1); }

// face_from_xyz: src/cubed_sphere_transforms_impl.hpp:8-32
SB_HD int face_from_xyz(double x, double y, double z) {
  double ax = fabs(x), ay = fabs(y), az = fabs(z);
  if ((ax >= ay) && (ax >= az)) return x >= 0 ? 0 : 2;
  if ((ay >= ax) && (ay >= az)) return y >= 0 ? 1 : 3;
  return z >= 0 ? 4 : 5;
}

// xyz_from_xieta: src/cubed_sphere_transforms_impl.hpp:34-65
SB_HD void xyz_from_xieta(double xi, double eta, int face, double* xyz) {
  double X = tan(xi), Y = tan(eta);
  double r = 1.0 / sqrt(1 + X * X + Y * Y);
  switch (face) {
    case 0: xyz[0] = r; xyz[1] = X * xyz[0]; xyz[2] = Y * xyz[0]; break;
    case 1: xyz[1] = r; xyz[0] = -X * xyz[1]; xyz[2] = Y * xyz[1]; break;
    case 2: xyz[0] = -r; xyz[1] = X * xyz[0]; xyz[2] = -Y * xyz[0]; break;
    case 3: xyz[1] = -r; xyz[0] = -X * xyz[1]; xyz[2] = -Y * xyz[1]; break;
    case 4: xyz[2] = r; xyz[0] = -Y * xyz[2]; xyz[1] = X * xyz[2]; break;
    default: xyz[2] = -r; xyz[0] = -Y * xyz[2]; xyz[1] = -X * xyz[2]; break;
  }
}

// xieta_from_xyz for a given face: src/cubed_sphere_transforms_impl.hpp:100-123
SB_HD void xieta_from_xyz_face(double x, double y, double z, int face, double& xi, double& eta) {
  switch (face) {
    case 0: xi = atan(y / x); eta = atan(z / x); break;
    case 1: xi = atan(-x / y); eta = atan(z / y); break;
    case 2: xi = atan(y / x); eta = atan(-z / x); break;
    case 3: xi = atan(-x / y); eta = atan(-z / y); break;
    case 4: xi = atan(y / z); eta = atan(-x / z); break;
    default: xi = atan(-y / z); eta = atan(-x / z); break;
  }
}

// project_to_sphere: src/general_utils_impl.hpp:179-185
SB_HD void project_to_sphere(double& x, double& y, double& z) {
  double n = sqrt(x * x + y * y + z * z);
  x /= n;
  y /= n;
  z /= n;
}

// Unit-square bounds of a panel of the uniform quadtree ([-1,1] scaled by
// pi/4 on the sphere; exact dyadic numbers).
struct Bounds {
  double min_xi, max_xi, min_eta, max_eta;
};

// Point location by tree descent (point_locate_panel,
// src/interp_funcs_impl.hpp:114-142), with child ids and bounds computed from
// the uniform quadtree's numbering (refine_cube,
// src/initialize_cubed_sphere.cpp:64-141) instead of read from a panel table.
// Returns the leaf panel id; xi/eta are the point's coordinates on its face.
SB_HD int locate_leaf(double x, double y, double z, int levels, double& xi, double& eta, Bounds& b,
                      unsigned& err) {
  int face = face_from_xyz(x, y, z);
  xieta_from_xyz_face(x, y, z, face, xi, eta);
  b.min_xi = -1;
  b.max_xi = 1;
  b.min_eta = -1;
  b.max_eta = 1;
  int id = face;
  for (int lev = 0; lev < levels - 1; lev++) {
    double mid_xi = 0.5 * kPi / 4.0 * (b.max_xi + b.min_xi);
    double mid_eta = 0.5 * kPi / 4.0 * (b.max_eta + b.min_eta);
    double ux = 0.5 * (b.max_xi + b.min_xi), ue = 0.5 * (b.max_eta + b.min_eta);
    int c;
    if ((xi >= mid_xi) && (eta >= mid_eta)) {
      c = 0;
      b.min_xi = ux;
      b.min_eta = ue;
    } else if ((xi <= mid_xi) && (eta >= mid_eta)) {
      c = 1;
      b.max_xi = ux;
      b.min_eta = ue;
    } else if ((xi <= mid_xi) && (eta <= mid_eta)) {
      c = 2;
      b.max_xi = ux;
      b.max_eta = ue;
    } else if ((xi >= mid_xi) && (eta <= mid_eta)) {
      c = 3;
      b.min_xi = ux;
      b.max_eta = ue;
    } else {
      err |= kErrNonFinite;  // NaN coordinates
      c = 0;
      b.min_xi = ux;
      b.min_eta = ue;
    }
    id = level_start(lev + 1) + 4 * (id - level_start(lev)) + c;
  }
  return id;
}

// One direction of interp_vals_bli (src/interp_funcs_impl.hpp:11-112):
// barycentric Lagrange basis on Chebyshev extrema of [lo, hi].  cosv[i] holds
// cos(pi*i/d) and w[i] the barycentric weights (1/2, -1, 1, ..., +-1/2).
SB_HD void bli_1d(double t, double lo, double hi, int d, const double* cosv, const double* w, double* f,
                  unsigned& err) {
  double range = 0.5 * (hi - lo), offset = 0.5 * (hi + lo);
  if (t < lo - 1e-15 || t > hi + 1e-15) err |= kErrOutOfPanel;
  if (d == 0) {
    f[0] = 1;
    return;
  }
  int hit = -1;
  for (int i = 0; i <= d; i++) {
    double c = cosv[i] * range + offset;
    if (hit < 0 && fabs(t - c) < 1e-15) hit = i;
  }
  if (hit >= 0) {
    for (int i = 0; i <= d; i++) f[i] = (i == hit) ? 1.0 : 0.0;
    return;
  }
  double den = 0;
  for (int i = 0; i <= d; i++) {
    double v = w[i] / (t - (cosv[i] * range + offset));
    f[i] = v;
    den += v;
  }
  for (int i = 0; i <= d; i++) f[i] /= den;
}

}  // namespace sbslpm
