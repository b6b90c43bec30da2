/* CPU restatement of the reference's BVE and SWE backward semi-Lagrangian hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path and the "port"
 * CPU baseline.  The product library never links or calls this file.
 *
 * Every function cites the reference source (file:line, relative to the
 * reference checkout) whose arithmetic it restates.  Expressions keep the
 * reference's operand order and every accumulation keeps the reference's
 * single-thread order (its atomics become owner-computes sums visited in the
 * same order), so the results match the reference built by oracle/Makefile
 * bit for bit when both use the same libm.  Parity is pinned by
 * tests/test_oracle_golden.py against vectors that tests/golden/make_golden.py
 * produced from the reference itself.
 */
#include "bslpm_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define ORC_PI 3.14159265358979323846
#define MAXQ 121

static int g_orc_error = 0;
int orc_error(void) { return g_orc_error; }
void orc_clear_error(void) { g_orc_error = 0; }

/* ---------------- geometry: src/cubed_sphere_transforms_impl.hpp ---------- */

/* face_from_xyz: src/cubed_sphere_transforms_impl.hpp:8-32 */
static int face_from_xyz(double x, double y, double z) {
  double ax = fabs(x), ay = fabs(y), az = fabs(z);
  if ((ax >= ay) && (ax >= az)) return x >= 0 ? 0 : 2;
  if ((ay >= ax) && (ay >= az)) return y >= 0 ? 1 : 3;
  return z >= 0 ? 4 : 5;
}

/* xyz_from_xieta: src/cubed_sphere_transforms_impl.hpp:34-65 */
static void xyz_from_xieta(double xi, double eta, int face, double* xyz) {
  double X = tan(xi), Y = tan(eta);
  switch (face) {
    case 0: xyz[0] = 1.0 / sqrt(1 + X * X + Y * Y); xyz[1] = X * xyz[0]; xyz[2] = Y * xyz[0]; break;
    case 1: xyz[1] = 1.0 / sqrt(1 + X * X + Y * Y); xyz[0] = -X * xyz[1]; xyz[2] = Y * xyz[1]; break;
    case 2: xyz[0] = -1.0 / sqrt(1 + X * X + Y * Y); xyz[1] = X * xyz[0]; xyz[2] = -Y * xyz[0]; break;
    case 3: xyz[1] = -1.0 / sqrt(1 + X * X + Y * Y); xyz[0] = -X * xyz[1]; xyz[2] = -Y * xyz[1]; break;
    case 4: xyz[2] = 1.0 / sqrt(1 + X * X + Y * Y); xyz[0] = -Y * xyz[2]; xyz[1] = X * xyz[2]; break;
    case 5: xyz[2] = -1.0 / sqrt(1 + X * X + Y * Y); xyz[0] = -Y * xyz[2]; xyz[1] = -X * xyz[2]; break;
    default: g_orc_error = 3; xyz[0] = xyz[1] = xyz[2] = 0; break;
  }
}

/* xieta_from_xyz with a given face: src/cubed_sphere_transforms_impl.hpp:100-123 */
static void xieta_from_xyz_face(double x, double y, double z, int face, double* xieta) {
  switch (face) {
    case 0: xieta[0] = atan(y / x); xieta[1] = atan(z / x); break;
    case 1: xieta[0] = atan(-x / y); xieta[1] = atan(z / y); break;
    case 2: xieta[0] = atan(y / x); xieta[1] = atan(-z / x); break;
    case 3: xieta[0] = atan(-x / y); xieta[1] = atan(-z / y); break;
    case 4: xieta[0] = atan(y / z); xieta[1] = atan(-x / z); break;
    default: xieta[0] = atan(-y / z); xieta[1] = atan(-x / z); break;
  }
}

/* xieta_from_xyz choosing the face itself: src/cubed_sphere_transforms_impl.hpp:67-98.
 * Its branch structure picks the same face as face_from_xyz. */
static void xieta_from_xyz(double x, double y, double z, double* xieta) {
  xieta_from_xyz_face(x, y, z, face_from_xyz(x, y, z), xieta);
}

/* project_to_sphere: src/general_utils_impl.hpp:179-185 */
static void project_to_sphere(double* x, double* y, double* z) {
  double n = sqrt(*x * *x + *y * *y + *z * *z);
  *x /= n;
  *y /= n;
  *z /= n;
}

/* gcdist, sphere_tri_area: src/general_utils.cpp:21-44 */
static double gcdist(const double* p1, const double* p2) {
  double dp = p1[0] * p2[0] + p1[1] * p2[1] + p1[2] * p2[2];
  if (dp > 1.0) dp = 1.0;
  if (dp < -1.0) dp = -1.0;
  return acos(dp);
}
static double sphere_tri_area(const double* p1, const double* p2, const double* p3) {
  double p1n[3], p2n[3], p3n[3], a, b, c, s, z;
  memcpy(p1n, p1, sizeof p1n);
  memcpy(p2n, p2, sizeof p2n);
  memcpy(p3n, p3, sizeof p3n);
  p2n[0] -= p3[0], p2n[1] -= p3[1], p2n[2] -= p3[2];
  p3n[0] -= p1[0], p3n[1] -= p1[1], p3n[2] -= p1[2];
  p1n[0] -= p2[0], p1n[1] -= p2[1], p1n[2] -= p2[2];
  a = acos(1 - 0.5 * (p2n[0] * p2n[0] + p2n[1] * p2n[1] + p2n[2] * p2n[2]));
  b = acos(1 - 0.5 * (p3n[0] * p3n[0] + p3n[1] * p3n[1] + p3n[2] * p3n[2]));
  c = acos(1 - 0.5 * (p1n[0] * p1n[0] + p1n[1] * p1n[1] + p1n[2] * p1n[2]));
  s = (a + b + c) / 2;
  z = tan(s / 2) * tan((s - a) / 2) * tan((s - b) / 2) * tan((s - c) / 2);
  return 4 * atan(sqrt(z));
}

/* ---------------- tree: src/initialize_cubed_sphere.cpp ------------------- */

int orc_panel_count(int levels) { return 2 * ((1 << (2 * levels)) - 1); }
int orc_leaf_count(int levels) { return 6 * (1 << (2 * (levels - 1))); }
static int level_start(int level) { return 2 * ((1 << (2 * level)) - 1); }

/* cubed_sphere_panels_init + refine_cube + cubed_sphere_init_2:
 * src/initialize_cubed_sphere.cpp:64-234 */
void orc_panels_init(int levels, orc_panel* p) {
  int P = orc_panel_count(levels);
  memset(p, 0, sizeof(orc_panel) * (size_t)P);
  for (int i = 0; i < 6; i++) {
    p[i].id = i;
    p[i].face = i;
    p[i].min_xi = -1;
    p[i].max_xi = 1;
    p[i].min_eta = -1;
    p[i].max_eta = 1;
    p[i].level = 0;
    p[i].parent = -1;
  }
  for (int i = 0; i < 4; i++) {
    p[i].top = 4;
    p[i].bot = 5;
  }
  p[0].left = 3; p[0].right = 1;
  p[1].left = 0; p[1].right = 2;
  p[2].left = 1; p[2].right = 3;
  p[3].left = 2; p[3].right = 0;
  p[4].top = 2; p[4].left = 3; p[4].bot = 0; p[4].right = 1;
  p[5].top = 0; p[5].left = 3; p[5].bot = 2; p[5].right = 1;

  for (int level = 0; level < levels - 1; level++) {
    int n = 6 * (1 << (2 * level));
    int ls = level_start(level + 1), ps = level_start(level);
    for (int i = 0; i < n; i++) {
      int start = ls + 4 * i;
      orc_panel* par = &p[ps + i];
      for (int j = 0; j < 4; j++) {
        p[start + j].id = start + j;
        p[start + j].face = par->face;
        p[start + j].parent = ps + i;
        p[start + j].level = par->level + 1;
      }
      double max_xi = par->max_xi, min_xi = par->min_xi, max_eta = par->max_eta, min_eta = par->min_eta;
      double mid_xi = 0.5 * (max_xi + min_xi), mid_eta = 0.5 * (max_eta + min_eta);
      p[start].max_xi = max_xi; p[start].min_xi = mid_xi; p[start].max_eta = max_eta; p[start].min_eta = mid_eta;
      p[start + 1].max_xi = mid_xi; p[start + 1].min_xi = min_xi; p[start + 1].max_eta = max_eta; p[start + 1].min_eta = mid_eta;
      p[start + 2].max_xi = mid_xi; p[start + 2].min_xi = min_xi; p[start + 2].max_eta = mid_eta; p[start + 2].min_eta = min_eta;
      p[start + 3].max_xi = max_xi; p[start + 3].min_xi = mid_xi; p[start + 3].max_eta = mid_eta; p[start + 3].min_eta = min_eta;
      int pt = par->top - ps, pl = par->left - ps, pb = par->bot - ps, pr = par->right - ps;
      p[start].top = ls + 4 * pt + 3; p[start].left = ls + 4 * i + 1; p[start].bot = ls + 4 * i + 3; p[start].right = ls + 4 * pr + 1;
      p[start + 1].top = ls + 4 * pt + 2; p[start + 1].left = ls + 4 * pl; p[start + 1].bot = ls + 4 * i + 2; p[start + 1].right = ls + 4 * i;
      p[start + 2].top = ls + 4 * i + 1; p[start + 2].left = ls + 4 * pl + 3; p[start + 2].bot = ls + 4 * pb + 1; p[start + 2].right = ls + 4 * i + 3;
      p[start + 3].top = ls + 4 * i; p[start + 3].left = ls + 4 * i + 2; p[start + 3].bot = ls + 4 * pb; p[start + 3].right = ls + 4 * pr + 2;
      for (int j = 0; j < 4; j++) par->child[j] = start + j;
    }
  }
  for (int i = 0; i < P; i++) {
    p[i].is_leaf = (p[i].level == levels - 1);
    double max_xi = p[i].max_xi * ORC_PI / 4.0, min_xi = p[i].min_xi * ORC_PI / 4.0;
    double max_eta = p[i].max_eta * ORC_PI / 4.0, min_eta = p[i].min_eta * ORC_PI / 4.0;
    double mid_xi = 0.5 * (max_xi + min_xi), mid_eta = 0.5 * (max_eta + min_eta);
    double p1[3], p2[3], p3[3], p4[3], pc[3];
    xyz_from_xieta(max_xi, max_eta, p[i].face, p1);
    xyz_from_xieta(max_xi, min_eta, p[i].face, p2);
    xyz_from_xieta(min_xi, min_eta, p[i].face, p3);
    xyz_from_xieta(min_xi, max_eta, p[i].face, p4);
    xyz_from_xieta(mid_xi, mid_eta, p[i].face, pc);
    double d1 = gcdist(p1, pc), d2 = gcdist(p2, pc), d3 = gcdist(p3, pc), d4 = gcdist(p4, pc);
    p[i].radius = fmax(d1, fmax(d2, fmax(d3, d4)));
    p[i].area = sphere_tri_area(p1, p2, p3) + sphere_tri_area(p1, p3, p4);
  }
}

/* interp_init: src/interp_funcs.cpp:11-73.  With exact_cc the Clenshaw-Curtis
 * weights are the exact ones (the reference's formula leaves the middle node
 * weight at zero for odd degree and is not exact for even degree). */
void orc_interp_init(int degree, int exact_cc, double* info) {
  int d = degree, n = d + 1;
  double cheb[11], bw[11], cc[11];
  if (d == 0) {
    cheb[0] = 0;
    bw[0] = 1;
  } else {
    for (int i = 0; i < n; i++) {
      cheb[i] = cos(ORC_PI / d * i);
      if (fabs(cheb[i]) < 1e-16) cheb[i] = 0;
      bw[i] = (i == 0) ? 0.5 : (i == d ? 0.5 * pow(-1, i) : pow(-1, i));
    }
  }
  for (int i = 0; i < n; i++) cc[i] = 0;
  if (!exact_cc) {
    double vec[6];
    for (int i = 0; i < d / 2 + 1; i++) vec[i] = 2;
    vec[0] = 1;
    for (int i = 1; i < d / 2 + 1; i++) vec[i] = 2.0 / (1 - 4 * i * i);
    for (int i = 0; i < d / 2 + 1; i++) {
      double sum = 0;
      for (int j = 0; j < d / 2 + 1; j++) sum += 2 * cos(2 * i * j * ORC_PI / d) / d * vec[j];
      cc[i] = sum;
    }
    cc[0] *= 0.5;
    for (int i = 0; i < d / 2; i++) cc[d - i] = cc[i];
  } else if (d == 0) {
    cc[0] = 2;
  } else {
    /* w_i = (c_i/d) [1 - sum_{j=1}^{floor(d/2)} b_j cos(2 j theta_i) / (4 j^2 - 1)],
     * c_i = 1 at the end nodes else 2, b_j = 1 for j = d/2 else 2. */
    for (int i = 0; i < n; i++) {
      double th = ORC_PI * i / d, s = 1.0;
      for (int j = 1; j <= d / 2; j++) {
        double b = (2 * j == d) ? 1.0 : 2.0;
        s -= b * cos(2 * j * th) / (4.0 * j * j - 1);
      }
      cc[i] = ((i == 0 || i == d) ? 1.0 : 2.0) / d * s;
    }
  }
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) {
      int idx = i * n + j;
      info[4 * idx + 0] = cheb[i];
      info[4 * idx + 1] = cheb[j];
      info[4 * idx + 2] = bw[i] * bw[j];
      info[4 * idx + 3] = cc[i] * cc[j];
    }
}

/* cube_sphere_spec_points / compute_point_panel: src/initialize_cubed_sphere.cpp:236-288 */
void orc_spec_points(int levels, int degree, const orc_panel* p, const double* interp, double* x, double* y,
                     double* z, double* area) {
  int q = (degree + 1) * (degree + 1);
  int off = level_start(levels - 1), P = orc_panel_count(levels);
  for (int i = off; i < P; i++) {
    double max_xi = ORC_PI / 4.0 * p[i].max_xi, min_xi = ORC_PI / 4.0 * p[i].min_xi;
    double max_eta = ORC_PI / 4.0 * p[i].max_eta, min_eta = ORC_PI / 4.0 * p[i].min_eta;
    double xi_range = 0.5 * (max_xi - min_xi), xi_offset = 0.5 * (max_xi + min_xi);
    double eta_range = 0.5 * (max_eta - min_eta), eta_offset = 0.5 * (max_eta + min_eta);
    for (int j = 0; j < q; j++) {
      double xyz[3];
      xyz_from_xieta(xi_offset + xi_range * interp[4 * j], eta_offset + eta_range * interp[4 * j + 1], p[i].face,
                     xyz);
      size_t o = (size_t)(i - off) * q + j;
      x[o] = xyz[0];
      y[o] = xyz[1];
      z[o] = xyz[2];
      area[o] = interp[4 * j + 3] * p[i].area / 4.0;
    }
  }
}

/* dual_tree_traversal: src/fmm_funcs.cpp:17-123 (FIFO queue of panel pairs). */
long orc_dual_tree_traversal(int levels, const orc_panel* p, double theta, int* list, long cap) {
  long qcap = 1 << 16, head = 0, tail = 0, count = 0;
  int* qt = (int*)malloc(sizeof(int) * qcap);
  int* qs = (int*)malloc(sizeof(int) * qcap);
#define PUSH(t, s)                                                 \
  do {                                                             \
    if (tail == qcap) {                                            \
      long live = tail - head;                                     \
      memmove(qt, qt + head, sizeof(int) * live);                  \
      memmove(qs, qs + head, sizeof(int) * live);                  \
      head = 0;                                                    \
      tail = live;                                                 \
      if (tail + 8 > qcap) {                                       \
        qcap *= 2;                                                 \
        qt = (int*)realloc(qt, sizeof(int) * qcap);                \
        qs = (int*)realloc(qs, sizeof(int) * qcap);                \
      }                                                            \
    }                                                              \
    qt[tail] = (t);                                                \
    qs[tail] = (s);                                                \
    tail++;                                                        \
  } while (0)
#define EMIT(t, s, ty)              \
  do {                              \
    if (count < cap) {              \
      list[3 * count] = (t);        \
      list[3 * count + 1] = (s);    \
      list[3 * count + 2] = (ty);   \
    }                               \
    count++;                        \
  } while (0)
  for (int i = 0; i < 6; i++)
    for (int j = 0; j < 6; j++) PUSH(i, j);
  while (tail > head) {
    int t = qt[head], s = qs[head];
    head++;
    double xi1 = ORC_PI / 4.0 * 0.5 * (p[t].min_xi + p[t].max_xi);
    double xi2 = ORC_PI / 4.0 * 0.5 * (p[s].min_xi + p[s].max_xi);
    double eta1 = ORC_PI / 4.0 * 0.5 * (p[t].min_eta + p[t].max_eta);
    double eta2 = ORC_PI / 4.0 * 0.5 * (p[s].min_eta + p[s].max_eta);
    double c1[3], c2[3];
    xyz_from_xieta(xi1, eta1, p[t].face, c1);
    xyz_from_xieta(xi2, eta2, p[s].face, c2);
    double dist = gcdist(c1, c2), sep = 100;
    if (dist > 1e-16) sep = (p[t].radius + p[s].radius) / dist;
    if (sep < theta) {
      int ty = 0;
      if (p[t].level < levels - 1) ty += 2;
      if (p[s].level < levels - 1) ty += 1;
      EMIT(t, s, ty);
    } else if (p[t].is_leaf && p[s].is_leaf) {
      EMIT(t, s, 0);
    } else if (p[t].is_leaf) {
      for (int c = 0; c < 4; c++) PUSH(t, p[s].child[c]);
    } else if (p[s].is_leaf) {
      for (int c = 0; c < 4; c++) PUSH(p[t].child[c], s);
    } else if (p[t].level <= p[s].level) {
      for (int c = 0; c < 4; c++) PUSH(p[t].child[c], s);
    } else {
      for (int c = 0; c < 4; c++) PUSH(t, p[s].child[c]);
    }
  }
#undef PUSH
#undef EMIT
  free(qt);
  free(qs);
  return count;
}

/* ---------------- interpolation: src/interp_funcs_impl.hpp ---------------- */

/* interp_vals_bli: src/interp_funcs_impl.hpp:11-112.  Out-of-panel input sets
 * the oracle error flag (the reference aborts). */
static void bli_core(double* basis, double xi, double eta, double min_xi, double max_xi, double min_eta,
                     double max_eta, int d, int check) {
  double xi_range = 0.5 * (max_xi - min_xi), xi_offset = 0.5 * (max_xi + min_xi);
  double eta_range = 0.5 * (max_eta - min_eta), eta_offset = 0.5 * (max_eta + min_eta);
  double cheb_xi[11], cheb_eta[11], w[11], fx[11], fe[11], val;
  if (check && (xi < min_xi - 1e-15 || xi > max_xi + 1e-15 || eta < min_eta - 1e-15 || eta > max_eta + 1e-15))
    g_orc_error = 1;
  for (int i = 0; i < (d + 1) * (d + 1); i++) basis[i] = 0.0;
  if (d == 0) {
    cheb_xi[0] = xi_offset;
    cheb_eta[0] = eta_offset;
    w[0] = 1;
  } else {
    for (int i = 0; i < d + 1; i++) {
      cheb_xi[i] = cos(ORC_PI * i / d) * xi_range + xi_offset;
      cheb_eta[i] = cos(ORC_PI * i / d) * eta_range + eta_offset;
      w[i] = (i == 0) ? 0.5 : (i == d ? 0.5 * pow(-1, i) : pow(-1, i));
    }
  }
  int found = 0;
  for (int i = 0; i < d + 1; i++) {
    if (fabs(xi - cheb_xi[i]) < 1e-15) {
      found = 1;
      for (int j = 0; j < d + 1; j++) fx[j] = 0;
      fx[i] = 1;
      break;
    }
  }
  if (!found) {
    double den = 0;
    for (int i = 0; i < d + 1; i++) {
      val = w[i] / (xi - cheb_xi[i]);
      fx[i] = val;
      den += val;
    }
    for (int i = 0; i < d + 1; i++) fx[i] /= den;
  }
  found = 0;
  for (int i = 0; i < d + 1; i++) {
    if (fabs(eta - cheb_eta[i]) < 1e-15) {
      found = 1;
      for (int j = 0; j < d + 1; j++) fe[j] = 0;
      fe[i] = 1;
      break;
    }
  }
  if (!found) {
    double den = 0;
    for (int i = 0; i < d + 1; i++) {
      val = w[i] / (eta - cheb_eta[i]);
      fe[i] = val;
      den += val;
    }
    for (int i = 0; i < d + 1; i++) fe[i] /= den;
  }
  for (int i = 0; i < d + 1; i++)
    for (int j = 0; j < d + 1; j++) basis[i * (d + 1) + j] = fx[i] * fe[j];
}

void orc_interp_vals_bli(double* basis, double xi, double eta, double min_xi, double max_xi, double min_eta,
                         double max_eta, int d) {
  bli_core(basis, xi, eta, min_xi, max_xi, min_eta, max_eta, d, 1);
}

/* point_locate_panel: src/interp_funcs_impl.hpp:114-142 */
int orc_point_locate_panel(const orc_panel* p, double x, double y, double z) {
  int cur = face_from_xyz(x, y, z);
  double xe[2];
  xieta_from_xyz_face(x, y, z, cur, xe);
  double xi = xe[0], eta = xe[1];
  while (!p[cur].is_leaf) {
    double mid_xi = 0.5 * ORC_PI / 4.0 * (p[cur].max_xi + p[cur].min_xi);
    double mid_eta = 0.5 * ORC_PI / 4.0 * (p[cur].max_eta + p[cur].min_eta);
    if ((xi >= mid_xi) && (eta >= mid_eta)) cur = p[cur].child[0];
    else if ((xi <= mid_xi) && (eta >= mid_eta)) cur = p[cur].child[1];
    else if ((xi <= mid_xi) && (eta <= mid_eta)) cur = p[cur].child[2];
    else if ((xi >= mid_xi) && (eta <= mid_eta)) cur = p[cur].child[3];
    else {
      g_orc_error = 2; /* NaN coordinates */
      return cur;
    }
  }
  return cur;
}

/* BLI of one point at the located leaf with bounds pi/4.0 * (panel bounds):
 * the call pattern of src/bve_time_step.cpp:45-46, 143-144, 222-223. */
static void bli_at_leaf(const orc_panel* p, int leaf, double xi, double eta, int d, double* basis) {
  orc_interp_vals_bli(basis, xi, eta, ORC_PI / 4.0 * p[leaf].min_xi, ORC_PI / 4.0 * p[leaf].max_xi,
                      ORC_PI / 4.0 * p[leaf].min_eta, ORC_PI / 4.0 * p[leaf].max_eta, d);
}

/* ---------------- FMM passes: src/fmm_funcs.cpp, src/fmm_funcs_impl.hpp --- */

/* upward_pass + base_pots + child_to_parent: src/fmm_funcs.cpp:341-355,
 * src/fmm_funcs_impl.hpp:17-71.  Parents accumulate children in ascending
 * child index, then child point i, as the reference's sequential atomics do. */
void orc_upward_pass(int levels, int degree, const orc_panel* p, const double* interp, const double* area,
                     const double* pots, double* proxy) {
  int q = (degree + 1) * (degree + 1), P = orc_panel_count(levels), A = orc_leaf_count(levels);
  int off = P - A;
  memset(proxy, 0, sizeof(double) * (size_t)P * q);
  for (size_t i = 0; i < (size_t)A * q; i++) proxy[(size_t)off * q + i] = area[i] * pots[i];
  for (int lev = levels - 1; lev >= 1; lev--) {
    int plo = level_start(lev - 1), phi = level_start(lev);
#pragma omp parallel for schedule(static)
    for (int par = plo; par < phi; par++) {
      double min_xi = p[par].min_xi * ORC_PI / 4.0, max_xi = p[par].max_xi * ORC_PI / 4.0;
      double min_eta = p[par].min_eta * ORC_PI / 4.0, max_eta = p[par].max_eta * ORC_PI / 4.0;
      double vals[MAXQ];
      for (int c = 0; c < 4; c++) {
        int k = p[par].child[c];
        double xi_off = ORC_PI / 4.0 * 0.5 * (p[k].min_xi + p[k].max_xi);
        double xi_scale = ORC_PI / 4.0 * 0.5 * (p[k].max_xi - p[k].min_xi);
        double eta_off = ORC_PI / 4.0 * 0.5 * (p[k].min_eta + p[k].max_eta);
        double eta_scale = ORC_PI / 4.0 * 0.5 * (p[k].max_eta - p[k].min_eta);
        for (int i = 0; i < q; i++) {
          double xi = interp[4 * i] * xi_scale + xi_off, eta = interp[4 * i + 1] * eta_scale + eta_off;
          orc_interp_vals_bli(vals, xi, eta, min_xi, max_xi, min_eta, max_eta, degree);
          for (int j = 0; j < q; j++) proxy[(size_t)par * q + j] += vals[j] * proxy[(size_t)k * q + i];
        }
      }
    }
  }
}

/* downward_pass_3 + parent_to_child_3 + child_panel_copy:
 * src/fmm_funcs.cpp:374-392, src/fmm_funcs_impl.hpp:123-188 */
void orc_downward_pass_3(int levels, int degree, const orc_panel* p, const double* interp, double* t1, double* t2,
                         double* t3, double* s1, double* s2, double* s3) {
  int q = (degree + 1) * (degree + 1), P = orc_panel_count(levels), A = orc_leaf_count(levels);
  for (int lev = 0; lev < levels - 1; lev++) {
    int plo = level_start(lev), phi = level_start(lev + 1);
#pragma omp parallel for schedule(static)
    for (int i = plo; i < phi; i++) {
      double min_xi = p[i].min_xi * ORC_PI / 4.0, max_xi = p[i].max_xi * ORC_PI / 4.0;
      double min_eta = p[i].min_eta * ORC_PI / 4.0, max_eta = p[i].max_eta * ORC_PI / 4.0;
      double vals[MAXQ];
      for (int c = 0; c < 4; c++) {
        int ch = p[i].child[c];
        double xi_off = ORC_PI / 4.0 * 0.5 * (p[ch].min_xi + p[ch].max_xi);
        double xi_scale = ORC_PI / 4.0 * 0.5 * (p[ch].max_xi - p[ch].min_xi);
        double eta_off = ORC_PI / 4.0 * 0.5 * (p[ch].min_eta + p[ch].max_eta);
        double eta_scale = ORC_PI / 4.0 * 0.5 * (p[ch].max_eta - p[ch].min_eta);
        for (int k = 0; k < q; k++) {
          double xi = interp[4 * k] * xi_scale + xi_off, eta = interp[4 * k + 1] * eta_scale + eta_off;
          orc_interp_vals_bli(vals, xi, eta, min_xi, max_xi, min_eta, max_eta, degree);
          for (int l = 0; l < q; l++) {
            t1[(size_t)ch * q + k] += vals[l] * t1[(size_t)i * q + l];
            t2[(size_t)ch * q + k] += vals[l] * t2[(size_t)i * q + l];
            t3[(size_t)ch * q + k] += vals[l] * t3[(size_t)i * q + l];
          }
        }
      }
    }
  }
  size_t off = (size_t)(P - A) * q;
  for (size_t i = 0; i < (size_t)A * q; i++) {
    s1[i] = t1[off + i];
    s2[i] = t2[off + i];
    s3[i] = t3[off + i];
  }
}

/* Proxy point j of panel pn as the interaction kernel computes it:
 * src/fmm_interactions/bve_vel_impl.hpp:90-108. */
static void proxy_point(const orc_panel* p, int pn, const double* interp, int j, double* xyz) {
  double xi_off = ORC_PI / 4 * 0.5 * (p[pn].max_xi + p[pn].min_xi);
  double xi_scale = ORC_PI / 4 * 0.5 * (p[pn].max_xi - p[pn].min_xi);
  double eta_off = ORC_PI / 4 * 0.5 * (p[pn].max_eta + p[pn].min_eta);
  double eta_scale = ORC_PI / 4 * 0.5 * (p[pn].max_eta - p[pn].min_eta);
  xyz_from_xieta(interp[4 * j] * xi_scale + xi_off, interp[4 * j + 1] * eta_scale + eta_off, p[pn].face, xyz);
}

/* One panel-pair block of bve_vel_panel_interaction:
 * src/fmm_interactions/bve_vel_impl.hpp:85-122.  Sums for each target point
 * run over source points k in order. */
static void bve_pair_block(const orc_panel* p, const double* interp, int q, int t, int s, const double* dx,
                           const double* dy, const double* dz, const double* src, double eps, double* t1,
                           double* t2, double* t3) {
  double xs[MAXQ], ys[MAXQ], zs[MAXQ];
  for (int k = 0; k < q; k++) {
    double xyz_s[3];
    proxy_point(p, s, interp, k, xyz_s);
    double x_s = xyz_s[0] + dx[(size_t)s * q + k], y_s = xyz_s[1] + dy[(size_t)s * q + k],
           z_s = xyz_s[2] + dz[(size_t)s * q + k];
    project_to_sphere(&x_s, &y_s, &z_s);
    xs[k] = x_s;
    ys[k] = y_s;
    zs[k] = z_s;
  }
  for (int j = 0; j < q; j++) {
    double xt[3];
    proxy_point(p, t, interp, j, xt);
    double a1 = t1[(size_t)t * q + j], a2 = t2[(size_t)t * q + j], a3 = t3[(size_t)t * q + j];
    for (int k = 0; k < q; k++) {
      double dp = xt[0] * xs[k] + xt[1] * ys[k] + xt[2] * zs[k];
      double g = -0.07957747154594767 / (1.0 - dp + eps) * src[(size_t)s * q + k];
      a1 += g * (xt[1] * zs[k] - xt[2] * ys[k]);
      a2 += g * (xt[2] * xs[k] - xt[0] * zs[k]);
      a3 += g * (xt[0] * ys[k] - xt[1] * xs[k]);
    }
    t1[(size_t)t * q + j] = a1;
    t2[(size_t)t * q + j] = a2;
    t3[(size_t)t * q + j] = a3;
  }
}

/* bve_vel_interactions: src/fmm_interactions/bve_vel.cpp:9-37 with one rank.
 * Entries are grouped by target panel (stable, so each target still sees its
 * sources in list order) and target panels run in parallel. */
void orc_bve_vel_interactions(int levels, int degree, const orc_panel* p, const double* interp, long n_list,
                              const int* list, const double* disp_x, const double* disp_y, const double* disp_z,
                              const double* source, double eps, double* t1, double* t2, double* t3) {
  int q = (degree + 1) * (degree + 1), P = orc_panel_count(levels);
  long* start = (long*)calloc((size_t)P + 1, sizeof(long));
  long* order = (long*)malloc(sizeof(long) * (size_t)(n_list > 0 ? n_list : 1));
  for (long i = 0; i < n_list; i++) start[list[3 * i] + 1]++;
  for (int i = 0; i < P; i++) start[i + 1] += start[i];
  long* fill = (long*)malloc(sizeof(long) * (size_t)P);
  for (int i = 0; i < P; i++) fill[i] = start[i];
  for (long i = 0; i < n_list; i++) order[fill[list[3 * i]]++] = i;
#pragma omp parallel for schedule(dynamic, 16)
  for (int t = 0; t < P; t++)
    for (long e = start[t]; e < start[t + 1]; e++)
      bve_pair_block(p, interp, q, t, list[3 * order[e] + 1], disp_x, disp_y, disp_z, source, eps, t1, t2, t3);
  free(start);
  free(order);
  free(fill);
}

void orc_bve_direct_velocity(int levels, int degree, const orc_panel* p, const double* interp, const double* disp_x,
                             const double* disp_y, const double* disp_z, const double* source, double eps,
                             double* t1, double* t2, double* t3) {
  int q = (degree + 1) * (degree + 1), P = orc_panel_count(levels), A = orc_leaf_count(levels);
  int off = P - A;
#pragma omp parallel for schedule(dynamic, 4)
  for (int t = off; t < P; t++)
    for (int s = off; s < P; s++) bve_pair_block(p, interp, q, t, s, disp_x, disp_y, disp_z, source, eps, t1, t2, t3);
}

/* ---------------- treecode with decoupled proxy degree (Mode C) ----------
 *
 * The reference's irregular-point FMM (the "_ll" functions) applied to the
 * particle grid: a cubed-sphere quadtree of tree_levels levels whose leaves
 * hold npl particles each (the particles of the leaf's descendant grid panels,
 * which are consecutive in the [leaf panel][q] arrays), (n+1)^2 Chebyshev
 * proxies of degree n on every tree panel at fixed positions, and bounds in
 * radians as in initialize_cube_sphere_irreg_points
 * (src/initialize_cubed_sphere.cpp:446-592).
 *
 *   upward     base_pots_ll + child_to_parent_ll (src/fmm_funcs_impl.hpp:190-268,
 *              src/fmm_funcs.cpp:394-405)
 *   list       dual_tree_traversal_irreg (src/fmm_funcs.cpp:125-231): the
 *              FIFO traversal of orc_dual_tree_traversal on the tree panels
 *   pairs      swe_vel_panel_interaction_ll (src/fmm_interactions/swe_vel_impl.hpp:180-287),
 *              rotational part (zero divergence), typed pp / pc / cp / cc
 *   downward   parent_to_child_3_ll + child_panel_interp_3_ll
 *              (src/fmm_funcs_impl.hpp:270-364, src/fmm_funcs.cpp:407-419)
 *
 * typed = 1 follows the reference's typing: a well-separated pair uses the
 * particles of a side whose panel is at the deepest tree level and the
 * proxies otherwise (pp, pc, cp, cc).  typed = 0 evaluates every
 * well-separated pair proxy x proxy (the design of this library's treecode).
 * Pairs that fail the MAC are leaf pairs, particle x particle, in both.
 * Sources may be displaced (positions off the grid): they are anterpolated in
 * the coordinates of their own leaf's face with the barycentric formula
 * extended past the leaf, where the reference would stop (Kokkos::abort,
 * src/interp_funcs_impl.hpp:22-33); for particles on the grid the two agree. */

typedef struct {
  int L, d, q, n, n1, qx, npl, Lf, Pf, Af, offf;
  orc_panel* tp;
  double* px; /* [Pf][qx][3] proxy positions */
} bltc_tree;

/* tree levels: panels are split while they hold more than leaf_size
 * particles (src/initialize_cubed_sphere.cpp:473-474) */
static void bltc_tree_init(int levels, int degree, int leaf_size, int n, bltc_tree* t) {
  t->L = levels;
  t->d = degree;
  t->q = (degree + 1) * (degree + 1);
  t->n = n;
  t->n1 = n + 1;
  t->qx = t->n1 * t->n1;
  int m = 0;
  long npl = t->q;
  while (npl * 4 <= leaf_size && m < levels - 1) {
    npl *= 4;
    m++;
  }
  t->npl = (int)npl;
  t->Lf = levels - m;
  t->Pf = orc_panel_count(t->Lf);
  t->Af = orc_leaf_count(t->Lf);
  t->offf = t->Pf - t->Af;
  t->tp = (orc_panel*)malloc(sizeof(orc_panel) * (size_t)t->Pf);
  orc_panels_init(t->Lf, t->tp);
  t->px = (double*)malloc(sizeof(double) * 3 * (size_t)t->Pf * t->qx);
  for (int p = 0; p < t->Pf; p++) {
    /* proxy (j, k): xi = cos(pi j/n) xi_scale + xi_off (swe_vel_impl.hpp:227-240) */
    double mn = ORC_PI / 4.0 * t->tp[p].min_xi, mx = ORC_PI / 4.0 * t->tp[p].max_xi;
    double me = ORC_PI / 4.0 * t->tp[p].min_eta, xe = ORC_PI / 4.0 * t->tp[p].max_eta;
    double xi_off = 0.5 * (mn + mx), xi_scale = 0.5 * (mx - mn), eta_off = 0.5 * (me + xe),
           eta_scale = 0.5 * (xe - me);
    for (int j = 0; j < t->n1; j++)
      for (int k = 0; k < t->n1; k++) {
        double xi = cos(ORC_PI * j / n) * xi_scale + xi_off, eta = cos(ORC_PI * k / n) * eta_scale + eta_off;
        xyz_from_xieta(xi, eta, t->tp[p].face, t->px + 3 * ((size_t)p * t->qx + j * t->n1 + k));
      }
  }
}

static void bltc_tree_free(bltc_tree* t) {
  free(t->tp);
  free(t->px);
}

static void panel_rad(const orc_panel* p, double* b) {
  b[0] = ORC_PI / 4.0 * p->min_xi;
  b[1] = ORC_PI / 4.0 * p->max_xi;
  b[2] = ORC_PI / 4.0 * p->min_eta;
  b[3] = ORC_PI / 4.0 * p->max_eta;
}

/* interp_vals_bli (src/interp_funcs_impl.hpp:11-112) without its range check
 * when check == 0. */
static void bli2(double* basis, double xi, double eta, const double* b, int d, int check) {
  bli_core(basis, xi, eta, b[0], b[1], b[2], b[3], d, check);
}

void orc_bltc_shape(int levels, int degree, int leaf_size, int* tree_levels, int* npl) {
  int m = 0;
  long n = (degree + 1) * (degree + 1);
  while (n * 4 <= leaf_size && m < levels - 1) {
    n *= 4;
    m++;
  }
  *tree_levels = levels - m;
  *npl = (int)n;
}

/* base_pots_ll (src/fmm_funcs_impl.hpp:190-222) at the sources' positions
 * (leaf face, extended basis), then child_to_parent_ll level by level
 * (src/fmm_funcs_impl.hpp:224-268; src/fmm_funcs.cpp:394-405): each parent
 * adds its children in id order, child nodes (j, k) in order. */
static void bltc_upward(const bltc_tree* t, const double* sx, const double* sy, const double* sz, const double* w,
                        double* S) {
  int qx = t->qx, n = t->n;
  memset(S, 0, sizeof(double) * (size_t)t->Pf * qx);
#pragma omp parallel for schedule(static)
  for (int f = 0; f < t->Af; f++) {
    int pn = t->offf + f;
    double b[4], bas[MAXQ], xe[2];
    panel_rad(&t->tp[pn], b);
    for (int k = 0; k < t->npl; k++) {
      size_t i = (size_t)f * t->npl + k;
      xieta_from_xyz_face(sx[i], sy[i], sz[i], t->tp[pn].face, xe);
      bli2(bas, xe[0], xe[1], b, n, 0);
      for (int m = 0; m < qx; m++) S[(size_t)pn * qx + m] += bas[m] * w[i];
    }
  }
  for (int lev = t->Lf - 1; lev >= 1; lev--) {
    int plo = level_start(lev - 1), phi = level_start(lev);
#pragma omp parallel for schedule(static)
    for (int par = plo; par < phi; par++) {
      double bp[4], bc[4], bas[MAXQ];
      panel_rad(&t->tp[par], bp);
      for (int c = 0; c < 4; c++) {
        int ch = t->tp[par].child[c];
        panel_rad(&t->tp[ch], bc);
        double xi_off = 0.5 * (bc[0] + bc[1]), xi_scale = 0.5 * (bc[1] - bc[0]);
        double eta_off = 0.5 * (bc[2] + bc[3]), eta_scale = 0.5 * (bc[3] - bc[2]);
        for (int j = 0; j < t->n1; j++)
          for (int k = 0; k < t->n1; k++) {
            double xi = cos(ORC_PI / n * j) * xi_scale + xi_off, eta = cos(ORC_PI / n * k) * eta_scale + eta_off;
            bli2(bas, xi, eta, bp, n, 1);
            double v = S[(size_t)ch * qx + j * t->n1 + k];
            for (int m = 0; m < qx; m++) S[(size_t)par * qx + m] += bas[m] * v;
          }
      }
    }
  }
}

/* parent_to_child_3_ll level by level, then child_panel_interp_3_ll at the
 * targets (src/fmm_funcs_impl.hpp:270-364): T (3 x Pf x qx) in place, u
 * (3 x N) accumulated term by term. */
static void bltc_downward(const bltc_tree* t, const double* tx, const double* ty, const double* tz, double* T,
                          double* u) {
  int qx = t->qx, n = t->n;
  size_t pn = (size_t)t->Pf * qx, N = (size_t)t->Af * t->npl;
  for (int lev = 0; lev < t->Lf - 1; lev++) {
    int plo = level_start(lev), phi = level_start(lev + 1);
#pragma omp parallel for schedule(static)
    for (int par = plo; par < phi; par++) {
      double bp[4], bc[4], bas[MAXQ];
      panel_rad(&t->tp[par], bp);
      for (int c = 0; c < 4; c++) {
        int ch = t->tp[par].child[c];
        panel_rad(&t->tp[ch], bc);
        double xi_off = 0.5 * (bc[0] + bc[1]), xi_scale = 0.5 * (bc[1] - bc[0]);
        double eta_off = 0.5 * (bc[2] + bc[3]), eta_scale = 0.5 * (bc[3] - bc[2]);
        for (int k = 0; k < qx; k++) {
          int k1 = k / t->n1, k2 = k % t->n1;
          double xi = cos(ORC_PI / n * k1) * xi_scale + xi_off, eta = cos(ORC_PI / n * k2) * eta_scale + eta_off;
          bli2(bas, xi, eta, bp, n, 1);
          for (int f = 0; f < 3; f++) {
            double a = T[f * pn + (size_t)ch * qx + k];
            for (int l = 0; l < qx; l++) a += bas[l] * T[f * pn + (size_t)par * qx + l];
            T[f * pn + (size_t)ch * qx + k] = a;
          }
        }
      }
    }
  }
#pragma omp parallel for schedule(static)
  for (int f = 0; f < t->Af; f++) {
    int pnl = t->offf + f;
    double b[4], bas[MAXQ], xe[2];
    panel_rad(&t->tp[pnl], b);
    for (int j = 0; j < t->npl; j++) {
      size_t i = (size_t)f * t->npl + j;
      xieta_from_xyz_face(tx[i], ty[i], tz[i], t->tp[pnl].face, xe);
      bli2(bas, xe[0], xe[1], b, n, 1);
      for (int c = 0; c < 3; c++) {
        double a = u[c * N + i];
        for (int k = 0; k < qx; k++) a += bas[k] * T[c * pn + (size_t)pnl * qx + k];
        u[c * N + i] = a;
      }
    }
  }
}

/* The MAC of dual_tree_traversal_irreg (src/fmm_funcs.cpp:149-162), with the
 * same arithmetic as orc_dual_tree_traversal. */
static int bltc_well_separated(const orc_panel* p, int t, int s, double theta) {
  double xi1 = ORC_PI / 4.0 * 0.5 * (p[t].min_xi + p[t].max_xi);
  double xi2 = ORC_PI / 4.0 * 0.5 * (p[s].min_xi + p[s].max_xi);
  double eta1 = ORC_PI / 4.0 * 0.5 * (p[t].min_eta + p[t].max_eta);
  double eta2 = ORC_PI / 4.0 * 0.5 * (p[s].min_eta + p[s].max_eta);
  double c1[3], c2[3];
  xyz_from_xieta(xi1, eta1, p[t].face, c1);
  xyz_from_xieta(xi2, eta2, p[s].face, c2);
  double dist = gcdist(c1, c2), sep = 100;
  if (dist > 1e-16) sep = (p[t].radius + p[s].radius) / dist;
  return sep < theta;
}

/* One list entry of swe_vel_panel_interaction_ll
 * (src/fmm_interactions/swe_vel_impl.hpp:256-284): targets j in order, sources
 * k in order; out receives 3 strided sums per target.  Rotational part with
 * sources s (strengths sv); with sd, the divergent part with sources s2
 * (strengths sd).  The reference's sources of both fields coincide; here the
 * vorticity sources may be displaced while the divergence sources stay on the
 * grid (swe_vel_panel_interaction_2, src/fmm_interactions/swe_vel_impl.hpp:124-141),
 * and where they coincide the arithmetic is the reference's. */
typedef struct {
  const double* xyz;                 /* interleaved positions, or NULL */
  const double *x, *y, *z, *w;       /* positions (when xyz is NULL) and strengths */
} bltc_src;

static void bltc_block(int nt, const double* txyz, size_t tstride, const double* tx, const double* ty,
                       const double* tz, int ns, bltc_src s1, const bltc_src* s2, double eps, double* o1, double* o2,
                       double* o3) {
  for (int j = 0; j < nt; j++) {
    double x_t = txyz ? txyz[3 * j] : tx[j], y_t = txyz ? txyz[3 * j + 1] : ty[j], z_t = txyz ? txyz[3 * j + 2] : tz[j];
    double a1 = o1[j * tstride], a2 = o2[j * tstride], a3 = o3[j * tstride];
    for (int k = 0; k < ns; k++) {
      double x_s = s1.xyz ? s1.xyz[3 * k] : s1.x[k], y_s = s1.xyz ? s1.xyz[3 * k + 1] : s1.y[k],
             z_s = s1.xyz ? s1.xyz[3 * k + 2] : s1.z[k];
      double dp = x_t * x_s + y_t * y_s + z_t * z_s;
      double gf = 0.07957747154594767 / (1.0 - dp + eps);
      double gf1 = -gf * s1.w[k];
      if (s2) {
        double x2 = s2->xyz ? s2->xyz[3 * k] : s2->x[k], y2 = s2->xyz ? s2->xyz[3 * k + 1] : s2->y[k],
               z2 = s2->xyz ? s2->xyz[3 * k + 2] : s2->z[k];
        double dp2 = x_t * x2 + y_t * y2 + z_t * z2;
        double gf2 = 0.07957747154594767 / (1.0 - dp2 + eps) * s2->w[k];
        a1 += gf1 * (y_t * z_s - z_t * y_s) + gf2 * (x2 - x_t * dp2);
        a2 += gf1 * (z_t * x_s - x_t * z_s) + gf2 * (y2 - y_t * dp2);
        a3 += gf1 * (x_t * y_s - y_t * x_s) + gf2 * (z2 - z_t * dp2);
      } else {
        a1 += gf1 * (y_t * z_s - z_t * y_s);
        a2 += gf1 * (z_t * x_s - x_t * z_s);
        a3 += gf1 * (x_t * y_s - y_t * x_s);
      }
    }
    o1[j * tstride] = a1;
    o2[j * tstride] = a2;
    o3[j * tstride] = a3;
  }
}

/* The interaction list on the tree: entries grouped by target panel (stable,
 * so each target sees its sources in list order), target panels in parallel.
 * u (3 x N) receives particle-target sums, T (3 x Pf x qx) proxy-target sums.
 * Particle sources p1 (rotational) and, for the SWE, p2 (divergent), proxy
 * strengths S and S2 at the fixed proxies. */
static void bltc_interactions(const bltc_tree* t, long nl, const int* list, double theta, int typed,
                              const double* tx, const double* ty, const double* tz, bltc_src p1, const double* S,
                              const bltc_src* p2, const double* S2, double eps, double* u, double* T) {
  int Pf = t->Pf, qx = t->qx, npl = t->npl;
  size_t pn = (size_t)Pf * qx, N = (size_t)t->Af * npl;
  long* start = (long*)calloc((size_t)Pf + 1, sizeof(long));
  long* order = (long*)malloc(sizeof(long) * (size_t)(nl > 0 ? nl : 1));
  long* fill = (long*)malloc(sizeof(long) * (size_t)Pf);
  for (long i = 0; i < nl; i++) start[list[3 * i] + 1]++;
  for (int i = 0; i < Pf; i++) start[i + 1] += start[i];
  for (int i = 0; i < Pf; i++) fill[i] = start[i];
  for (long i = 0; i < nl; i++) order[fill[list[3 * i]]++] = i;
  const int deepest = t->Lf - 1;
#pragma omp parallel for schedule(dynamic, 4)
  for (int tp = 0; tp < Pf; tp++) {
    for (long e = start[tp]; e < start[tp + 1]; e++) {
      int s = list[3 * order[e] + 1];
      int near = !bltc_well_separated(t->tp, tp, s, theta);
      int tpart = near || (typed && t->tp[tp].level == deepest);
      int spart = near || (typed && t->tp[s].level == deepest);
      size_t t0 = (size_t)(tp - t->offf) * npl, s0 = (size_t)(s - t->offf) * npl;
      double* o = tpart ? u + t0 : T + (size_t)tp * qx;
      size_t stride = tpart ? N : pn;
      const double* txyz = tpart ? NULL : t->px + 3 * (size_t)tp * qx;
      int nt = tpart ? npl : qx;
      if (spart) {
        bltc_src a = {NULL, p1.x + s0, p1.y + s0, p1.z + s0, p1.w + s0}, b;
        if (p2) b = (bltc_src){NULL, p2->x + s0, p2->y + s0, p2->z + s0, p2->w + s0};
        bltc_block(nt, txyz, 1, tx + t0, ty + t0, tz + t0, npl, a, p2 ? &b : NULL, eps, o, o + stride,
                   o + 2 * stride);
      } else {
        const double* sxyz = t->px + 3 * (size_t)s * qx;
        bltc_src a = {sxyz, NULL, NULL, NULL, S + (size_t)s * qx}, b = {sxyz, NULL, NULL, NULL, NULL};
        if (p2) b.w = S2 + (size_t)s * qx;
        bltc_block(nt, txyz, 1, tx + t0, ty + t0, tz + t0, qx, a, p2 ? &b : NULL, eps, o, o + stride,
                   o + 2 * stride);
      }
    }
  }
  free(start);
  free(order);
  free(fill);
}

long orc_bltc_list(int levels, int degree, int leaf_size, int n, double theta, int* list, long cap) {
  bltc_tree t;
  bltc_tree_init(levels, degree, leaf_size, n, &t);
  long nl = orc_dual_tree_traversal(t.Lf, t.tp, theta, list, cap);
  bltc_tree_free(&t);
  return nl;
}

void orc_bltc_upward(int levels, int degree, int leaf_size, int n, const double* sx, const double* sy,
                     const double* sz, const double* w, double* proxy) {
  bltc_tree t;
  bltc_tree_init(levels, degree, leaf_size, n, &t);
  bltc_upward(&t, sx, sy, sz, w, proxy);
  bltc_tree_free(&t);
}

void orc_bltc_downward(int levels, int degree, int leaf_size, int n, double* T, const double* tx, const double* ty,
                       const double* tz, double* u) {
  bltc_tree t;
  bltc_tree_init(levels, degree, leaf_size, n, &t);
  bltc_downward(&t, tx, ty, tz, T, u);
  bltc_tree_free(&t);
}

void orc_bltc_velocity(int levels, int degree, int leaf_size, int n, double theta, double eps, int typed,
                       const double* tx, const double* ty, const double* tz, const double* sx, const double* sy,
                       const double* sz, const double* w, double* u) {
  bltc_tree t;
  bltc_tree_init(levels, degree, leaf_size, n, &t);
  size_t pn = (size_t)t.Pf * t.qx, N = (size_t)t.Af * t.npl;
  long nl = orc_dual_tree_traversal(t.Lf, t.tp, theta, NULL, 0);
  int* list = (int*)malloc(sizeof(int) * 3 * (size_t)(nl > 0 ? nl : 1));
  orc_dual_tree_traversal(t.Lf, t.tp, theta, list, nl);
  double* S = (double*)calloc(pn, sizeof(double));
  double* T = (double*)calloc(3 * pn, sizeof(double));
  memset(u, 0, sizeof(double) * 3 * N);
  bltc_upward(&t, sx, sy, sz, w, S);
  bltc_src p1 = {NULL, sx, sy, sz, w};
  bltc_interactions(&t, nl, list, theta, typed, tx, ty, tz, p1, S, NULL, NULL, eps, u, T);
  bltc_downward(&t, tx, ty, tz, T, u);
  free(S);
  free(T);
  free(list);
  bltc_tree_free(&t);
}

void orc_bltc_velocity_swe(int levels, int degree, int leaf_size, int n, double theta, double eps, int typed,
                           const double* tx, const double* ty, const double* tz, const double* sx, const double* sy,
                           const double* sz, const double* w, const double* dx, const double* dy, const double* dz,
                           const double* wd, double* u) {
  bltc_tree t;
  bltc_tree_init(levels, degree, leaf_size, n, &t);
  size_t pn = (size_t)t.Pf * t.qx, N = (size_t)t.Af * t.npl;
  long nl = orc_dual_tree_traversal(t.Lf, t.tp, theta, NULL, 0);
  int* list = (int*)malloc(sizeof(int) * 3 * (size_t)(nl > 0 ? nl : 1));
  orc_dual_tree_traversal(t.Lf, t.tp, theta, list, nl);
  double* S = (double*)calloc(pn, sizeof(double));
  double* S2 = (double*)calloc(pn, sizeof(double));
  double* T = (double*)calloc(3 * pn, sizeof(double));
  memset(u, 0, sizeof(double) * 3 * N);
  bltc_upward(&t, sx, sy, sz, w, S);
  bltc_upward(&t, dx, dy, dz, wd, S2);
  bltc_src p1 = {NULL, sx, sy, sz, w}, p2 = {NULL, dx, dy, dz, wd};
  bltc_interactions(&t, nl, list, theta, typed, tx, ty, tz, p1, S, &p2, S2, eps, u, T);
  bltc_downward(&t, tx, ty, tz, T, u);
  free(S);
  free(S2);
  free(T);
  free(list);
  bltc_tree_free(&t);
}

/* ---------------- stepper: src/bve_time_step.cpp ------------------------- */

/* BLI of a field at (x,y,z) in its located leaf: the locate + BLI + gather
 * pattern of src/bve_time_step.cpp:220-237. */
static int locate_and_basis(const orc_panel* p, int d, double x, double y, double z, double* basis) {
  double xe[2];
  xieta_from_xyz(x, y, z, xe);
  int leaf = orc_point_locate_panel(p, x, y, z);
  bli_at_leaf(p, leaf, xe[0], xe[1], d, basis);
  return leaf;
}

/* bve_find_departure_points: src/bve_time_step.cpp:172-309.  v_k holds the
 * x, y, z components as three consecutive A x q blocks. */
void orc_bve_departure(int levels, int degree, const orc_panel* p, const double* x, const double* y,
                       const double* z, const double* v0, const double* v1, const double* v2, const double* v3,
                       double dt, double* dep_x, double* dep_y, double* dep_z) {
  int q = (degree + 1) * (degree + 1), P = orc_panel_count(levels), A = orc_leaf_count(levels);
  int off = P - A;
  size_t n = (size_t)A * q;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < A; i++) {
    double b[MAXQ];
    for (int j = 0; j < q; j++) {
      size_t o = (size_t)i * q + j;
      double k1x = v3[o], k1y = v3[n + o], k1z = v3[2 * n + o];
      double xx = x[o] - 0.5 * dt * k1x, yy = y[o] - 0.5 * dt * k1y, zz = z[o] - 0.5 * dt * k1z;
      project_to_sphere(&xx, &yy, &zz);
      int leaf = locate_and_basis(p, degree, xx, yy, zz, b);
      double k2x = 0, k2y = 0, k2z = 0;
      for (int m = 0; m < q; m++) {
        size_t g = (size_t)(leaf - off) * q + m;
        k2x += v2[g] * b[m];
        k2y += v2[n + g] * b[m];
        k2z += v2[2 * n + g] * b[m];
      }
      xx = x[o] - 0.5 * dt * k2x, yy = y[o] - 0.5 * dt * k2y, zz = z[o] - 0.5 * dt * k2z;
      project_to_sphere(&xx, &yy, &zz);
      leaf = locate_and_basis(p, degree, xx, yy, zz, b);
      double k3x = 0, k3y = 0, k3z = 0;
      for (int m = 0; m < q; m++) {
        size_t g = (size_t)(leaf - off) * q + m;
        k3x += v1[g] * b[m];
        k3y += v1[n + g] * b[m];
        k3z += v1[2 * n + g] * b[m];
      }
      xx = x[o] - dt * k3x, yy = y[o] - dt * k3y, zz = z[o] - dt * k3z;
      project_to_sphere(&xx, &yy, &zz);
      leaf = locate_and_basis(p, degree, xx, yy, zz, b);
      double k4x = 0, k4y = 0, k4z = 0;
      for (int m = 0; m < q; m++) {
        size_t g = (size_t)(leaf - off) * q + m;
        k4x += v0[g] * b[m];
        k4y += v0[n + g] * b[m];
        k4z += v0[2 * n + g] * b[m];
      }
      xx = x[o] - 1.0 / 6.0 * dt * k1x, yy = y[o] - 1.0 / 6.0 * dt * k1y, zz = z[o] - 1.0 / 6.0 * dt * k1z;
      project_to_sphere(&xx, &yy, &zz);
      xx -= -1.0 / 3.0 * dt * k2x, yy -= -1.0 / 3.0 * dt * k2y, zz -= -1.0 / 3.0 * dt * k2z;
      project_to_sphere(&xx, &yy, &zz);
      xx -= -1.0 / 3.0 * dt * k3x, yy -= -1.0 / 3.0 * dt * k3y, zz -= -1.0 / 3.0 * dt * k3z;
      project_to_sphere(&xx, &yy, &zz);
      xx -= -1.0 / 6.0 * dt * k4x, yy -= -1.0 / 6.0 * dt * k4y, zz -= -1.0 / 6.0 * dt * k4z;
      project_to_sphere(&xx, &yy, &zz);
      dep_x[o] = xx;
      dep_y[o] = yy;
      dep_z[o] = zz;
    }
  }
}

/* bve_departure_to_target: src/bve_time_step.cpp:15-67 */
void orc_bve_remap(int levels, int degree, const orc_panel* p, const double* z, const double* dep_x,
                   const double* dep_y, const double* dep_z, const double* vors, int T, const double* tracers,
                   double omega, double* new_vors, double* new_tracers) {
  int q = (degree + 1) * (degree + 1), P = orc_panel_count(levels), A = orc_leaf_count(levels);
  int off = P - A;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < A; i++) {
    double b[MAXQ];
    for (int j = 0; j < q; j++) {
      size_t o = (size_t)i * q + j;
      int leaf = locate_and_basis(p, degree, dep_x[o], dep_y[o], dep_z[o], b);
      for (int k = 0; k < T; k++) new_tracers[o * T + k] = 0;
      double vor = 0;
      for (int m = 0; m < q; m++) {
        size_t g = (size_t)(leaf - off) * q + m;
        vor += vors[g] * b[m];
        for (int k = 0; k < T; k++) new_tracers[o * T + k] += tracers[g * T + k] * b[m];
      }
      vor += 2 * omega * dep_z[o];
      new_vors[o] = vor - 2 * omega * z[o];
    }
  }
}

/* bve_disp_update: src/bve_time_step.cpp:69-105 (leaves; disp rows offset). */
static void disp_update(int A, int q, int off, const double* x, const double* y, const double* z, const double* vel,
                        const double* vor, double* new_vor, double* dx, double* dy, double* dz, double dt,
                        double omega) {
  size_t n = (size_t)A * q;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < A; i++)
    for (int j = 0; j < q; j++) {
      size_t o = (size_t)i * q + j;
      double xx = x[o] + vel[o] * dt, yy = y[o] + vel[n + o] * dt, zz = z[o] + vel[2 * n + o] * dt;
      project_to_sphere(&xx, &yy, &zz);
      new_vor[o] = vor[o] + 2 * omega * z[o] - 2 * omega * zz;
      size_t d = (size_t)(i + off) * q + j;
      dx[d] = dt * vel[o];
      dy[d] = dt * vel[n + o];
      dz[d] = dt * vel[2 * n + o];
    }
}

/* bve_disp_interp: src/bve_time_step.cpp:107-160 (non-leaf panels). */
static void disp_interp(const orc_panel* p, int off, int d, const double* interp, double* dx, double* dy,
                        double* dz) {
  int q = (d + 1) * (d + 1);
#pragma omp parallel for schedule(static)
  for (int i = 0; i < off; i++) {
    double xi_off = ORC_PI / 4 * 0.5 * (p[i].max_xi + p[i].min_xi);
    double xi_scale = ORC_PI / 4 * 0.5 * (p[i].max_xi - p[i].min_xi);
    double eta_off = ORC_PI / 4 * 0.5 * (p[i].max_eta + p[i].min_eta);
    double eta_scale = ORC_PI / 4 * 0.5 * (p[i].max_eta - p[i].min_eta);
    double b[MAXQ], xyz[3];
    for (int j = 0; j < q; j++) {
      double xi = interp[4 * j] * xi_scale + xi_off, eta = interp[4 * j + 1] * eta_scale + eta_off;
      xyz_from_xieta(xi, eta, p[i].face, xyz);
      int leaf = orc_point_locate_panel(p, xyz[0], xyz[1], xyz[2]);
      bli_at_leaf(p, leaf, xi, eta, d, b);
      double ax = 0, ay = 0, az = 0;
      for (int m = 0; m < q; m++) {
        ax += dx[(size_t)leaf * q + m] * b[m];
        ay += dy[(size_t)leaf * q + m] * b[m];
        az += dz[(size_t)leaf * q + m] * b[m];
      }
      dx[(size_t)i * q + j] = ax;
      dy[(size_t)i * q + j] = ay;
      dz[(size_t)i * q + j] = az;
    }
  }
}

/* One velocity evaluation (one RK4 stage): up pass, interactions, down pass.
 * src/bve_time_step.cpp:321-348 and the repeated stage blocks after it. */
static void velocity_eval(const orc_bve_problem* pb, const double* eff_vor, const double* dx, const double* dy,
                          const double* dz, double* proxy, double* t1, double* t2, double* t3, double* vel) {
  int q = (pb->degree + 1) * (pb->degree + 1), P = orc_panel_count(pb->levels), A = orc_leaf_count(pb->levels);
  size_t n = (size_t)A * q, pq = (size_t)P * q;
  if (pb->mode == 2) {
    /* treecode: sources at the displaced particles (the leaf rows of the
     * displacement), strengths area * effective vorticity, targets at the grid */
    int off = P - A;
    double* s = (double*)malloc(sizeof(double) * 4 * n);
    for (int i = 0; i < A; i++)
      for (int j = 0; j < q; j++) {
        size_t o = (size_t)i * q + j, dd = (size_t)(i + off) * q + j;
        double xx = pb->x[o] + dx[dd], yy = pb->y[o] + dy[dd], zz = pb->z[o] + dz[dd];
        project_to_sphere(&xx, &yy, &zz);
        s[o] = xx;
        s[n + o] = yy;
        s[2 * n + o] = zz;
        s[3 * n + o] = pb->area[o] * eff_vor[o];
      }
    orc_bltc_velocity(pb->levels, pb->degree, pb->leaf_size, pb->proxy_degree, pb->theta, pb->kernel_eps, pb->typed,
                      pb->x, pb->y, pb->z, s, s + n, s + 2 * n, s + 3 * n, vel);
    free(s);
    return;
  }
  orc_upward_pass(pb->levels, pb->degree, pb->panels, pb->interp, pb->area, eff_vor, proxy);
  memset(t1, 0, sizeof(double) * pq);
  memset(t2, 0, sizeof(double) * pq);
  memset(t3, 0, sizeof(double) * pq);
  if (pb->mode == 1)
    orc_bve_direct_velocity(pb->levels, pb->degree, pb->panels, pb->interp, dx, dy, dz, proxy, pb->kernel_eps, t1,
                            t2, t3);
  else
    orc_bve_vel_interactions(pb->levels, pb->degree, pb->panels, pb->interp, pb->n_list, pb->list, dx, dy, dz,
                             proxy, pb->kernel_eps, t1, t2, t3);
  orc_downward_pass_3(pb->levels, pb->degree, pb->panels, pb->interp, t1, t2, t3, vel, vel + n, vel + 2 * n);
}

/* bve_forcing (src/forcing_funcs.cpp:82-96): eff = vor without forcing;
 * with it, bve_ssw_forcing (type 1, :6-43) or bve_ssw_forcing_2 (type 2,
 * :45-80) per leaf panel, points in order, bcomp kept from the panel's
 * previous point where lat <= 0 as the reference's loop keeps it. */
static void bve_forcing(const orc_bve_problem* pb, const double* vor, double* eff) {
  int A = orc_leaf_count(pb->levels), q = (pb->degree + 1) * (pb->degree + 1);
  if (pb->forcing == 0) {
    memcpy(eff, vor, sizeof(double) * (size_t)A * q);
    return;
  }
  double Tp = 4.0, Tf = 4.0 + 11.0, theta1 = ORC_PI / 3.0, time = pb->time;
  for (int i = 0; i < A; i++) {
    double lat, lon, acomp, bcomp = 0, ccomp;
    for (int j = 0; j < q; j++) {
      size_t o = (size_t)i * q + j;
      double x = pb->x[o], y = pb->y[o], z = pb->z[o];
      lat = ORC_PI / 2.0 - atan2(sqrt(x * x + y * y), z); /* xyz_to_latlon, src/general_utils_impl.hpp:230-235 */
      lon = atan2(y, x);
      if (time / 86400.0 < Tp) acomp = 0.5 * (1.0 - cos(ORC_PI * (time / 86400.0) / Tp));
      else if (time / 86400.0 < Tf - Tp) acomp = 1.0;
      else if (time / 86400.0 < Tf) acomp = 0.5 * (1.0 - cos(ORC_PI + ORC_PI * ((time / 86400.0) - Tf + Tp) / Tp));
      else acomp = 0.0;
      if (lat > 0) {
        ccomp = pow(tan(theta1), 2) / pow(tan(lat), 2);
        bcomp = ccomp * exp(1.0 - ccomp);
      }
      if (pb->forcing == 1) eff[o] = vor[o] + 0.6 * pb->omega * acomp * bcomp * cos(lon);
      else eff[o] = vor[o] + 1.2 * pb->omega * acomp * bcomp * cos(2.0 * lon);
    }
  }
}

/* bve_back_rk4_step: src/bve_time_step.cpp:311-419; the effective vorticity
 * of every stage is bve_forcing of the (displaced) relative vorticity at the
 * step's time. */
void orc_bve_step(const orc_bve_problem* pb, double* vors, double* vel_x, double* vel_y, double* vel_z,
                  double* tracers) {
  int d = pb->degree, q = (d + 1) * (d + 1), P = orc_panel_count(pb->levels), A = orc_leaf_count(pb->levels);
  int off = P - A, T = pb->tracer_count;
  size_t n = (size_t)A * q, pq = (size_t)P * q;
  double* dx = (double*)calloc(pq, sizeof(double));
  double* dy = (double*)calloc(pq, sizeof(double));
  double* dz = (double*)calloc(pq, sizeof(double));
  double* proxy = (double*)calloc(pq, sizeof(double));
  double* t1 = (double*)calloc(pq, sizeof(double));
  double* t2 = (double*)calloc(pq, sizeof(double));
  double* t3 = (double*)calloc(pq, sizeof(double));
  double* v[4];
  for (int k = 0; k < 4; k++) v[k] = (double*)calloc(3 * n, sizeof(double));
  double* dvor = (double*)calloc(n, sizeof(double));
  double* dep = (double*)calloc(3 * n, sizeof(double));
  double* nv = (double*)calloc(n, sizeof(double));
  double* ntr = (double*)calloc(n * (T > 0 ? T : 1), sizeof(double));
  double* eff = (double*)calloc(n, sizeof(double));

  bve_forcing(pb, vors, eff);
  velocity_eval(pb, eff, dx, dy, dz, proxy, t1, t2, t3, v[0]);
  const double fr[3] = {0.5, 0.5, 1.0};
  for (int s = 1; s < 4; s++) {
    disp_update(A, q, off, pb->x, pb->y, pb->z, v[s - 1], vors, dvor, dx, dy, dz, fr[s - 1] * pb->dt, pb->omega);
    if (pb->mode != 2) disp_interp(pb->panels, off, d, pb->interp, dx, dy, dz);
    bve_forcing(pb, dvor, eff);
    velocity_eval(pb, eff, dx, dy, dz, proxy, t1, t2, t3, v[s]);
  }
  orc_bve_departure(pb->levels, d, pb->panels, pb->x, pb->y, pb->z, v[0], v[1], v[2], v[3], pb->dt, dep, dep + n,
                    dep + 2 * n);
  orc_bve_remap(pb->levels, d, pb->panels, pb->z, dep, dep + n, dep + 2 * n, vors, T, tracers, pb->omega, nv, ntr);
  memcpy(vors, nv, sizeof(double) * n);
  if (T > 0) memcpy(tracers, ntr, sizeof(double) * n * T);
  memcpy(vel_x, v[0], sizeof(double) * n);
  memcpy(vel_y, v[0] + n, sizeof(double) * n);
  memcpy(vel_z, v[0] + 2 * n, sizeof(double) * n);
  free(dx); free(dy); free(dz); free(proxy); free(t1); free(t2); free(t3);
  for (int k = 0; k < 4; k++) free(v[k]);
  free(dvor); free(dep); free(nv); free(ntr); free(eff);
}

/* inv_lap: src/direct_sum_impl.hpp:20-27 (row i sums over j in order). */
void orc_direct_sum_inv_lap(int n, const double* x, const double* y, const double* z, const double* area,
                            const double* pots, double* soln) {
#pragma omp parallel for schedule(static)
  for (int i = 0; i < n; i++) {
    double acc = soln[i];
    for (int j = 0; j < n; j++) {
      if (i != j) {
        double dp = x[i] * x[j] + y[i] * y[j] + z[i] * z[j];
        acc += -0.07957747154594767 * log(1 - dp) * area[j] * pots[j];
      }
    }
    soln[i] = acc;
  }
}

/* ---------------- output path: src/interp_funcs.hpp, src/general_utils_impl.hpp ---------------- */

/* latlon_interp_host::operator() (src/interp_funcs.hpp:38-70) over the whole
 * (lat, lon) grid, as interp_to_latlon_host (src/interp_funcs.hpp:72-77) runs
 * it: the point of latitude lats[i] / longitude lons[j] (degrees), its leaf
 * by point_locate_panel_2 (src/interp_funcs.cpp:175-203, the same descent as
 * point_locate_panel), the face-free xieta_from_xyz, interp_vals_bli at the
 * leaf and the sum over m, n in order.  data is [leaf][q]; out is [nlat][nlon]. */
void orc_interp_to_latlon(int levels, int degree, const orc_panel* p, const double* data, int nlat,
                          const double* lats, int nlon, const double* lons, double* out) {
  int q = (degree + 1) * (degree + 1), off = orc_panel_count(levels) - orc_leaf_count(levels);
  double basis[MAXQ], xe[2];
  for (int i = 0; i < nlat; i++)
    for (int j = 0; j < nlon; j++) {
      double lat = lats[i] * ORC_PI / 180.0, lon = lons[j] * ORC_PI / 180.0;
      double x = cos(lat) * cos(lon), y = cos(lat) * sin(lon), z = sin(lat);
      int panel = orc_point_locate_panel(p, x, y, z);
      xieta_from_xyz(x, y, z, xe);
      orc_interp_vals_bli(basis, xe[0], xe[1], ORC_PI / 4.0 * p[panel].min_xi, ORC_PI / 4.0 * p[panel].max_xi,
                          ORC_PI / 4.0 * p[panel].min_eta, ORC_PI / 4.0 * p[panel].max_eta, degree);
      double acc = 0;
      for (int m = 0; m < degree + 1; m++)
        for (int n = 0; n < degree + 1; n++) {
          int k = m * (degree + 1) + n;
          acc += basis[k] * data[(long)(panel - off) * q + k];
        }
      out[(long)i * nlon + j] = acc;
    }
}

/* xyz_vel_to_uv_vel (src/general_utils_impl.hpp:195-229): zonal and
 * meridional components of a tangent velocity, zero within 1e-16 of a pole. */
void orc_xyz_vel_to_uv_vel(long n, const double* x, const double* y, const double* z, const double* vx,
                           const double* vy, const double* vz, double* u, double* v) {
  for (long i = 0; i < n; i++) {
    double xx = x[i], yy = y[i], zz = z[i], xc = vx[i], yc = vy[i], zc = vz[i];
    if (fabs(zz) < 1 - 1e-16) {
      u[i] = (-yy * xc + xx * yc) / sqrt(xx * xx + yy * yy);
      v[i] = -((xx * xc + yy * yc) * zz - (xx * xx + yy * yy) * zc) / sqrt(xx * xx + yy * yy);
    } else {
      u[i] = 0;
      v[i] = 0;
    }
  }
}

/* ---------------- Poisson FMM: src/fmm_interactions/inverse_poisson*.{hpp,cpp} ---------------- */

/* poisson_fmm_interactions (src/fmm_interactions/inverse_poisson.cpp:9-34)
 * with one rank: for each list entry, poisson_panel_interaction
 * (src/fmm_interactions/inverse_poisson_impl.hpp:22-52) adds
 * -1/(4 pi) log(1 - x_t.x_s) w_s over the two panels' proxy points, skipping
 * pairs with x_t.x_s >= 1 - 1e-15.  Entries grouped by target panel (stable),
 * sources in list order, source points k in order. */
void orc_poisson_fmm_interactions(int levels, int degree, const orc_panel* p, const double* interp, long n_list,
                                  const int* list, const double* source, double* target) {
  int q = (degree + 1) * (degree + 1), P = orc_panel_count(levels);
  long* start = (long*)calloc((size_t)P + 1, sizeof(long));
  long* order = (long*)malloc(sizeof(long) * (size_t)(n_list > 0 ? n_list : 1));
  for (long i = 0; i < n_list; i++) start[list[3 * i] + 1]++;
  for (int i = 0; i < P; i++) start[i + 1] += start[i];
  long* fill = (long*)malloc(sizeof(long) * (size_t)P);
  for (int i = 0; i < P; i++) fill[i] = start[i];
  for (long i = 0; i < n_list; i++) order[fill[list[3 * i]]++] = i;
#pragma omp parallel for schedule(dynamic, 16)
  for (int t = 0; t < P; t++) {
    double xt[3], xs[3];
    for (long e = start[t]; e < start[t + 1]; e++) {
      int s = list[3 * order[e] + 1];
      for (int j = 0; j < q; j++) {
        proxy_point(p, t, interp, j, xt);
        double a = target[(size_t)t * q + j];
        for (int k = 0; k < q; k++) {
          proxy_point(p, s, interp, k, xs);
          double dp = xt[0] * xs[0] + xt[1] * xs[1] + xt[2] * xs[2];
          if (dp < 1.0 - 1e-15) a += -0.07957747154594767 * log(1 - dp) * source[(size_t)s * q + k];
        }
        target[(size_t)t * q + j] = a;
      }
    }
  }
  free(start);
  free(order);
  free(fill);
}

/* downward_pass (src/fmm_funcs.cpp:357-372): parent_to_child per level, then
 * child_panel_copy of the leaves; the one-field form of downward_pass_3. */
void orc_downward_pass(int levels, int degree, const orc_panel* p, const double* interp, double* t, double* s) {
  int q = (degree + 1) * (degree + 1), P = orc_panel_count(levels);
  double* z = (double*)calloc((size_t)2 * P * q, sizeof(double));
  double* zs = (double*)calloc((size_t)2 * orc_leaf_count(levels) * q, sizeof(double));
  orc_downward_pass_3(levels, degree, p, interp, t, z, z + (size_t)P * q, s, zs, zs + (size_t)orc_leaf_count(levels) * q);
  free(z);
  free(zs);
}

/* ---------------- shallow water v2 ---------------- */

/* One panel-pair block of swe_vel_panel_interaction_2
 * (src/fmm_interactions/swe_vel_impl.hpp:104-146): the rotational term at the
 * displaced, re-projected source points, the divergent term at the fixed
 * source points; per target, the two terms of source k are added in that
 * order (the reference's two atomic adds per component). */
static void swe_pair_block(const orc_panel* p, const double* interp, int q, int t, int s, const double* dx,
                           const double* dy, const double* dz, const double* sv, const double* sd, double eps,
                           double* t1, double* t2, double* t3) {
  double fx[MAXQ][3], mv[MAXQ][3];
  for (int k = 0; k < q; k++) {
    proxy_point(p, s, interp, k, fx[k]);
    double x_s = fx[k][0] + dx[(size_t)s * q + k], y_s = fx[k][1] + dy[(size_t)s * q + k],
           z_s = fx[k][2] + dz[(size_t)s * q + k];
    project_to_sphere(&x_s, &y_s, &z_s);
    mv[k][0] = x_s;
    mv[k][1] = y_s;
    mv[k][2] = z_s;
  }
  for (int j = 0; j < q; j++) {
    double xt[3];
    proxy_point(p, t, interp, j, xt);
    double a1 = t1[(size_t)t * q + j], a2 = t2[(size_t)t * q + j], a3 = t3[(size_t)t * q + j];
    for (int k = 0; k < q; k++) {
      const double* m = mv[k];
      const double* f = fx[k];
      double dp = xt[0] * m[0] + xt[1] * m[1] + xt[2] * m[2];
      double dp2 = xt[0] * f[0] + xt[1] * f[1] + xt[2] * f[2];
      double g1 = -(0.07957747154594767 / (1.0 - dp + eps)) * sv[(size_t)s * q + k];
      double g2 = 0.07957747154594767 / (1.0 - dp2 + eps) * sd[(size_t)s * q + k];
      a1 += g1 * (xt[1] * m[2] - xt[2] * m[1]);
      a2 += g1 * (xt[2] * m[0] - xt[0] * m[2]);
      a3 += g1 * (xt[0] * m[1] - xt[1] * m[0]);
      a1 += g2 * (f[0] - xt[0] * dp2);
      a2 += g2 * (f[1] - xt[1] * dp2);
      a3 += g2 * (f[2] - xt[2] * dp2);
    }
    t1[(size_t)t * q + j] = a1;
    t2[(size_t)t * q + j] = a2;
    t3[(size_t)t * q + j] = a3;
  }
}

/* swe_vel_interactions_2: src/fmm_interactions/swe_vel.cpp:39-67 with one
 * rank; grouped by target panel as orc_bve_vel_interactions. */
void orc_swe_vel_interactions(int levels, int degree, const orc_panel* p, const double* interp, long n_list,
                              const int* list, const double* disp_x, const double* disp_y, const double* disp_z,
                              const double* src_vor, const double* src_div, double eps, double* t1, double* t2,
                              double* t3) {
  int q = (degree + 1) * (degree + 1), P = orc_panel_count(levels);
  long* start = (long*)calloc((size_t)P + 1, sizeof(long));
  long* order = (long*)malloc(sizeof(long) * (size_t)(n_list > 0 ? n_list : 1));
  long* fill = (long*)malloc(sizeof(long) * (size_t)P);
  for (long i = 0; i < n_list; i++) start[list[3 * i] + 1]++;
  for (int i = 0; i < P; i++) start[i + 1] += start[i];
  for (int i = 0; i < P; i++) fill[i] = start[i];
  for (long i = 0; i < n_list; i++) order[fill[list[3 * i]]++] = i;
#pragma omp parallel for schedule(dynamic, 16)
  for (int t = 0; t < P; t++)
    for (long e = start[t]; e < start[t + 1]; e++)
      swe_pair_block(p, interp, q, t, list[3 * order[e] + 1], disp_x, disp_y, disp_z, src_vor, src_div, eps, t1, t2,
                     t3);
  free(start);
  free(order);
  free(fill);
}

/* The three-point finite-difference derivative along one direction of a
 * (d+1) x (d+1) panel grid, fd_deriv_xi / fd_deriv_eta
 * (src/deriv_funcs_impl.hpp:94-185): node k at cos(k pi / d) scaled to
 * [lo, hi], one-sided second-order weights at the two end nodes, the
 * non-uniform centred weights inside (the shorter neighbouring gap is h).
 * Values of the line are f[base + k * stride]; xi lines have stride d + 1
 * (base = the eta index), eta lines stride 1 (base = xi index * (d + 1)). */
static void fd_line(double* out, const double* f, int d, double lo, double hi, int base, int stride) {
  const double scale = 0.5 * (hi - lo), off = 0.5 * (hi + lo);
  {
    const double n0 = hi, n1 = cos(ORC_PI / d) * scale + off, n2 = cos(ORC_PI * 2.0 / d) * scale + off;
    const double h = n0 - n1, ratio = (n0 - n2) / (n0 - n1);
    const double w0 = -1.0 - 1.0 / ratio, w1 = ratio / (ratio - 1.0), w2 = -1.0 / (ratio * ratio - ratio);
    int a = base;
    out[a] = (w0 * f[a] + w1 * f[a + stride] + w2 * f[a + 2 * stride]) / h;
    a = base + d * stride;
    out[a] = -(w0 * f[a] + w1 * f[a - stride] + w2 * f[a - 2 * stride]) / h;
  }
  for (int k = 1; k < d; k++) {
    const double n0 = cos((k - 1) * ORC_PI / d) * scale + off, n1 = cos(k * ORC_PI / d) * scale + off,
                 n2 = cos((k + 1) * ORC_PI / d) * scale + off;
    const double g1 = n0 - n1, g2 = n1 - n2, h = fmin(g1, g2), ratio = fmax(g1 / h, g2 / h);
    double w0, w1, w2;
    if (g1 < g2) {
      w0 = -ratio / (ratio + 1.0);
      w1 = (ratio - 1.0) / ratio;
      w2 = 1.0 / (ratio * ratio + ratio);
    } else {
      w0 = -1.0 / (ratio * ratio + ratio);
      w1 = (1.0 - ratio) / ratio;
      w2 = ratio / (ratio + 1.0);
    }
    const int a = base + k * stride;
    out[a] = (w0 * f[a - stride] + w1 * f[a] + w2 * f[a + stride]) / h;
  }
}

static void fd_xi(double* out, const double* f, int d, double lo, double hi) {
  for (int j = 0; j <= d; j++) fd_line(out, f, d, lo, hi, j, d + 1);
}

static void fd_eta(double* out, const double* f, int d, double lo, double hi) {
  for (int i = 0; i <= d; i++) fd_line(out, f, d, lo, hi, i * (d + 1), 1);
}

/* spatial_filter_vals (src/deriv_funcs_impl.hpp:391-441): each value takes
 * (1 - c) of itself plus c / 4 of a distance-weighted pair of neighbours in
 * each direction (the two nearer nodes on the reference interval [-1, 1]),
 * c = 0.0005. */
static void spatial_filter(double* out, const double* f, int d) {
  const double c = 0.0005;
  for (int i = 0; i <= d; i++) {
    const double xi = cos(ORC_PI * i / d);
    const int ia = i == 0 ? 1 : i - 1, ib = i == 0 ? 2 : (i == d ? i - 2 : i + 1);
    const double xd1 = fabs(xi - cos(ORC_PI * ia / d)), xd2 = fabs(xi - cos(ORC_PI * ib / d));
    for (int j = 0; j <= d; j++) {
      const double eta = cos(ORC_PI * j / d);
      const int ja = j == 0 ? 1 : j - 1, jb = j == 0 ? 2 : (j == d ? j - 2 : j + 1);
      const double ed1 = fabs(eta - cos(ORC_PI * ja / d)), ed2 = fabs(eta - cos(ORC_PI * jb / d));
      const int k = i * (d + 1) + j;
      const double f1 = f[ia * (d + 1) + j], f2 = f[ib * (d + 1) + j], f3 = f[i * (d + 1) + ja],
                   f4 = f[i * (d + 1) + jb];
      double v = (1.0 - c) * f[k];
      v += 0.25 * c / (xd1 + xd2) * xd1 * f2;
      v += 0.25 * c / (xd1 + xd2) * xd2 * f1;
      v += 0.25 * c / (ed1 + ed2) * ed1 * f4;
      v += 0.25 * c / (ed1 + ed2) * ed2 * f3;
      out[k] = v;
    }
  }
}

/* The panel's node tangents X = tan(xi), Y = tan(eta) at node (i, j). */
static void node_tan(int d, int i, int j, double min_xi, double max_xi, double min_eta, double max_eta, double* X,
                     double* Y) {
  const double xi = cos(ORC_PI * i / d) * (0.5 * (max_xi - min_xi)) + 0.5 * (min_xi + max_xi);
  const double eta = cos(ORC_PI * j / d) * (0.5 * (max_eta - min_eta)) + 0.5 * (min_eta + max_eta);
  *X = tan(xi);
  *Y = tan(eta);
}

/* single_panel_lap_fd (src/deriv_funcs_impl.hpp:510-560): the surface
 * Laplacian in gnomonic coordinates from the finite differences (the mixed
 * derivative as the mean of the two orders), then the spatial filter. */
static void panel_lap(double* out, const double* f, double mnx, double mxx, double mne, double mxe, int d) {
  double fx[MAXQ], fe[MAXQ], fxx[MAXQ], fee[MAXQ], fxe[MAXQ], fex[MAXQ], lap[MAXQ];
  fd_xi(fx, f, d, mnx, mxx);
  fd_eta(fe, f, d, mne, mxe);
  fd_xi(fxx, fx, d, mnx, mxx);
  fd_eta(fee, fe, d, mne, mxe);
  fd_eta(fxe, fx, d, mne, mxe);
  fd_xi(fex, fe, d, mnx, mxx);
  for (int i = 0; i <= d; i++)
    for (int j = 0; j <= d; j++) {
      const int k = i * (d + 1) + j;
      double X, Y;
      node_tan(d, i, j, mnx, mxx, mne, mxe, &X, &Y);
      const double C2 = 1 + X * X, D2 = 1 + Y * Y, delta = 1 + X * X + Y * Y;
      const double mix = 0.5 * (fxe[k] + fex[k]);
      lap[k] = delta * (fxx[k] / C2 + fee[k] / D2 + 2.0 * X * Y / (C2 * D2) * mix);
    }
  spatial_filter(out, lap, d);
}

/* single_panel_curl_rad_comp_fd (src/deriv_funcs_impl.hpp:591-619): the
 * radial component of the curl of the tangent field (a, b) given by its
 * gnomonic components, then the spatial filter. */
static void panel_curl_rad(double* out, const double* a, const double* b, double mnx, double mxx, double mne,
                           double mxe, int d) {
  double ax[MAXQ], bx[MAXQ], ae[MAXQ], be[MAXQ], curl[MAXQ];
  fd_xi(ax, a, d, mnx, mxx);
  fd_xi(bx, b, d, mnx, mxx);
  fd_eta(ae, a, d, mne, mxe);
  fd_eta(be, b, d, mne, mxe);
  for (int i = 0; i <= d; i++)
    for (int j = 0; j <= d; j++) {
      const int k = i * (d + 1) + j;
      double X, Y;
      node_tan(d, i, j, mnx, mxx, mne, mxe, &X, &Y);
      const double C = sqrt(1 + X * X), D = sqrt(1 + Y * Y), delta = 1 + X * X + Y * Y;
      curl[k] = -sqrt(delta) * (X * Y / (C * D) * (be[k] / D - ax[k] / C) - ae[k] / D + bx[k] / C);
    }
  spatial_filter(out, curl, d);
}

/* single_panel_div_fd (src/deriv_funcs_impl.hpp:661-698): the divergence of
 * the tangent field (a, b), no filter. */
static void panel_div(double* out, const double* a, const double* b, double mnx, double mxx, double mne, double mxe,
                      int d) {
  double as[MAXQ], bs[MAXQ], ax[MAXQ], be[MAXQ];
  for (int i = 0; i <= d; i++)
    for (int j = 0; j <= d; j++) {
      const int k = i * (d + 1) + j;
      double X, Y;
      node_tan(d, i, j, mnx, mxx, mne, mxe, &X, &Y);
      const double delta = 1 + X * X + Y * Y;
      as[k] = a[k] / sqrt(delta);
      bs[k] = b[k] / sqrt(delta);
    }
  fd_xi(ax, as, d, mnx, mxx);
  fd_eta(be, bs, d, mne, mxe);
  for (int i = 0; i <= d; i++)
    for (int j = 0; j <= d; j++) {
      const int k = i * (d + 1) + j;
      double X, Y;
      node_tan(d, i, j, mnx, mxx, mne, mxe, &X, &Y);
      const double C = sqrt(1 + X * X), D = sqrt(1 + Y * Y), delta = 1 + X * X + Y * Y;
      out[k] = pow(delta, 1.5) / (C * D) * (ax[k] / C + be[k] / D);
    }
}

/* xietavec_from_xyzvec (src/cubed_sphere_transforms_impl.hpp:242-276): a
 * tangent vector's gnomonic components at (x, y, z), from its longitude and
 * colatitude components; within 1e-16 of a pole the x and y components. */
static void xieta_vec(double* xc, double* ec, double vx, double vy, double vz, double x, double y, double z) {
  double xe[2];
  xieta_from_xyz(x, y, z, xe);
  const int face = face_from_xyz(x, y, z);
  if (!(fabs(z) < 1 - 1e-16)) {
    *xc = vx;
    *ec = vy;
    return;
  }
  const double lon = (-y * vx + x * vy) / sqrt(x * x + y * y);
  const double colat = ((x * vx + y * vy) * z - (x * x + y * y) * vz) / sqrt(x * x + y * y);
  const double X = tan(xe[0]), Y = tan(xe[1]), X2 = X * X, Y2 = Y * Y;
  const double C = sqrt(1 + X2), D = sqrt(1 + Y2), delta = 1 + X2 + Y2;
  if (face <= 3) {
    *xc = C * D / sqrt(delta) * lon;
    *ec = -1.0 * colat + X * Y / sqrt(delta) * lon;
  } else {
    const double sg = face == 4 ? 1.0 : -1.0;
    *xc = sg / sqrt(X2 + Y2) * (D * X * colat - D * Y / sqrt(delta) * lon);
    *ec = sg / sqrt(X2 + Y2) * (C * Y * colat + C * X / sqrt(delta) * lon);
  }
}

/* swe_tendency_computation_2 (src/swe_time_step_2_impl.hpp:41-127): per leaf
 * panel, the vorticity tendency -delta (zeta + 2 Omega z) - 2 Omega v_z, the
 * divergence tendency curl_r((zeta + 2 Omega z) v) - (g/a) lap(surface) -
 * lap(|v|^2 / 2) and the height tendency div(h v), the last two zero within
 * 1e-5 of the poles.  The reference hard-codes g/a = 9.81 / 6371000. */
void orc_swe_tendencies(int levels, int degree, const orc_panel* p, const double* x, const double* y,
                        const double* z, const double* vx, const double* vy, const double* vz, const double* vors,
                        const double* divs, const double* height, const double* surface, double omega,
                        double g_over_a, double* vor_t, double* div_t, double* h_t) {
  const int d = degree, q = (d + 1) * (d + 1), P = orc_panel_count(levels), A = orc_leaf_count(levels);
  const int off = P - A;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < A; i++) {
    const orc_panel* pp = &p[i + off];
    const double mnx = ORC_PI / 4.0 * pp->min_xi, mxx = ORC_PI / 4.0 * pp->max_xi;
    const double mne = ORC_PI / 4.0 * pp->min_eta, mxe = ORC_PI / 4.0 * pp->max_eta;
    double va[MAXQ], vb[MAXQ], ha[MAXQ], hb[MAXQ], sf[MAXQ], ke[MAXQ];
    double curl[MAXQ], hlap[MAXQ], klap[MAXQ], hdiv[MAXQ];
    for (int j = 0; j < q; j++) {
      const size_t o = (size_t)i * q + j;
      xieta_vec(&va[j], &vb[j], vx[o], vy[o], vz[o], x[o], y[o], z[o]);
      ha[j] = height[o] * va[j];
      hb[j] = height[o] * vb[j];
      const double zetaf = vors[o] + 2 * omega * z[o];
      va[j] *= zetaf;
      vb[j] *= zetaf;
      sf[j] = surface[o];
      ke[j] = 0.5 * (vx[o] * vx[o] + vy[o] * vy[o] + vz[o] * vz[o]);
    }
    panel_curl_rad(curl, va, vb, mnx, mxx, mne, mxe, d);
    panel_lap(hlap, sf, mnx, mxx, mne, mxe, d);
    panel_lap(klap, ke, mnx, mxx, mne, mxe, d);
    panel_div(hdiv, ha, hb, mnx, mxx, mne, mxe, d);
    for (int j = 0; j < q; j++) {
      const size_t o = (size_t)i * q + j;
      const double abs_vor = vors[o] + 2.0 * omega * z[o];
      vor_t[o] = -divs[o] * abs_vor - 2.0 * omega * vz[o];
      div_t[o] = curl[j] - hlap[j] * g_over_a - klap[j];
      h_t[o] = hdiv[j];
      if (1.0 - fabs(z[o]) < 1e-5) {
        div_t[o] = 0.0;
        h_t[o] = 0.0;
      }
    }
  }
}

/* unify_boundary_vals (src/initialize_cubed_sphere.cpp:364-370): every copy
 * of a point shared by panels takes the mean of the copies (sums in panel
 * order).  map: [leaf][q] -> distinct point, counts: copies per point. */
void orc_swe_unify(int n, const int* map, const int* counts, int points, double* vals) {
  double* acc = (double*)calloc((size_t)points, sizeof(double));
  for (int i = 0; i < n; i++) acc[map[i]] += vals[i];
  for (int i = 0; i < n; i++) vals[i] = acc[map[i]] / counts[map[i]];
  free(acc);
}

/* One velocity evaluation of the SWE step: vorticity strengths (area_v x
 * vor) and divergence strengths (area x div) up, the two-field interactions
 * at the displacement (dx, dy, dz), down into vel (3 x A x q). */
static void swe_velocity(const orc_swe_problem* pb, const double* area_v, const double* vor, const double* div,
                         const double* dx, const double* dy, const double* dz, double* sv, double* sd, double* t1,
                         double* t2, double* t3, double* vel) {
  const int q = (pb->degree + 1) * (pb->degree + 1), P = orc_panel_count(pb->levels), A = orc_leaf_count(pb->levels);
  const size_t n = (size_t)A * q, pq = (size_t)P * q;
  orc_upward_pass(pb->levels, pb->degree, pb->panels, pb->interp, area_v, vor, sv);
  orc_upward_pass(pb->levels, pb->degree, pb->panels, pb->interp, pb->area, div, sd);
  memset(t1, 0, sizeof(double) * pq);
  memset(t2, 0, sizeof(double) * pq);
  memset(t3, 0, sizeof(double) * pq);
  orc_swe_vel_interactions(pb->levels, pb->degree, pb->panels, pb->interp, pb->n_list, pb->list, dx, dy, dz, sv, sd,
                           pb->kernel_eps, t1, t2, t3);
  memset(vel, 0, sizeof(double) * 3 * n);
  orc_downward_pass_3(pb->levels, pb->degree, pb->panels, pb->interp, t1, t2, t3, vel, vel + n, vel + 2 * n);
}

/* swe_back_rk4_step_2 (src/swe_time_step_2.cpp:785-1035), topography none
 * (the effective height is the height).  Stage s > 0 displaces the sources
 * by dt_s times the previous stage's velocity (dt/2, dt/2, dt; leaves, then
 * the non-leaf proxies interpolated, swe_displacement_upward_pass_2
 * :486-496) and evaluates the velocity of the sources with the previous
 * stage's tendencies applied over dt/2 (swe_apply_tendencies_2 :384-414, the
 * vorticity strength with the area scaled by 1 + dt/2 div); after every
 * stage the reference unifies the first stage's velocity (its
 * unify_boundary_vals calls name vel_x/y/z), so that velocity is unified four
 * times and the later ones never.  Tendencies of stages 1-3 (the fourth
 * reaches no result) use the original vorticity and divergence with the
 * stage's height, minus the base divergence and height tendencies
 * (modify_tendencies :765-783), unified.  Arrival values are forward Euler
 * with the first tendencies (swe_compute_arrival_values_2 :555-626; its
 * interpolations of the later vorticity tendencies reach no output and are
 * not evaluated), the departure search is the BVE one on the four stage
 * velocities (swe_find_departure_points_2 :663-763), and the arrival
 * vorticity and the tracers are remapped without a planetary term
 * (swe_departure_to_target_2 :40-64). */
void orc_swe_step(const orc_swe_problem* pb, double* vors, double* divs, double* height, double* vel_x,
                  double* vel_y, double* vel_z, double* tracers) {
  const int d = pb->degree, q = (d + 1) * (d + 1), P = orc_panel_count(pb->levels), A = orc_leaf_count(pb->levels);
  const int off = P - A, T = pb->tracer_count;
  const size_t n = (size_t)A * q, pq = (size_t)P * q;
  double* dx = (double*)calloc(pq, sizeof(double));
  double* dy = (double*)calloc(pq, sizeof(double));
  double* dz = (double*)calloc(pq, sizeof(double));
  double* sv = (double*)calloc(pq, sizeof(double));
  double* sd = (double*)calloc(pq, sizeof(double));
  double* t1 = (double*)calloc(pq, sizeof(double));
  double* t2 = (double*)calloc(pq, sizeof(double));
  double* t3 = (double*)calloc(pq, sizeof(double));
  double* v[4];
  double* tend[3];
  for (int k = 0; k < 4; k++) v[k] = (double*)calloc(3 * n, sizeof(double));
  for (int k = 0; k < 3; k++) tend[k] = (double*)calloc(3 * n, sizeof(double));
  double* dvor = (double*)calloc(n, sizeof(double));
  double* ddiv = (double*)calloc(n, sizeof(double));
  double* dh = (double*)calloc(n, sizeof(double));
  double* darea = (double*)calloc(n, sizeof(double));
  double* dep = (double*)calloc(3 * n, sizeof(double));
  double* nv = (double*)calloc(n, sizeof(double));
  double* ntr = (double*)calloc(n * (T > 0 ? T : 1), sizeof(double));
  const double fr[3] = {0.5, 0.5, 1.0};
  for (int s = 0; s < 4; s++) {
    const double* hs = height;  /* the stage's height (and surface) */
    if (s == 0) {
      swe_velocity(pb, pb->area, vors, divs, dx, dy, dz, sv, sd, t1, t2, t3, v[0]);
    } else {
      const double h = fr[s - 1] * pb->dt, ha = 0.5 * pb->dt;
      const double* vp = v[s - 1];
      for (int i = 0; i < A; i++)
        for (int j = 0; j < q; j++) {
          const size_t o = (size_t)i * q + j, g = (size_t)(i + off) * q + j;
          dx[g] = h * vp[o];
          dy[g] = h * vp[n + o];
          dz[g] = h * vp[2 * n + o];
        }
      disp_interp(pb->panels, off, d, pb->interp, dx, dy, dz);
      const double* tp = tend[s - 1];
      for (size_t o = 0; o < n; o++) {
        dvor[o] = vors[o] + ha * tp[o];
        ddiv[o] = divs[o] + ha * tp[n + o];
        dh[o] = height[o] + ha * tp[2 * n + o];
        darea[o] = pb->area[o] * (1.0 + ha * divs[o]);
      }
      swe_velocity(pb, darea, dvor, ddiv, dx, dy, dz, sv, sd, t1, t2, t3, v[s]);
      hs = dh;
    }
    for (int c = 0; c < 3; c++) orc_swe_unify((int)n, pb->map, pb->counts, pb->point_count, v[0] + c * n);
    if (s < 3) {
      double* tq = tend[s];
      orc_swe_tendencies(pb->levels, d, pb->panels, pb->x, pb->y, pb->z, v[s], v[s] + n, v[s] + 2 * n, vors, divs,
                         hs, hs, pb->omega, pb->g_over_a, tq, tq + n, tq + 2 * n);
      for (size_t o = 0; o < n; o++) {
        tq[n + o] -= pb->base_div[o];
        tq[2 * n + o] -= pb->base_h[o];
      }
      for (int c = 0; c < 3; c++) orc_swe_unify((int)n, pb->map, pb->counts, pb->point_count, tq + c * n);
    }
  }
  /* arrival values and the departure search */
  for (size_t o = 0; o < n; o++) {
    nv[o] = vors[o] + pb->dt * tend[0][o];
    divs[o] = divs[o] + pb->dt * tend[0][n + o];
    height[o] = height[o] + pb->dt * tend[0][2 * n + o];
  }
  orc_bve_departure(pb->levels, d, pb->panels, pb->x, pb->y, pb->z, v[0], v[1], v[2], v[3], pb->dt, dep, dep + n,
                    dep + 2 * n);
  orc_bve_remap(pb->levels, d, pb->panels, pb->z, dep, dep + n, dep + 2 * n, nv, T, tracers, 0.0, vors, ntr);
  if (T > 0) memcpy(tracers, ntr, sizeof(double) * n * T);
  memcpy(vel_x, v[0], sizeof(double) * n);
  memcpy(vel_y, v[0] + n, sizeof(double) * n);
  memcpy(vel_z, v[0] + 2 * n, sizeof(double) * n);
  free(dx); free(dy); free(dz); free(sv); free(sd); free(t1); free(t2); free(t3);
  for (int k = 0; k < 4; k++) free(v[k]);
  for (int k = 0; k < 3; k++) free(tend[k]);
  free(dvor); free(ddiv); free(dh); free(darea); free(dep); free(nv); free(ntr);
}
