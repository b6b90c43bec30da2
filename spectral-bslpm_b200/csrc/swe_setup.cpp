// Host-side set-up of the shallow-water step: the map from grid points to
// distinct positions (edge points shared by neighbouring panels), and the
// static per-panel tables of the finite-difference tendencies.  Every table
// entry is computed with the reference's own expressions, operand order and
// libm, once per context.
#include <cmath>
#include <cstdint>
#include <unordered_map>
#include <vector>

#include "geometry.cuh"
#include "internal.hpp"

namespace sbslpm {

namespace {

constexpr double kCell = 1e9;       // hash cells of 1e-9: far above the 1e-15 match tolerance,
constexpr double kEdge = 1e-3;      // far below the spacing of distinct grid points
constexpr double kMatchTol = 1e-15;  // src/initialize_cubed_sphere.cpp:305

struct Key {
  int64_t a, b, c;
  bool operator==(const Key& o) const { return a == o.a && b == o.b && c == o.c; }
};
struct KeyHash {
  size_t operator()(const Key& k) const {
    uint64_t h = (uint64_t)k.a * 0x9E3779B97F4A7C15ull;
    h ^= (uint64_t)k.b + 0x7F4A7C159E3779B9ull + (h << 6) + (h >> 2);
    h ^= (uint64_t)k.c + 0x94D049BB133111EBull + (h << 6) + (h >> 2);
    return (size_t)h;
  }
};

}  // namespace

// cubed_sphere_2d_to_1d (src/initialize_cubed_sphere.cpp:290-326): a point
// joins the first distinct position (in order of discovery) whose stored
// coordinates are all within 1e-15 of its own, else it starts a new one.  The
// reference scans every position found so far; here positions are bucketed in
// cells of 1e-9 and only the point's cell and, near a cell edge, the
// neighbouring cells are scanned, which finds the same first match.
long unique_points(long n_leaves, int q, const double* x, const double* y, const double* z, int* two_d_to_1d,
                   std::vector<int>& counts) {
  std::unordered_map<Key, std::vector<int>, KeyHash> cells;
  std::vector<double> ux, uy, uz;
  counts.clear();
  const long n = n_leaves * q;
  cells.reserve((size_t)n);
  for (long o = 0; o < n; o++) {
    const double p[3] = {x[o], y[o], z[o]};
    int64_t base[3];
    int lo[3], hi[3];
    for (int k = 0; k < 3; k++) {
      const double s = p[k] * kCell, f = std::floor(s);
      base[k] = (int64_t)f;
      lo[k] = (s - f) < kEdge ? -1 : 0;
      hi[k] = (s - f) > 1.0 - kEdge ? 1 : 0;
    }
    int best = -1;
    for (int da = lo[0]; da <= hi[0]; da++)
      for (int db = lo[1]; db <= hi[1]; db++)
        for (int dc = lo[2]; dc <= hi[2]; dc++) {
          auto it = cells.find(Key{base[0] + da, base[1] + db, base[2] + dc});
          if (it == cells.end()) continue;
          for (int u : it->second) {
            if (best >= 0 && u >= best) break;  // ids in a cell are increasing
            if (std::fabs(p[0] - ux[u]) < kMatchTol && std::fabs(p[1] - uy[u]) < kMatchTol &&
                std::fabs(p[2] - uz[u]) < kMatchTol) {
              best = u;
              break;
            }
          }
        }
    if (best < 0) {
      best = (int)ux.size();
      ux.push_back(p[0]);
      uy.push_back(p[1]);
      uz.push_back(p[2]);
      counts.push_back(0);
      cells[Key{base[0], base[1], base[2]}].push_back(best);
    }
    counts[best]++;
    two_d_to_1d[o] = best;
  }
  return (long)ux.size();
}

// Finite-difference weights along one direction of a panel with bounds
// [mn, mx] (fd_deriv_xi / fd_deriv_eta, src/deriv_funcs_impl.hpp:94-185):
// row 0 the one-sided end stencil, rows 1..d-1 the interior stencils, each
// (w0, w1, w2, h).
static void fd_weights(double mn, double mx, int degree, double* W) {
  const double scale = 0.5 * (mx - mn);
  const double offset = 0.5 * (mx + mn);
  {
    const double x0 = mx;
    const double x1 = std::cos(kPi / degree) * scale + offset;
    const double x2 = std::cos(kPi * 2.0 / degree) * scale + offset;
    const double h = x0 - x1;
    const double ratio = (x0 - x2) / (x0 - x1);
    W[0] = -1.0 - 1.0 / ratio;
    W[1] = ratio / (ratio - 1.0);
    W[2] = -1.0 / (ratio * ratio - ratio);
    W[3] = h;
  }
  for (int i = 1; i < degree; i++) {
    const double x0 = std::cos((i - 1) * kPi / degree) * scale + offset;
    const double x1 = std::cos(i * kPi / degree) * scale + offset;
    const double x2 = std::cos((i + 1) * kPi / degree) * scale + offset;
    const double d1 = x0 - x1, d2 = x1 - x2;
    const double h = std::fmin(d1, d2);
    const double ratio = std::fmax(d1 / h, d2 / h);
    double* w = W + 4 * i;
    if (d1 < d2) {
      w[0] = -ratio / (ratio + 1.0);
      w[1] = (ratio - 1.0) / ratio;
      w[2] = 1.0 / (ratio * ratio + ratio);
    } else {
      w[0] = -1.0 / (ratio * ratio + ratio);
      w[1] = (1.0 - ratio) / ratio;
      w[2] = ratio / (ratio + 1.0);
    }
    w[3] = h;
  }
  for (int k = 0; k < 4; k++) W[4 * degree + k] = W[k];  // the far end reuses the end stencil
}

void build_swe_tables(int degree, const std::vector<sbslpm_panel>& panels, int offset, long n_leaves,
                      const double* x, const double* y, const double* z, std::vector<double>& fd,
                      std::vector<double>& ntan, std::vector<double>& pow15, std::vector<double>& filt,
                      std::vector<double>& ptan, std::vector<int>& pface) {
  const int n1 = degree + 1, q = n1 * n1;
  fd.assign((size_t)n_leaves * 2 * n1 * 4, 0.0);
  ntan.assign((size_t)n_leaves * 2 * n1, 0.0);
  pow15.assign((size_t)n_leaves * q, 0.0);
  for (long a = 0; a < n_leaves; a++) {
    const sbslpm_panel& p = panels[offset + a];
    // swe_tendency_computation_2 passes the bounds scaled by pi/4 (src/swe_time_step_2_impl.hpp:41-44)
    const double min_xi = kPi / 4.0 * p.min_xi, max_xi = kPi / 4.0 * p.max_xi;
    const double min_eta = kPi / 4.0 * p.min_eta, max_eta = kPi / 4.0 * p.max_eta;
    fd_weights(min_xi, max_xi, degree, &fd[(size_t)a * 2 * n1 * 4]);
    fd_weights(min_eta, max_eta, degree, &fd[(size_t)a * 2 * n1 * 4 + n1 * 4]);
    // node coordinates of single_panel_lap_fd / _curl_rad_comp_fd / _div_fd
    // (src/deriv_funcs_impl.hpp:521-535, 601-612, 666-677)
    const double xs = 0.5 * (max_xi - min_xi), xo = 0.5 * (min_xi + max_xi);
    const double es = 0.5 * (max_eta - min_eta), eo = 0.5 * (min_eta + max_eta);
    double* nt = &ntan[(size_t)a * 2 * n1];
    for (int i = 0; i < n1; i++) {
      nt[i] = std::tan(std::cos(kPi * i / degree) * xs + xo);
      nt[n1 + i] = std::tan(std::cos(kPi * i / degree) * es + eo);
    }
    for (int i = 0; i < n1; i++)
      for (int j = 0; j < n1; j++) {
        const double X = nt[i], Y = nt[n1 + j];
        const double delta = 1 + X * X + Y * Y;
        pow15[(size_t)a * q + i * n1 + j] = std::pow(delta, 1.5);
      }
  }
  // spatial_filter_vals neighbour weights (src/deriv_funcs_impl.hpp:391-441)
  const double coeff = 0.0005;
  filt.assign((size_t)2 * n1, 0.0);
  for (int i = 0; i < n1; i++) {
    const double xi = std::cos(kPi * i / degree);
    double d1, d2;
    if (i == 0) {
      d1 = std::fabs(xi - std::cos(kPi * (i + 1) / degree));
      d2 = std::fabs(xi - std::cos(kPi * (i + 2) / degree));
    } else if (i == degree) {
      d1 = std::fabs(xi - std::cos(kPi * (i - 1) / degree));
      d2 = std::fabs(xi - std::cos(kPi * (i - 2) / degree));
    } else {
      d1 = std::fabs(xi - std::cos(kPi * (i - 1) / degree));
      d2 = std::fabs(xi - std::cos(kPi * (i + 1) / degree));
    }
    filt[2 * i] = 0.25 * coeff / (d1 + d2) * d1;
    filt[2 * i + 1] = 0.25 * coeff / (d1 + d2) * d2;
  }
  // each grid point's own tan(xi), tan(eta) and face, as xietavec_from_xyzvec
  // derives them from its coordinates (src/cubed_sphere_transforms_impl.hpp:245-253)
  const long n = n_leaves * q;
  ptan.assign((size_t)2 * n, 0.0);
  pface.assign((size_t)n, 0);
  for (long o = 0; o < n; o++) {
    const int face = face_from_xyz(x[o], y[o], z[o]);
    double xi, eta;
    xieta_from_xyz_face(x[o], y[o], z[o], face, xi, eta);
    ptan[2 * o] = std::tan(xi);
    ptan[2 * o + 1] = std::tan(eta);
    pface[o] = face;
  }
}

}  // namespace sbslpm
