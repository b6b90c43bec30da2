// Host-side setup of the cubed-sphere tree: panel table, interpolation table,
// leaf points, interaction list and the RunConfig namelist reader.  These run
// once per problem on the CPU (as in the reference) and feed the device-side
// precomputation in context.cu.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <deque>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "geometry.cuh"
#include "internal.hpp"

namespace sbslpm {

namespace {

// gcdist: src/general_utils.cpp:43-46
double gcdist(const double* p1, const double* p2) {
  double dp = p1[0] * p2[0] + p1[1] * p2[1] + p1[2] * p2[2];
  dp = dp > 1.0 ? 1.0 : (dp < -1.0 ? -1.0 : dp);
  return std::acos(dp);
}

// sphere_tri_area (spherical excess by L'Huilier): src/general_utils.cpp:25-41
double sphere_tri_area(const double* p1, const double* p2, const double* p3) {
  double e1[3], e2[3], e3[3];
  for (int i = 0; i < 3; i++) {
    e1[i] = p2[i] - p3[i];  // side opposite p1
    e2[i] = p3[i] - p1[i];
    e3[i] = p1[i] - p2[i];
  }
  double a = std::acos(1 - 0.5 * (e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2]));
  double b = std::acos(1 - 0.5 * (e2[0] * e2[0] + e2[1] * e2[1] + e2[2] * e2[2]));
  double c = std::acos(1 - 0.5 * (e3[0] * e3[0] + e3[1] * e3[1] + e3[2] * e3[2]));
  double s = (a + b + c) / 2;
  double z = std::tan(s / 2) * std::tan((s - a) / 2) * std::tan((s - b) / 2) * std::tan((s - c) / 2);
  return 4 * std::atan(std::sqrt(z));
}

int* child_slot(sbslpm_panel& p, int c) {
  return c == 0 ? &p.child1 : c == 1 ? &p.child2 : c == 2 ? &p.child3 : &p.child4;
}

}  // namespace

int child_of(const sbslpm_panel& p, int c) {
  return c == 0 ? p.child1 : c == 1 ? p.child2 : c == 2 ? p.child3 : p.child4;
}

void build_panels(int levels, std::vector<sbslpm_panel>& P) {
  int n = 2 * ((1 << (2 * levels)) - 1);
  P.assign(n, sbslpm_panel{});
  // the six faces and their neighbours: src/initialize_cubed_sphere.cpp:187-220
  static const int edges[6][4] = {{4, 3, 5, 1}, {4, 0, 5, 2}, {4, 1, 5, 3}, {4, 2, 5, 0}, {2, 3, 0, 1}, {0, 3, 2, 1}};
  for (int f = 0; f < 6; f++) {
    sbslpm_panel& p = P[f];
    p.id = f;
    p.face = f;
    p.min_xi = p.min_eta = -1;
    p.max_xi = p.max_eta = 1;
    p.level = 0;
    p.parent_id = -1;
    p.id_top_edge = edges[f][0];
    p.id_left_edge = edges[f][1];
    p.id_bot_edge = edges[f][2];
    p.id_right_edge = edges[f][3];
  }
  // quadrisection, children in the order (+xi,+eta), (-xi,+eta), (-xi,-eta),
  // (+xi,-eta): refine_cube, src/initialize_cubed_sphere.cpp:64-141
  for (int lev = 0; lev + 1 < levels; lev++) {
    int ps = level_start(lev), cs = level_start(lev + 1), cnt = 6 * (1 << (2 * lev));
    for (int i = 0; i < cnt; i++) {
      sbslpm_panel& par = P[ps + i];
      int base = cs + 4 * i;
      double mx = 0.5 * (par.max_xi + par.min_xi), me = 0.5 * (par.max_eta + par.min_eta);
      double lo_xi[4] = {mx, par.min_xi, par.min_xi, mx}, hi_xi[4] = {par.max_xi, mx, mx, par.max_xi};
      double lo_eta[4] = {me, me, par.min_eta, par.min_eta}, hi_eta[4] = {par.max_eta, par.max_eta, me, me};
      int t = par.id_top_edge - ps, l = par.id_left_edge - ps, b = par.id_bot_edge - ps, r = par.id_right_edge - ps;
      int top[4] = {cs + 4 * t + 3, cs + 4 * t + 2, base + 1, base};
      int left[4] = {base + 1, cs + 4 * l, cs + 4 * l + 3, base + 2};
      int bot[4] = {base + 3, base + 2, cs + 4 * b + 1, cs + 4 * b};
      int right[4] = {cs + 4 * r + 1, base, base + 3, cs + 4 * r + 2};
      for (int c = 0; c < 4; c++) {
        sbslpm_panel& ch = P[base + c];
        ch.id = base + c;
        ch.face = par.face;
        ch.parent_id = ps + i;
        ch.level = par.level + 1;
        ch.min_xi = lo_xi[c];
        ch.max_xi = hi_xi[c];
        ch.min_eta = lo_eta[c];
        ch.max_eta = hi_eta[c];
        ch.id_top_edge = top[c];
        ch.id_left_edge = left[c];
        ch.id_bot_edge = bot[c];
        ch.id_right_edge = right[c];
        *child_slot(par, c) = base + c;
      }
    }
  }
  // leaf flag, radius and area: cubed_sphere_init_2, src/initialize_cubed_sphere.cpp:143-183
  for (int i = 0; i < n; i++) {
    sbslpm_panel& p = P[i];
    p.is_leaf = (p.level == levels - 1);
    double max_xi = p.max_xi * kPi / 4.0, min_xi = p.min_xi * kPi / 4.0;
    double max_eta = p.max_eta * kPi / 4.0, min_eta = p.min_eta * kPi / 4.0;
    double mid_xi = 0.5 * (max_xi + min_xi), mid_eta = 0.5 * (max_eta + min_eta);
    double c1[3], c2[3], c3[3], c4[3], cc[3];
    xyz_from_xieta(max_xi, max_eta, p.face, c1);
    xyz_from_xieta(max_xi, min_eta, p.face, c2);
    xyz_from_xieta(min_xi, min_eta, p.face, c3);
    xyz_from_xieta(min_xi, max_eta, p.face, c4);
    xyz_from_xieta(mid_xi, mid_eta, p.face, cc);
    double d1 = gcdist(c1, cc), d2 = gcdist(c2, cc), d3 = gcdist(c3, cc), d4 = gcdist(c4, cc);
    p.radius = std::fmax(d1, std::fmax(d2, std::fmax(d3, d4)));
    p.area = sphere_tri_area(c1, c2, c3) + sphere_tri_area(c1, c3, c4);
  }
}

// Chebyshev-extrema nodes, barycentric weights and Clenshaw-Curtis weights:
// interp_init, src/interp_funcs.cpp:11-73.  exact_cc replaces the reference's
// CC formula (which leaves the middle weight at zero for odd degree) by the
// exact weights w_i = (c_i/d)(1 - sum_j b_j cos(2 j theta_i)/(4j^2-1)).
void build_interp(int d, bool exact_cc, std::vector<double>& info) {
  int n = d + 1;
  std::vector<double> node(n), bw(n), cc(n, 0.0);
  for (int i = 0; i < n; i++) {
    if (d == 0) {
      node[i] = 0;
      bw[i] = 1;
      continue;
    }
    node[i] = std::cos(kPi / d * i);
    if (std::fabs(node[i]) < 1e-16) node[i] = 0;
    bw[i] = (i == 0) ? 0.5 : (i == d ? 0.5 * std::pow(-1, i) : std::pow(-1, i));
  }
  if (d == 0) {
    cc[0] = 2;
  } else if (!exact_cc) {
    int h = d / 2 + 1;
    std::vector<double> vec(h, 2.0);
    vec[0] = 1;
    for (int j = 1; j < h; j++) vec[j] = 2.0 / (1 - 4 * j * j);
    for (int i = 0; i < h; i++) {
      double s = 0;
      for (int j = 0; j < h; j++) s += 2 * std::cos(2 * i * j * kPi / d) / d * vec[j];
      cc[i] = s;
    }
    cc[0] *= 0.5;
    for (int i = 0; i < d / 2; i++) cc[d - i] = cc[i];
  } else {
    for (int i = 0; i < n; i++) {
      double th = kPi * i / d, s = 1.0;
      for (int j = 1; j <= d / 2; j++) s -= ((2 * j == d) ? 1.0 : 2.0) * std::cos(2 * j * th) / (4.0 * j * j - 1);
      cc[i] = ((i == 0 || i == d) ? 1.0 : 2.0) / d * s;
    }
  }
  info.assign((size_t)n * n * 4, 0.0);
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) {
      double* o = &info[4 * (size_t)(i * n + j)];
      o[0] = node[i];
      o[1] = node[j];
      o[2] = bw[i] * bw[j];
      o[3] = cc[i] * cc[j];
    }
}

// Breadth-first dual tree traversal: dual_tree_traversal, src/fmm_funcs.cpp:17-123.
// Same queue discipline, MAC and refinement rule, so the list (and its order)
// is the reference's.
void build_interactions(int levels, const std::vector<sbslpm_panel>& P, double theta,
                        std::vector<sbslpm_interact_pair>& out) {
  std::vector<char> near;
  build_interactions_flagged(levels, P, theta, out, near);
}

// The same traversal, also recording which pairs failed the MAC (near leaf
// pairs); the reference's type codes do not separate them from
// well-separated leaf pairs, both are type 0.
void build_interactions_flagged(int levels, const std::vector<sbslpm_panel>& P, double theta,
                                std::vector<sbslpm_interact_pair>& out, std::vector<char>& near) {
  out.clear();
  near.clear();
  std::deque<std::pair<int, int>> work;
  for (int t = 0; t < 6; t++)
    for (int s = 0; s < 6; s++) work.emplace_back(t, s);
  std::vector<std::array<double, 3>> centre(P.size());
  for (size_t i = 0; i < P.size(); i++) {
    const sbslpm_panel& p = P[i];
    double xi = kPi / 4.0 * 0.5 * (p.min_xi + p.max_xi), eta = kPi / 4.0 * 0.5 * (p.min_eta + p.max_eta);
    xyz_from_xieta(xi, eta, p.face, centre[i].data());
  }
  while (!work.empty()) {
    auto [t, s] = work.front();
    work.pop_front();
    const sbslpm_panel &pt = P[t], &ps = P[s];
    double dist = gcdist(centre[t].data(), centre[s].data());
    double sep = dist > 1e-16 ? (pt.radius + ps.radius) / dist : 100.0;
    if (sep < theta) {
      int type = (pt.level < levels - 1 ? 2 : 0) + (ps.level < levels - 1 ? 1 : 0);
      out.push_back({t, s, type});
      near.push_back(0);
    } else if (pt.is_leaf && ps.is_leaf) {
      out.push_back({t, s, 0});
      near.push_back(1);
    } else {
      bool split_target = !pt.is_leaf && (ps.is_leaf || pt.level <= ps.level);
      for (int c = 0; c < 4; c++)
        work.emplace_back(split_target ? child_of(pt, c) : t, split_target ? s : child_of(ps, c));
    }
  }
}

// Leaf points and quadrature areas: compute_point_panel,
// src/initialize_cubed_sphere.cpp:236-278.
void build_points(int levels, int d, const std::vector<sbslpm_panel>& P, const double* interp, double* x, double* y,
                  double* z, double* area) {
  int q = (d + 1) * (d + 1), off = level_start(levels - 1);
  for (size_t i = off; i < P.size(); i++) {
    const sbslpm_panel& p = P[i];
    double max_xi = kPi / 4.0 * p.max_xi, min_xi = kPi / 4.0 * p.min_xi;
    double max_eta = kPi / 4.0 * p.max_eta, min_eta = kPi / 4.0 * p.min_eta;
    double xr = 0.5 * (max_xi - min_xi), xo = 0.5 * (max_xi + min_xi);
    double er = 0.5 * (max_eta - min_eta), eo = 0.5 * (max_eta + min_eta);
    for (int j = 0; j < q; j++) {
      double xyz[3];
      xyz_from_xieta(xo + xr * interp[4 * j], eo + er * interp[4 * j + 1], p.face, xyz);
      size_t o = (i - off) * q + j;
      x[o] = xyz[0];
      y[o] = xyz[1];
      z[o] = xyz[2];
      area[o] = interp[4 * j + 3] * p.area / 4.0;
    }
  }
}

// The proxy point j of panel p as the interaction kernel places it
// (src/fmm_interactions/bve_vel_impl.hpp:90-108): node * half-width + centre.
void proxy_point(const sbslpm_panel& p, const double* interp, int j, double* xyz) {
  double xo = kPi / 4 * 0.5 * (p.max_xi + p.min_xi), xs = kPi / 4 * 0.5 * (p.max_xi - p.min_xi);
  double eo = kPi / 4 * 0.5 * (p.max_eta + p.min_eta), es = kPi / 4 * 0.5 * (p.max_eta - p.min_eta);
  xyz_from_xieta(interp[4 * j] * xs + xo, interp[4 * j + 1] * es + eo, p.face, xyz);
}

void host_bli(double* basis, double xi, double eta, double min_xi, double max_xi, double min_eta, double max_eta,
              int d, unsigned& err) {
  double cosv[kMaxDegree + 1], w[kMaxDegree + 1], fx[kMaxDegree + 1], fe[kMaxDegree + 1];
  for (int i = 0; i <= d; i++) {
    cosv[i] = d == 0 ? 0.0 : std::cos(kPi * i / d);
    w[i] = d == 0 ? 1.0 : (i == 0 ? 0.5 : (i == d ? 0.5 * std::pow(-1, i) : std::pow(-1, i)));
  }
  bli_1d(xi, min_xi, max_xi, d, cosv, w, fx, err);
  bli_1d(eta, min_eta, max_eta, d, cosv, w, fe, err);
  for (int i = 0; i <= d; i++)
    for (int j = 0; j <= d; j++) basis[i * (d + 1) + j] = fx[i] * fe[j];
}

// namelist reader: read_run_config, src/io_utils.cpp:11-92
bool read_namelist(const char* path, sbslpm_config* cfg, std::string& msg) {
  std::ifstream f(path);
  if (!f) {
    msg = std::string("namelist not found: ") + path;
    return false;
  }
  std::string line;
  bool forcing_on = cfg->forcing != SBSLPM_FORCING_NONE, stop = false;
  std::string forcing_type = cfg->forcing == SBSLPM_FORCING_SSW2 ? "ssw2" : "ssw";
  while (!stop && std::getline(f, line)) {
    std::stringstream ss(line);
    std::string key, val;
    std::getline(ss, key, '=');
    std::getline(ss, val);
    try {
      if (key == "levels") cfg->levels = std::stoi(val);
      else if (key == "interp_degree") cfg->interp_degree = std::min(std::stoi(val), kMaxDegree);
      else if (key == "theta") cfg->fmm_theta = std::stod(val);
      else if (key == "kernel_eps") cfg->kernel_eps = std::stod(val);
      else if (key == "omega") cfg->omega = std::stod(val);
      else if (key == "delta_t") cfg->dt = std::stoi(val);
      else if (key == "dt") cfg->dt = std::stod(val);
      else if (key == "tracers") {
        std::stringstream ts(val);
        std::string t;
        cfg->tracer_count = 0;
        while (std::getline(ts, t, ',')) cfg->tracer_count++;
      } else if (key == "velocity") cfg->velocity = (val == "direct") ? SBSLPM_VEL_DIRECT : SBSLPM_VEL_FMM;
      else if (key == "precision") cfg->precision = (val == "mixed") ? SBSLPM_MIXED : SBSLPM_FP64;
      else if (key == "exact_cc") cfg->exact_cc = std::stoi(val) != 0;
      else if (key == "proxy_degree") cfg->proxy_degree = std::stoi(val);
      else if (key == "leaf_size") cfg->leaf_size = std::stoi(val);
      else if (key == "g_over_a") cfg->g_over_a = std::stod(val);
      else if (key == "forcing") forcing_on = std::stoi(val) == 1;  // src/io_utils.cpp:69-72
      else if (key == "forcing_type") forcing_type = val;
      else if (key == "out_path" || key == "write_precision" || key == "write_output" || key == "grid_spacing" ||
               key == "end_time" || key == "output_vel" || key == "output_freq" || key == "initial_condition" ||
               key == "balance_ic" || key == "interp_output" || key == "topo_type") {
        // keys of the reference's drivers, not used on this path
      } else {
        stop = true;  // the reference stops at the first unknown key ("end")
      }
    } catch (const std::exception&) {
      msg = "bad value for namelist key '" + key + "': " + val;
      return false;
    }
  }
  // bve_forcing (src/forcing_funcs.cpp:82-96) knows the types "ssw" and "ssw2"
  if (!forcing_on) cfg->forcing = SBSLPM_FORCING_NONE;
  else if (forcing_type == "ssw") cfg->forcing = SBSLPM_FORCING_SSW;
  else if (forcing_type == "ssw2") cfg->forcing = SBSLPM_FORCING_SSW2;
  else {
    msg = "forcing_type must be ssw or ssw2, got '" + forcing_type + "'";
    return false;
  }
  return true;
}

}  // namespace sbslpm
