// Host-side set-up of the treecode with decoupled proxy degree, shared by the
// single-problem context and the batched ensemble: the particle grid's
// quadtree truncated so that a leaf holds at most leaf_size particles, degree-n
// Chebyshev proxies on every tree panel, the leaf-box 1-D bases of the
// particle grid, and the near / well-separated interaction lists.
#include <cmath>
#include <vector>

#include "context_internal.hpp"
#include "geometry.cuh"

namespace sbslpm {

// One-dimensional BLI basis of the parent's degree-d nodes at the nodes of a
// child in the upper (h = 0) or lower (h = 1) half of the parent, computed on
// face 0 as child_to_parent places the child nodes
// (src/fmm_funcs_impl.hpp:53-64).  out: [2][d+1][d+1].
void child_basis_1d(const std::vector<sbslpm_panel>& P, const BliTable& tab, int d, std::vector<double>& out,
                    unsigned& err) {
  const int n1 = d + 1;
  out.assign((size_t)2 * n1 * n1, 0.0);
  const sbslpm_panel& par = P[0];
  const double lo = par.min_xi * kPi / 4.0, hi = par.max_xi * kPi / 4.0;
  for (int h = 0; h < 2; h++) {
    const sbslpm_panel& ch = P[child_of(par, h == 0 ? 0 : 2)];  // child 0: upper half; child 2: lower half
    const double xo = kPi / 4.0 * 0.5 * (ch.min_xi + ch.max_xi), xs = kPi / 4.0 * 0.5 * (ch.max_xi - ch.min_xi);
    for (int i = 0; i < n1; i++) {
      double node = d == 0 ? 0.0 : std::cos(kPi / d * i);
      if (std::fabs(node) < 1e-16) node = 0;
      bli_1d(node * xs + xo, lo, hi, d, tab.cosv, tab.w, &out[((size_t)h * n1 + i) * n1], err);
    }
  }
}

void bli_table(int n, BliTable& t) {
  for (int i = 0; i <= n; i++) {
    t.cosv[i] = n == 0 ? 0.0 : std::cos(kPi * i / n);
    t.w[i] = n == 0 ? 1.0 : (i == 0 ? 0.5 : (i == n ? 0.5 * std::pow(-1, i) : std::pow(-1, i)));
  }
}

sbslpm_status build_tree_tables(int L, int d, const std::vector<sbslpm_panel>& grid, int leaf_size, int n,
                                TreeTables& t) {
  const int qp = (d + 1) * (d + 1), n1 = n + 1;
  int m = 0;
  long npl = qp;
  while (npl * 4 <= leaf_size && m < L - 1) {
    npl *= 4;
    m++;
  }
  t.n = n;
  t.qx = n1 * n1;
  t.npl = (int)npl;
  t.Lf = L - m;
  t.Pf = sbslpm_panel_count(t.Lf);
  t.Af = sbslpm_leaf_count(t.Lf);
  build_panels(t.Lf, t.fpanels);
  const int Pf = t.Pf, offf = t.Pf - t.Af, qx = t.qx;
  std::vector<double> interp_n;
  build_interp(n, false, interp_n);
  t.fpx.assign((size_t)3 * Pf * qx, 0.0);
  t.centre.assign((size_t)4 * Pf, 0.0);
  t.bounds.assign((size_t)4 * Pf, 0.0);
  t.face.assign(Pf, 0);
  const size_t pn = (size_t)Pf * qx;
  for (int p = 0; p < Pf; p++) {
    const sbslpm_panel& pp = t.fpanels[p];
    for (int j = 0; j < qx; j++) {
      double xyz[3];
      proxy_point(pp, interp_n.data(), j, xyz);
      for (int k = 0; k < 3; k++) t.fpx[k * pn + (size_t)p * qx + j] = xyz[k];
    }
    double xyz[3];
    xyz_from_xieta(kPi / 4.0 * 0.5 * (pp.min_xi + pp.max_xi), kPi / 4.0 * 0.5 * (pp.min_eta + pp.max_eta), pp.face,
                   xyz);
    for (int k = 0; k < 3; k++) t.centre[4 * (size_t)p + k] = xyz[k];
    t.bounds[4 * p + 0] = kPi / 4.0 * pp.min_xi;
    t.bounds[4 * p + 1] = kPi / 4.0 * pp.max_xi;
    t.bounds[4 * p + 2] = kPi / 4.0 * pp.min_eta;
    t.bounds[4 * p + 3] = kPi / 4.0 * pp.max_eta;
    t.face[p] = pp.face;
  }
  bli_table(n, t.ftab);
  unsigned err = 0;
  t.c1d.clear();
  if (t.Lf > 1) child_basis_1d(t.fpanels, t.ftab, n, t.c1d, err);

  // leaf-box basis of the particles of the first tree leaf (the same for every leaf)
  std::vector<double> interp_p;
  build_interp(d, false, interp_p);
  t.lx.assign((size_t)npl * n1, 0.0);
  t.ly.assign((size_t)npl * n1, 0.0);
  const sbslpm_panel& leaf = t.fpanels[offf];
  const double lo_x = kPi / 4.0 * leaf.min_xi, hi_x = kPi / 4.0 * leaf.max_xi;
  const double lo_e = kPi / 4.0 * leaf.min_eta, hi_e = kPi / 4.0 * leaf.max_eta;
  const int first_dp = level_start(L - 1);  // the first leaf's descendants come first
  for (long k = 0; k < npl; k++) {
    const sbslpm_panel& dp = grid[first_dp + k / qp];
    const int j = (int)(k % qp);
    double max_xi = kPi / 4.0 * dp.max_xi, min_xi = kPi / 4.0 * dp.min_xi;
    double max_eta = kPi / 4.0 * dp.max_eta, min_eta = kPi / 4.0 * dp.min_eta;
    double xi = 0.5 * (max_xi + min_xi) + 0.5 * (max_xi - min_xi) * interp_p[4 * j];
    double eta = 0.5 * (max_eta + min_eta) + 0.5 * (max_eta - min_eta) * interp_p[4 * j + 1];
    bli_1d(xi, lo_x, hi_x, n, t.ftab.cosv, t.ftab.w, &t.lx[k * n1], err);
    bli_1d(eta, lo_e, hi_e, n, t.ftab.cosv, t.ftab.w, &t.ly[k * n1], err);
  }
  if (err) {
    set_last_error("treecode set-up: a particle fell outside its leaf");
    return SBSLPM_ERR_OUT_OF_PANEL;
  }
  return SBSLPM_OK;
}

// Near leaf pairs (particle x particle, CSR by target leaf, sources relative
// to the first leaf) and well-separated pairs (proxy x proxy, CSR by target
// panel), each in traversal order within a target.
void build_tree_lists(const TreeTables& t, double theta, TreeLists& l) {
  std::vector<sbslpm_interact_pair> list;
  std::vector<char> near;
  build_interactions_flagged(t.Lf, t.fpanels, theta, list, near);
  tree_lists_from(t, std::move(list), near, l);
}

sbslpm_status device_tree_lists(const TreeTables& t, const std::vector<double>& theta, std::vector<TreeLists>& out,
                                cudaStream_t st) {
  std::vector<std::vector<sbslpm_interact_pair>> lists;
  std::vector<std::vector<char>> near;
  SB_TRY(device_dual_tree_traversal_multi(t.Lf, t.fpanels, theta, lists, &near, st));
  out.resize(theta.size());
  for (size_t m = 0; m < theta.size(); m++) tree_lists_from(t, std::move(lists[m]), near[m], out[m]);
  return SBSLPM_OK;
}

void tree_lists_from(const TreeTables& t, std::vector<sbslpm_interact_pair>&& list, const std::vector<char>& near,
                     TreeLists& l) {
  const int Pf = t.Pf, Af = t.Af, offf = Pf - Af;
  l.list = std::move(list);
  l.ns.assign(Af + 1, 0);
  l.cs.assign(Pf + 1, 0);
  for (size_t e = 0; e < l.list.size(); e++) {
    if (near[e]) l.ns[l.list[e].target_panel - offf + 1]++;
    else l.cs[l.list[e].target_panel + 1]++;
  }
  for (int i = 0; i < Af; i++) l.ns[i + 1] += l.ns[i];
  for (int i = 0; i < Pf; i++) l.cs[i + 1] += l.cs[i];
  l.nsrc.assign(l.ns[Af], 0);
  l.csrc.assign(l.cs[Pf], 0);
  std::vector<int> nf(l.ns.begin(), l.ns.end() - 1), cf(l.cs.begin(), l.cs.end() - 1);
  for (size_t e = 0; e < l.list.size(); e++) {
    if (near[e]) l.nsrc[nf[l.list[e].target_panel - offf]++] = l.list[e].source_panel - offf;
    else l.csrc[cf[l.list[e].target_panel]++] = l.list[e].source_panel;
  }
}

// Whether the mixed near field may evaluate its pairs in the expanded form
// (pair32x2_expanded).  That form rounds the denominator |b + s|^2 + eps to
// about 3u (|b| + |s|)^2 (u = 2^-24) where the difference form rounds it
// relative to |b + s|, so it is chosen only where that rounding stays below
// 2^-10 of eps for every near pair: eps >= 3 u 2^10 M with M the largest
// (|c_S - c_T| + 2 r_T + 2 r_S)^2 / 2 over the near leaf pairs (packed
// coordinates carry the factor 1/sqrt(2); twice the leaf radii leave room for
// the displaced sources of the later RK stages).  eps = 0 needs the
// difference form (its coincident pairs are skipped by a test of the
// denominator).
bool near_expanded_ok(const TreeTables& t, const TreeLists& l, double eps) {
  if (!(eps > 0)) return false;
  const int offf = t.Pf - t.Af;
  double m = 0;
  for (int T = 0; T < t.Af; T++)
    for (int e = l.ns[T]; e < l.ns[T + 1]; e++) {
      const int S = l.nsrc[e];
      const double* a = &t.centre[4 * (size_t)(offf + T)];
      const double* b = &t.centre[4 * (size_t)(offf + S)];
      const double dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
      const double r = std::sqrt(dx * dx + dy * dy + dz * dz) +
                       2.0 * (t.fpanels[offf + T].radius + t.fpanels[offf + S].radius);
      m = std::fmax(m, 0.5 * r * r);
    }
  return eps >= 3.0 * std::ldexp(1.0, -14) * m;
}

// Units of the first stage's two-sided near-field kernel from the near lists
// (CSR by target leaf): (T, S, e, e') for every entry e = (T <- S) with S > T
// whose mirror e' = (S <- T) is in S's list, (T, S, e, -1) for the diagonal
// entries and for entries without a mirror (evaluated one-sidedly).
void build_mutual_units(const std::vector<int>& ns, const std::vector<int>& nsrc, std::vector<int4>& units) {
  units.clear();
  const int leaves = (int)ns.size() - 1;
  for (int T = 0; T < leaves; T++)
    for (int e = ns[T]; e < ns[T + 1]; e++) {
      const int S = nsrc[e];
      int mirror = -1;
      if (S != T)
        for (int f = ns[S]; f < ns[S + 1]; f++)
          if (nsrc[f] == T) mirror = f;
      if (S == T || mirror < 0) units.push_back(make_int4(T, S, e, -1));
      else if (S > T) units.push_back(make_int4(T, S, e, mirror));
    }
}

}  // namespace sbslpm
