// Device kernels of the shallow-water (SWE v2) step, sm_100a.  Launch
// wrappers are in swe_kernels.cu (sources, interactions) and swe_fd.cu
// (finite-difference tendencies, edge unification, arrival values); the step
// orchestration is in context.cu.
#pragma once

#include <cuda_runtime.h>

#include "bve_kernels.cuh"

namespace sbslpm {

// Static SWE geometry of the leaf panels, built on the host once per context.
struct SweGeom {
  double g_over_a;        // scale of the height Laplacian (9.81/6371000 in the reference)
  long unique;            // distinct grid points (edge points shared by panels count once)
  const double* fd;       // [leaves][2][d+1][4]: finite-difference weights w0, w1, w2, h along xi (0) and eta (1);
                          // row 0 = one-sided end stencil, rows 1..d-1 = interior stencils
  const double* ntan;     // [leaves][2][d+1]: tan of the panel's node xi / eta
  const double* pow15;    // [leaves][q]: (1 + X^2 + Y^2)^1.5 at the panel nodes
  const double* filt;     // [d+1][2]: spatial-filter neighbour weights (same along xi and eta)
  const double* ptan;     // [leaves*q][2]: tan(xi), tan(eta) of each grid point's own position
  const int* pface;       // [leaves*q]: cube face of each grid point
  const int* ustart;      // [unique+1]: CSR of the grid points sharing one position, in [leaf][q] order
  const int* umem;        // [leaves*q]
  float4* srcf2;          // mixed: packed divergence sources [panels*q] (workspace)
};

// Sources of one velocity evaluation and the upward pass, both source fields
// (vorticity at displaced positions, divergence at the fixed proxies).
//   stage 0: strengths area*vor, area*div, no displacement
//   stage s: displacement dtd*vprev; vor + dts*tprev_vor, div + dts*tprev_div,
//            area*(1 + dts*div) (swe_apply_tendencies_2)
void launch_swe_upward(const StepGeom& g, const SweGeom& s, int stage, double dtd, double dts, const double* vprev,
                       const double* tprev, const double* x, const double* y, const double* z, const double* vors,
                       const double* divs, const double* area, double4* src, double4* src2, bool mixed,
                       cudaStream_t st);
// Direct velocity: leaf sources only (both fields).
void launch_swe_leaf_sources(const StepGeom& g, const SweGeom& s, int stage, double dtd, double dts,
                             const double* vprev, const double* tprev, const double* vors, const double* divs,
                             const double* area, double4* src, double4* src2, bool mixed, cudaStream_t st);
// Proxy-target velocities of both source fields over the interaction list
// (swe_vel_panel_interaction_2); tgt = 3 x panels*q, written.
void launch_swe_interactions(const StepGeom& g, const SweGeom& s, int precision, const double4* src,
                             const double4* src2, double* tgt, cudaStream_t st);
// Every leaf against every leaf (direct velocity), partials reduced in order.
void launch_swe_direct(const StepGeom& g, const SweGeom& s, int precision, const double4* src, const double4* src2,
                       double* vout, double* partial, int groups, cudaStream_t st);
// Piecewise API: sources from explicit displacements and strengths.
void launch_swe_sources_from_disp(const StepGeom& g, const SweGeom& s, const double* dx, const double* dy,
                                  const double* dz, const double* s_vor, const double* s_div, double4* src,
                                  double4* src2, bool mixed, cudaStream_t st);

// swe_tendency_computation_2 (+ modify_tendencies when base_div / base_h are
// given).  height used = h + dts*tprev_h when tprev is given (disp_heights).
// vel = 3 x leaves*q; tend = 3 x leaves*q (vor, div, h).
void launch_swe_tendency(const StepGeom& g, const SweGeom& s, const double* x, const double* y, const double* z,
                         const double* vel, const double* vors, const double* divs, const double* height,
                         const double* surface, double dts, const double* tprev, const double* base_div,
                         const double* base_h, double* tend, cudaStream_t st);
// unify_boundary_vals on up to three fields (null fields are skipped), rounds
// times in a row.
void launch_unify(const SweGeom& s, double* f0, double* f1, double* f2, int rounds, cudaStream_t st);
// Forward-Euler arrival values (swe_compute_arrival_values_2): avor = vor +
// dt*tend_vor; divs and height updated in place.
void launch_swe_arrival(const StepGeom& g, const double* tend1, double dt, const double* vors, double* divs,
                        double* height, double* avor, cudaStream_t st);

// Treecode velocity of the SWE step (bltc_swe.cu).  Leaf sources of both
// fields and their anterpolation onto the tree leaves' proxies (proxy: the
// vorticity proxies' .w, proxy2: the divergence proxies' .w): step mode from
// (stage, dtd, dts, vprev, tprev, vors, divs, area) as launch_swe_upward, or,
// with dispx/dispy/dispz, positions x + disp and strengths wv / wd given.
void launch_bltc_swe_sources(const TreeGeom& tg, const StepGeom& fg, const BliTable& tab, int stage, double dtd,
                             double dts, const double* vprev, const double* tprev, const double* x, const double* y,
                             const double* z, const double* vors, const double* divs, const double* area,
                             const double* dispx, const double* dispy, const double* dispz, const double* wv,
                             const double* wd, double4* psrc, float4* psrcf, double4* psrc2, float4* psrcf2,
                             double4* proxy, double4* proxy2, bool mixed, const double* gcentre, int gq,
                             cudaStream_t st);
// Near leaf pairs of both fields into splits x 3 x N velocity partials
// (leaves of at most 256 particles).  gcentre: the grid leaves' centres
// ([grid leaves][4], gq particles each): mixed precision packs the particle
// sources relative to them.
void launch_bltc_swe_near(const TreeGeom& tg, const StepGeom& fg, int precision, const double* x, const double* y,
                          const double* z, const double4* psrc, const double4* psrc2, const float4* psrcf,
                          const float4* psrcf2, double* near, int splits, const double* gcentre, int gq,
                          cudaStream_t st);

// Well-separated pairs of both fields on the treecode, mixed precision, over
// the chunks of the interaction list (cstart: a target panel's first chunk;
// partial: [chunks][6][q] float64) into tgt (3 x panels*q); proxy counts
// with swe_tree_cc_supported only.
bool swe_tree_cc_supported(int q);
void launch_swe_tree_cc(const StepGeom& fg, const float4* srcf2, const int4* chunks, int nchunks, const int* cstart,
                        double* partial, double* tgt, cudaStream_t st);

}  // namespace sbslpm
