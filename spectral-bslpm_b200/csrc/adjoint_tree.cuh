// Adjoint of the decoupled-degree treecode velocity; adjoint_tree.cu.
#pragma once

#include <cuda_runtime.h>

#include "bve_kernels.cuh"

namespace sbslpm {

// Transposed interaction lists (device CSR): for each source leaf the target
// leaves whose near list holds it (relative leaf indices), for each source
// panel the target panels whose well-separated list holds it.
struct TreeAdjointLists {
  const int* near_tstart;
  const int* near_ttgt;
  const int* cc_tstart;
  const int* cc_ttgt;
};

// Given vbar [3][N] (adjoint of one stage velocity) and that stage's particle
// sources psrc (positions, strengths), writes qbar [N] and ybar [3][N], the
// adjoints of the particle source strengths and positions.  Scratch: tbar
// [3][tree panels * q], qbl [tree panels * q].  mixed: the transposed near
// and well-separated pair sums in float32 on packed coordinates (the
// forward's mixed arithmetic), everything else float64.
void launch_tree_velocity_adjoint(const TreeGeom& tg, const StepGeom& fg, const BliTable& ftab,
                                  const TreeAdjointLists& tl, const double* x, const double* y, const double* z,
                                  const double* vbar, const double4* psrc, double* tbar, double* qbl, double* qbar,
                                  double* ybar, bool mixed, cudaStream_t st);

// The reference's spectral FMM (proxy = particle degree; float64, or mixed:
// float32 transposed pairs on packed coordinates): given vbar
// [3][leaves*q] and the stage's sources src [panels*q] (displaced proxies,
// strengths), writes qbar [panels*q] (strength adjoints, leaves final after
// the strengths' transposed upward pass), ybar_leaf [3][leaves*q] and ybar_nl
// [3][offset*q] (position adjoints of leaf and non-leaf proxies).  tstart /
// ttgt: the interaction list transposed (target panels by source panel).
// Scratch: tbar [3][panels*q].
void launch_spectral_velocity_adjoint(const StepGeom& g, const int* tstart, const int* ttgt, const double* vbar,
                                      const double4* src, double* tbar, double* qbar, double* ybar_leaf,
                                      double* ybar_nl, bool mixed, cudaStream_t st);
// The non-leaf proxies' displacement interpolation reversed: vbar [3][leaves*q]
// += the adjoint of the previous stage's velocity through ybar_nl (atomics).
void launch_nonleaf_positions_adjoint(const StepGeom& g, double h, const double* vprev, const double* ybar_nl,
                                      double* vbar, cudaStream_t st);

}  // namespace sbslpm
