// Adjoint (vector-Jacobian product) kernels of the BVE step; adjoint.cu.
#pragma once

#include <cuda_runtime.h>

#include "bve_kernels.cuh"

namespace sbslpm {

// Groups of targets the Biot-Savart VJP splits its sum into.
int adjoint_groups(long n_targets, long n_sources);
// Biot-Savart sum u_i = K x_i x sum_j q_j (y_j - x_i)/(|y_j - x_i|^2/2 + eps):
// given ubar [3][nt] at the targets, qbar [ns] and ybar [3][ns] of the sources
// (src: (y, q) per source).  partial: groups x 4 x ns doubles.
void launch_bs_vjp(long nt, const double* tx, const double* ty, const double* tz, const double* ux,
                   const double* uy, const double* uz, long ns, const double4* src, double eps, double* partial,
                   int groups, double* qbar, double* ybar, cudaStream_t st);
// The same for the step's particles in mixed precision (targets x and sources
// src both the context's [leaf][q] particles; float32 pairs on coordinates
// packed relative to their leaves' centres; groups of target leaves).
void launch_bs_vjp_leaves32(const StepGeom& g, const double* tx, const double* ty, const double* tz,
                            const double* ux, const double* uy, const double* uz, const double4* src, double* partial,
                            int groups, double* qbar, double* ybar, cudaStream_t st);
void launch_pack_sources(long n, const double* x, const double* y, const double* z, const double* q, double4* s,
                         cudaStream_t st);
// Adjoint of a stage's leaf sources (strength a (w + 2 Omega z - 2 Omega y_z),
// position proj(x + h vprev)): wbar += a qbar; vbar_prev += h J^T ybar'.
void launch_src_adjoint(long n, int stage, double h, double omega, const double* vprev, const double* x,
                        const double* y, const double* z, const double* area, const double* qbar, const double* ybar,
                        double* wbar, double* vbar_prev, cudaStream_t st);
// Adjoint of the departure search and remap from wbar_new: wbar (scattered,
// must start at zero), vb0..vb2 (scattered, must start at zero), vb3 (written).
void launch_depart_remap_adjoint(const StepGeom& g, const BliTable& tab, const double* x, const double* y,
                                 const double* z, const double* v0, const double* v1, const double* v2,
                                 const double* v3, double dt, const double* w, const double* wbar_new, double* wbar,
                                 double* vb0, double* vb1, double* vb2, double* vb3, cudaStream_t st);

}  // namespace sbslpm
