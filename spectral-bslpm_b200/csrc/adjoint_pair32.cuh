// Device helpers of the mixed-precision adjoint pair sums (adjoint.cu,
// adjoint_tree.cu).
#pragma once

#include <cuda_runtime.h>

#include "bve_kernels.cuh"
#include "device_common.cuh"

namespace sbslpm {
namespace dev {

// Mixed precision (float32 pairs on packed coordinates, as the forward
// kernels): d' = (y - x) kPackScale = a - x', a = y' + (c_S - c_T) kPackScale
// with y', x' relative to the source and target panels' centres, so
// |d'|^2 + eps = |d|^2/2 + eps and, with g = 1/(|d'|^2 + eps),
//   qbar = K sqrt2 sum g (c.d'),   ybar = K q sum [g c - 2 g^2 (c.d') d'].
// One source against two targets per instruction (paired FP32): A = (-x0, -x1,
// -y0, -y1), B = (-z0, -z1, cx0, cx1), C = (cy0, cy1, cz0, cz1) of the two
// targets; u = g (c.d') feeds q, g c feeds bc and u g d' feeds bd.
template <bool GUARD>
__device__ __forceinline__ void adj_pair32x2(const float2 ax, const float2 ay, const float2 az, const float4 A,
                                             const float4 B, const float4 C, const float2 eps2, float2& q,
                                             float2& bcx, float2& bcy, float2& bcz, float2& bdx, float2& bdy,
                                             float2& bdz) {
  const float2 dx = __fadd2_rn(ax, make_float2(A.x, A.y)), dy = __fadd2_rn(ay, make_float2(A.z, A.w)),
               dz = __fadd2_rn(az, make_float2(B.x, B.y));
  const float2 den = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __ffma2_rn(dz, dz, eps2)));
  float2 g = make_float2(recip_f32(den.x), recip_f32(den.y));
  if (GUARD) {
    g.x = den.x > 0.0f ? g.x : 0.0f;
    g.y = den.y > 0.0f ? g.y : 0.0f;
  }
  const float2 cx = make_float2(B.z, B.w), cy = make_float2(C.x, C.y), cz = make_float2(C.z, C.w);
  const float2 cd = __ffma2_rn(cx, dx, __ffma2_rn(cy, dy, __fmul2_rn(cz, dz)));
  const float2 u = __fmul2_rn(g, cd);
  q = __fadd2_rn(q, u);
  const float2 ug = __fmul2_rn(u, g);
  bcx = __ffma2_rn(g, cx, bcx);
  bcy = __ffma2_rn(g, cy, bcy);
  bcz = __ffma2_rn(g, cz, bcz);
  bdx = __ffma2_rn(ug, dx, bdx);
  bdy = __ffma2_rn(ug, dy, bdy);
  bdz = __ffma2_rn(ug, dz, bdz);
}

// Stages target k of a tile as half of a pair slot (see adj_pair32x2): its
// packed position relative to the target panel's centre ct, negated, and
// c = w x x (w: the adjoint three-vector at the target, x: its position).
__device__ __forceinline__ void adj_stage(float4* tile, int k, double x, double y, double z, double wa, double wb,
                                          double wc, const double* ct) {
  float* A = reinterpret_cast<float*>(tile + 3 * (k >> 1));
  const int h = k & 1;
  A[h] = (float)((ct[0] - x) * kPackScale);
  A[2 + h] = (float)((ct[1] - y) * kPackScale);
  A[4 + h] = (float)((ct[2] - z) * kPackScale);
  A[6 + h] = (float)(wb * z - wc * y);
  A[8 + h] = (float)(wc * x - wa * z);
  A[10 + h] = (float)(wa * y - wb * x);
}

// The zero partner of an odd target count: c = 0 contributes nothing.
__device__ __forceinline__ void adj_stage_zero(float4* tile, int k) {
  float* A = reinterpret_cast<float*>(tile + 3 * (k >> 1));
  const int h = k & 1;
  for (int m = 0; m < 6; m++) A[2 * m + h] = 0.0f;
}

}  // namespace dev
}  // namespace sbslpm
