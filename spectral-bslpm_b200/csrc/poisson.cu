// Poisson (inverse Laplacian) FMM of executables/poisson_eq_fmm.cpp on the
// device: the reference's upward pass, poisson_fmm_interactions
// (src/fmm_interactions/inverse_poisson.cpp:9-34) and downward_pass
// (src/fmm_funcs.cpp:357-372), on a spectral-FMM context (proxy degree = the
// particle degree).  The kernel -1/(4 pi) log(1 - x.y) is the reference's,
// evaluated as it writes it (1 - x.y, pairs with x.y >= 1 - 1e-15 skipped), so
// the solve is u with -Laplacian(u) = f for mean-zero f.
#include <cuda_runtime.h>

#include "context_internal.hpp"
#include "device_common.cuh"

using namespace sbslpm;

namespace {

constexpr double kInvLapConst = -0.07957747154594767;  // -1/(4 pi), as the reference writes it

// poisson_panel_interaction (src/fmm_interactions/inverse_poisson_impl.hpp:22-52)
// owner-computes: one CTA per target panel, one thread per target proxy,
// the target's sources staged in shared memory in list order.
__global__ void __launch_bounds__(128)
    k_poisson_interact(StepGeom g, const double* __restrict__ src, double* __restrict__ tgt) {
  __shared__ double4 s[128];
  const int t = blockIdx.x, j = threadIdx.x, q = g.q;
  const long pn = (long)g.panels * q;
  double tx = 0, ty = 0, tz = 0;
  if (j < q) {
    const long o = (long)t * q + j;
    tx = g.px[o];
    ty = g.px[pn + o];
    tz = g.px[2 * pn + o];
  }
  double acc = 0;
  for (int e = g.tgt_start[t]; e < g.tgt_start[t + 1]; e++) {
    const long sb = (long)__ldg(g.src_panel + e) * q;
    if (j < q) s[j] = make_double4(g.px[sb + j], g.px[pn + sb + j], g.px[2 * pn + sb + j], src[sb + j]);
    __syncthreads();
    if (j < q)
      for (int k = 0; k < q; k++) {
        const double4 v = s[k];
        const double dp = tx * v.x + ty * v.y + tz * v.z;
        if (dp < 1.0 - 1e-15) acc += kInvLapConst * log(1 - dp) * v.w;
      }
    __syncthreads();
  }
  if (j < q) tgt[(long)t * q + j] += acc;
}

sbslpm_status need_spectral_fmm(const sbslpm_ctx* c) {
  if (c->tree || c->cfg.velocity != SBSLPM_VEL_FMM)
    return set_last_error("the reference's spectral FMM passes need proxy_degree 0 and FMM velocity"), SBSLPM_ERR_CONFIG;
  if (c->q > 128) return set_last_error("interp_degree above 10"), SBSLPM_ERR_CONFIG;
  return SBSLPM_OK;
}

bool bad(const void* p) { return p == nullptr; }

// downward_pass of one field through the three-field device pass: the
// field in component 0 of the context's proxy-target buffer, the other two
// components zero (their results are not used).
void downward_one(sbslpm_ctx* c, cudaStream_t st) {
  const size_t pn = (size_t)c->P * c->q;
  cudaMemsetAsync(c->tgt + pn, 0, sizeof(double) * 2 * pn, st);
  launch_downward_fused(c->geom, c->tgt, nullptr, st);
}

}  // namespace

extern "C" {

sbslpm_status sbslpm_poisson_fmm_interactions(sbslpm_ctx* c, const double* source, double* target) {
  if (!c || bad(source) || bad(target)) return SBSLPM_ERR_ARG;
  SB_TRY(need_spectral_fmm(c));
  cudaStream_t st = c->stream();
  SB_LAUNCH(k_poisson_interact, (unsigned)c->P, 128, 0, st, c->geom, source, target);
  return finish(c);
}

sbslpm_status sbslpm_downward_pass(sbslpm_ctx* c, double* proxy_target, double* soln) {
  if (!c || bad(proxy_target) || bad(soln)) return SBSLPM_ERR_ARG;
  SB_TRY(need_spectral_fmm(c));
  cudaStream_t st = c->stream();
  const size_t pn = (size_t)c->P * c->q, ln = (size_t)c->A * c->q, off = (size_t)c->off * c->q;
  SB_CUDA(cudaMemcpyAsync(c->tgt, proxy_target, sizeof(double) * pn, cudaMemcpyDeviceToDevice, st));
  downward_one(c, st);
  SB_CUDA(cudaMemcpyAsync(proxy_target, c->tgt, sizeof(double) * pn, cudaMemcpyDeviceToDevice, st));
  SB_CUDA(cudaMemcpyAsync(soln, c->tgt + off, sizeof(double) * ln, cudaMemcpyDeviceToDevice, st));
  return finish(c);
}

sbslpm_status sbslpm_poisson_fmm(sbslpm_ctx* c, const double* area, const double* pots, double* soln) {
  if (!c || bad(area) || bad(pots) || bad(soln)) return SBSLPM_ERR_ARG;
  SB_TRY(need_spectral_fmm(c));
  cudaStream_t st = c->stream();
  const size_t pn = (size_t)c->P * c->q, ln = (size_t)c->A * c->q, off = (size_t)c->off * c->q;
  // upward pass: proxy source weights into component 1 of the proxy-target buffer
  SB_CUDA(cudaMemsetAsync(c->src, 0, sizeof(double4) * pn, st));
  launch_upward_fused(c->geom, 1, 0, 0.0, nullptr, nullptr, nullptr, nullptr, pots, area, c->src, false, st);
  launch_copy_strength(c->geom, c->src, c->tgt + pn, st);
  SB_CUDA(cudaMemsetAsync(c->tgt, 0, sizeof(double) * pn, st));
  SB_LAUNCH(k_poisson_interact, (unsigned)c->P, 128, 0, st, c->geom, c->tgt + pn, c->tgt);
  downward_one(c, st);
  SB_CUDA(cudaMemcpyAsync(soln, c->tgt + off, sizeof(double) * ln, cudaMemcpyDeviceToDevice, st));
  return finish(c);
}

}  // extern "C"
