// Biot-Savart direct sum for callers that cannot allocate device memory.
//
// sbslpm_direct_sum_bve sums its source groups into a scratch buffer that it
// obtains from the stream-ordered allocator on every call.  Some callers
// cannot let a library allocate: a host model that fixes its whole device
// footprint when it starts, or one that owns all device memory through its
// own allocator, must not see cudaMalloc / cudaMallocAsync / cudaFree calls
// appear inside the time loop.  This variant keeps its scratch in a
// fixed-size array compiled into the library instead.  The array is
// allocated when the library's module is loaded on a GPU and stays until the
// process exits (kNoAllocScratchDoubles doubles = 16 MiB per GPU).
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/sbslpm.h"
#include "bve_kernels.cuh"
#include "internal.hpp"

namespace sbslpm {
namespace {

constexpr long kNoAllocScratchDoubles = 1L << 21;  // 16 MiB: partial sums of at most 699,050 targets
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];

// In host code g_noalloc_scratch names a host-side shadow, not device memory:
// the device address must come from cudaGetSymbolAddress, once per device,
// with that device current.  The result is cached per device, so a device
// must not be reset (cudaDeviceReset) while the library is in use: the
// module reloads after a reset and the array may move.
constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_addr[kMaxDevices] = {};

sbslpm_status scratch_for_current_device(double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    set_last_error(std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    return SBSLPM_ERR_CUDA;
  }
  if (dev < 0 || dev >= kMaxDevices) {
    set_last_error("device ordinal beyond the no-alloc entry point's table");
    return SBSLPM_ERR_ARG;
  }
  std::lock_guard<std::mutex> lock(g_mu);
  if (g_addr[dev] == nullptr) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) {
      set_last_error(std::string("cudaGetSymbolAddress(no-alloc scratch): ") + cudaGetErrorString(e));
      return SBSLPM_ERR_CUDA;
    }
    g_addr[dev] = static_cast<double*>(p);
  }
  *out = g_addr[dev];
  return SBSLPM_OK;
}

}  // namespace
}  // namespace sbslpm

using namespace sbslpm;

extern "C" sbslpm_status sbslpm_direct_sum_bve_noalloc(long nt, const double* tx, const double* ty, const double* tz,
                                                       long ns, const double* sx, const double* sy, const double* sz,
                                                       const double* s, double eps, int precision, double* ux,
                                                       double* uy, double* uz, void* stream) {
  if (nt < 0 || ns < 0) return set_last_error("sbslpm_direct_sum_bve_noalloc: negative size"), SBSLPM_ERR_ARG;
  if (precision != SBSLPM_FP64 && precision != SBSLPM_MIXED)
    return set_last_error("sbslpm_direct_sum_bve_noalloc: unknown precision"), SBSLPM_ERR_ARG;
  if ((nt > 0 && (!tx || !ty || !tz || !ux || !uy || !uz)) || (ns > 0 && (!sx || !sy || !sz || !s)))
    return set_last_error("sbslpm_direct_sum_bve_noalloc: null array"), SBSLPM_ERR_ARG;
  // a host array handed to the kernels would fault the caller's context
  if (any_on_host({tx, ty, tz, sx, sy, sz, s, ux, uy, uz}))
    return set_last_error("sbslpm_direct_sum_bve_noalloc: an array is host memory (device pointers expected)"),
           SBSLPM_ERR_ARG;
  if (3 * nt > kNoAllocScratchDoubles) {
    set_last_error("sbslpm_direct_sum_bve_noalloc: " + std::to_string(nt) + " targets exceed its fixed scratch (" +
                   std::to_string(kNoAllocScratchDoubles / 3) + " targets at most); use sbslpm_direct_sum_bve");
    return SBSLPM_ERR_ARG;
  }
  if (nt == 0) return SBSLPM_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t e;
  if (ns == 0) {
    double* outs[3] = {ux, uy, uz};
    for (double* o : outs)
      if ((e = cudaMemsetAsync(o, 0, sizeof(double) * nt, st)) != cudaSuccess) break;
  } else {
    double* partial = nullptr;
    sbslpm_status status = scratch_for_current_device(&partial);
    if (status != SBSLPM_OK) return status;
    // every (group, target) slot of the scratch is written before it is read,
    // so nothing left by an earlier call needs clearing.  When the target
    // count leaves room for fewer source groups than the allocating entry
    // point would use, the sums are split into fewer groups: the same sum in
    // another order.
    long groups = direct_groups(nt, ns);
    long fit = kNoAllocScratchDoubles / (3 * nt);
    if (groups > fit) groups = fit;
    launch_direct_bve(nt, tx, ty, tz, ns, sx, sy, sz, s, eps, precision, partial, (int)groups, ux, uy, uz, st);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    set_last_error(std::string("sbslpm_direct_sum_bve_noalloc: ") + cudaGetErrorString(e));
    return SBSLPM_ERR_CUDA;
  }
  return SBSLPM_OK;
}
