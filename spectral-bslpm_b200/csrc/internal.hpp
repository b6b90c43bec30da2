// Internal declarations shared by the host setup code, the kernels and the
// C ABI implementation.
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <array>
#include <initializer_list>
#include <string>
#include <vector>

#include "../../include/sbslpm.h"

namespace sbslpm {

// An NVTX range over a scope of host code (the enqueueing of a step's
// phases): profilers show the stages on the CPU timeline and correlate them
// with their kernels; without a profiler attached a range costs a branch.
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

// True when any non-null pointer is host memory: the entry points that take
// device pointers reject those arguments instead of handing them to kernels.
inline bool any_on_host(std::initializer_list<const void*> ps) {
  for (const void* p : ps)
    if (p && sbslpm_pointer_on_device(p) == 0) return true;
  return false;
}

// setup_host.cpp
int child_of(const sbslpm_panel& p, int c);
void build_panels(int levels, std::vector<sbslpm_panel>& panels);
void build_interp(int degree, bool exact_cc, std::vector<double>& info);
void build_interactions(int levels, const std::vector<sbslpm_panel>& panels, double theta,
                        std::vector<sbslpm_interact_pair>& out);
void build_interactions_flagged(int levels, const std::vector<sbslpm_panel>& panels, double theta,
                                std::vector<sbslpm_interact_pair>& out, std::vector<char>& near);
void build_points(int levels, int degree, const std::vector<sbslpm_panel>& panels, const double* interp, double* x,
                  double* y, double* z, double* area);
void proxy_point(const sbslpm_panel& p, const double* interp, int j, double* xyz);
void host_bli(double* basis, double xi, double eta, double min_xi, double max_xi, double min_eta, double max_eta,
              int degree, unsigned& err);
bool read_namelist(const char* path, sbslpm_config* cfg, std::string& msg);

// swe_setup.cpp
long unique_points(long n_leaves, int q, const double* x, const double* y, const double* z, int* two_d_to_1d,
                   std::vector<int>& counts);
void build_swe_tables(int degree, const std::vector<sbslpm_panel>& panels, int offset, long n_leaves,
                      const double* x, const double* y, const double* z, std::vector<double>& fd,
                      std::vector<double>& ntan, std::vector<double>& pow15, std::vector<double>& filt,
                      std::vector<double>& ptan, std::vector<int>& pface);

void set_last_error(const std::string& msg);

// OK when the current device is `device` (the one a context or batch was
// created on, which owns its buffers and streams); otherwise an argument
// error naming both, so that no kernel is launched on another GPU with this
// device's memory.
inline sbslpm_status on_device(int device, const char* what) {
  int cur = -1;
  if (cudaGetDevice(&cur) != cudaSuccess) return set_last_error("cudaGetDevice failed"), SBSLPM_ERR_CUDA;
  if (cur == device) return SBSLPM_OK;
  set_last_error(std::string(what) + " was created on device " + std::to_string(device) + " but device " +
                 std::to_string(cur) + " is current: make its device current (cudaSetDevice) first");
  return SBSLPM_ERR_ARG;
}

// traversal.cu: dual_tree_traversal on the device (same list, same order as build_interactions);
// the multi form runs one traversal per theta in one launch series and, with
// near, records per pair whether it failed the MAC (build_interactions_flagged)
sbslpm_status device_dual_tree_traversal(int levels, const std::vector<sbslpm_panel>& P, double theta,
                                         std::vector<sbslpm_interact_pair>& out, cudaStream_t st);
sbslpm_status device_dual_tree_traversal_multi(int levels, const std::vector<sbslpm_panel>& P,
                                               const std::vector<double>& theta,
                                               std::vector<std::vector<sbslpm_interact_pair>>& out,
                                               std::vector<std::vector<char>>* near, cudaStream_t st);

}  // namespace sbslpm
