// Output path of the step drivers on the device: interpolation of a [leaf][q]
// field to a latitude-longitude grid (interp_to_latlon_host,
// src/interp_funcs.hpp:22-77, run on the host by the reference every output
// step) and the zonal / meridional velocity components (xyz_vel_to_uv_vel,
// src/general_utils_impl.hpp:195-229); the reference driver's output-grid rule
// (executables/bve_time_evo.cpp:93-95, 206-211).
#include <cuda_runtime.h>

#include <cmath>

#include "context_internal.hpp"
#include "device_common.cuh"

using namespace sbslpm;

namespace {

// One output point per thread: latitude lats[i], longitude lons[j] (degrees)
// to xyz, its leaf by tree descent (point_locate_panel_2,
// src/interp_funcs.cpp:175-203), the leaf's BLI basis at the point's (xi, eta)
// (xieta_from_xyz picks the same face as the descent) and the sum over the
// leaf's q values in m = i (d+1) + j order (src/interp_funcs.hpp:38-70).
template <int D>
__global__ void k_interp_latlon(StepGeom g, BliTable tab, const double* __restrict__ data,
                                const double* __restrict__ lats, int nlat, const double* __restrict__ lons, int nlon,
                                double* __restrict__ out) {
  const long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (idx >= (long)nlat * nlon) return;
  const int i = (int)(idx / nlon), j = (int)(idx % nlon);
  const double lat = lats[i] * kPi / 180.0, lon = lons[j] * kPi / 180.0;
  const double x = cos(lat) * cos(lon), y = cos(lat) * sin(lon), z = sin(lat);
  unsigned err = 0;
  dev::Basis<D> b;
  dev::locate_basis<D>(g, tab, x, y, z, b, err);
  out[idx] = dev::gather<D>(b, data);
  dev::flag(g.err, err);
}

// u = (-y vx + x vy) / sqrt(x^2 + y^2), v = -((x vx + y vy) z - (x^2 + y^2) vz)
// / sqrt(x^2 + y^2), both zero within 1e-16 of a pole.
__global__ void k_uv(long n, const double* __restrict__ x, const double* __restrict__ y,
                     const double* __restrict__ z, const double* __restrict__ vx, const double* __restrict__ vy,
                     const double* __restrict__ vz, double* __restrict__ u, double* __restrict__ v) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double xx = x[i], yy = y[i], zz = z[i], xc = vx[i], yc = vy[i], zc = vz[i];
  if (fabs(zz) < 1 - 1e-16) {
    u[i] = (-yy * xc + xx * yc) / sqrt(xx * xx + yy * yy);
    v[i] = -((xx * xc + yy * yc) * zz - (xx * xx + yy * yy) * zc) / sqrt(xx * xx + yy * yy);
  } else {
    u[i] = 0;
    v[i] = 0;
  }
}

bool bad(const void* p) { return p == nullptr; }

}  // namespace

extern "C" {

sbslpm_status sbslpm_interp_to_latlon(sbslpm_ctx* c, const double* data, int nlat, const double* lats, int nlon,
                                      const double* lons, double* out) {
  if (!c || nlat < 0 || nlon < 0 || (nlat > 0 && nlon > 0 && (bad(data) || bad(lats) || bad(lons) || bad(out))))
    return SBSLPM_ERR_ARG;
  const long n = (long)nlat * nlon;
  if (n == 0) return SBSLPM_OK;
  cudaStream_t st = c->stream();
  const unsigned grid = dev::blocks_for(n, 128);
#define SB_LL(D)                                                                                                   \
  case D:                                                                                                          \
    SB_LAUNCH(k_interp_latlon<D>, grid, 128, 0, st, c->geom, c->tab, data, lats, nlat, lons, nlon, out);          \
    break;
  switch (c->d) {
    SB_LL(0) SB_LL(1) SB_LL(2) SB_LL(3) SB_LL(4) SB_LL(5) SB_LL(6) SB_LL(7) SB_LL(8) SB_LL(9) SB_LL(10)
  }
#undef SB_LL
  return finish(c);
}

sbslpm_status sbslpm_xyz_vel_to_uv_vel(sbslpm_ctx* c, const double* x, const double* y, const double* z,
                                       const double* vel_x, const double* vel_y, const double* vel_z, double* vel_u,
                                       double* vel_v) {
  if (!c || bad(x) || bad(y) || bad(z) || bad(vel_x) || bad(vel_y) || bad(vel_z) || bad(vel_u) || bad(vel_v))
    return SBSLPM_ERR_ARG;
  const long n = (long)c->A * c->q;
  cudaStream_t st = c->stream();
  SB_LAUNCH(k_uv, dev::blocks_for(n, 256), 256, 0, st, n, x, y, z, vel_x, vel_y, vel_z, vel_u, vel_v);
  return finish(c);
}

sbslpm_status sbslpm_output_grid(long point_count, double* spacing, int* nlat, int* nlon, double* lats,
                                 double* lons) {
  if (point_count < 1 || !spacing || !nlat || !nlon) return SBSLPM_ERR_ARG;
  const double s = std::pow(2.0, std::floor(std::log2(std::sqrt(4 * kPi / (double)point_count) * 180.0 / kPi)));
  *spacing = s;
  *nlat = (int)(180.0 / s + 1.0);
  *nlon = (int)(360.0 / s);
  if (lats)
    for (int i = 0; i < *nlat; i++) lats[i] = -90.0 + s * i;
  if (lons)
    for (int i = 0; i < *nlon; i++) lons[i] = s * i;
  return SBSLPM_OK;
}

}  // extern "C"
