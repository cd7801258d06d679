// Box average of a regular latitude-longitude field onto scattered points (cells or edges):
// the ERA5 initialisation of the reference drivers (src/grid2mpas.f90:21-70, called through
// era2mpas in src/mpas_sw_driver.py:147-158).
//
// For each point: the nearest grid latitude and longitude (first minimum of |difference|, as
// Fortran's minloc), the block of up to 3 x 3 grid values around them (clamped at the array
// ends, no wrap in longitude), and their mean, summed latitude-fastest within each longitude
// (the element order of the Fortran section sum).  One thread per point; the two 1-D axes are
// staged in shared memory when they fit.  Built without FMA contraction, so every sum and the
// final division round as on the host.
#include <cuda_runtime.h>

#include "mpsw.h"
#include "mpsw_engine.h"
#include "mpsw_launch.cuh"

namespace mpsw {
namespace {

// first index of the minimum of |a[i] - x| over i < n
__device__ __forceinline__ int nearest(const double *a, int n, double x) {
  int best = 0;
  double bd = fabs(x - a[0]);
  for (int i = 1; i < n; i++) {
    const double d = fabs(x - a[i]);
    if (d < bd) {
      bd = d;
      best = i;
    }
  }
  return best;
}

__global__ void k_grid_to_points(int nlat, int nlon, const double *__restrict__ lat1d,
                                 const double *__restrict__ lon1d, const double *__restrict__ grid,
                                 long long n, const double *__restrict__ lat, const double *__restrict__ lon,
                                 double *out, int staged) {
  extern __shared__ double axes[];
  pdl_begin();
  const double *la = lat1d, *lo = lon1d;
  if (staged) {
    for (int i = threadIdx.x; i < nlat + nlon; i += blockDim.x) axes[i] = i < nlat ? lat1d[i] : lon1d[i - nlat];
    __syncthreads();
    la = axes;
    lo = axes + nlat;
  }
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int i0 = nearest(la, nlat, lat[t]), j0 = nearest(lo, nlon, lon[t]);
    const int i1 = i0 > 0 ? i0 - 1 : 0, i2 = i0 + 1 < nlat ? i0 + 1 : nlat - 1;
    const int j1 = j0 > 0 ? j0 - 1 : 0, j2 = j0 + 1 < nlon ? j0 + 1 : nlon - 1;
    double s = 0.0;
    for (int j = j1; j <= j2; j++)
      for (int i = i1; i <= i2; i++) s = s + grid[(size_t)i * nlon + j];
    out[t] = s / (double)((i2 - i1 + 1) * (j2 - j1 + 1));
  }
}

}  // namespace
}  // namespace mpsw

extern "C" int mpsw_grid_to_points(mpsw_handle *h, int nlat, int nlon, const double *lat1d, const double *lon1d,
                                   const double *grid, long long n, const double *lat, const double *lon,
                                   double *out, void *stream) {
  return mpsw::guarded(h, [&](mpsw::Engine &e) {
    using namespace mpsw;
    if (nlat < 1 || nlon < 1 || n < 0) throw EngineError(MPSW_ERR_ARG, "grid_to_points: empty grid or n < 0");
    if (!lat1d || !lon1d || !grid || (n && (!lat || !lon || !out)))
      throw EngineError(MPSW_ERR_ARG, "grid_to_points: null buffer");
    if (n == 0) return;
    e.need_device();
    const size_t axes = sizeof(double) * ((size_t)nlat + nlon);
    const int staged = axes <= 48 * 1024;
    const int block = 128;
    long long g = (n + block - 1) / block;
    if (g > 148LL * 32) g = 148LL * 32;
    g_launches++;
    launch_k(k_grid_to_points, LaunchCfg{(int)g, block, staged ? axes : 0}, (cudaStream_t)stream, nlat, nlon,
             lat1d, lon1d, grid, n, lat, lon, out, staged);
    cuda_check(cudaGetLastError(), "grid_to_points");
  });
}
