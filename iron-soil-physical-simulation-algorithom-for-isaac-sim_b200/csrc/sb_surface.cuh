// Consumer side of the step: dirty-tile tracking, tile / region downloads and
// batched bilinear surface queries (reference
// runtime/bulk_state_authority.py:156-231 kernels capture_surface,
// flag_surface_change, bilinear_surface; methods :733-781, :1138-1183,
// :1280-1328).  The free surface is b_eff + h.
#pragma once

#include "sb_common.cuh"
#include "sb_fv.cuh"

namespace sb {

template <bool FX>
__device__ __forceinline__ double free_surface(const typename FvTypes<FX>::B* b,
                                               const typename FvTypes<FX>::H* h, size_t gi,
                                               double Q, double datum) {
  if constexpr (FX) {
    return (double)((long long)b[gi] + (long long)h[gi]) * Q + datum;
  } else {
    return b[gi] + h[gi];
  }
}

template <bool FX>
__global__ void surface_capture_kernel(int ny, int nx, int pitch, double Q, double datum,
                                       const typename FvTypes<FX>::B* __restrict__ b,
                                       const typename FvTypes<FX>::H* __restrict__ h,
                                       double* __restrict__ before) {
  const long long n = (long long)ny * nx;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const size_t gi = (size_t)(i / nx) * pitch + (i % nx);
    before[i] = free_surface<FX>(b, h, gi, Q, datum);
  }
}

template <bool FX>
__global__ void surface_flag_kernel(int ny, int nx, int pitch, double Q, double datum,
                                    const typename FvTypes<FX>::B* __restrict__ b,
                                    const typename FvTypes<FX>::H* __restrict__ h,
                                    const double* __restrict__ before, int tile_size, int tiles_x,
                                    double tolerance, int* __restrict__ tile_flags) {
  const long long n = (long long)ny * nx;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(i / nx), c = (int)(i % nx);
    const double s = free_surface<FX>(b, h, (size_t)r * pitch + c, Q, datum);
    if (fabs(s - before[i]) > tolerance) tile_flags[(r / tile_size) * tiles_x + c / tile_size] = 1;
  }
}

// Free surface over rows [r0, r1) x cols [c0, c1), row-major into out.
template <bool FX>
__global__ void surface_region_kernel(int nx_region, int count, int r0, int c0, int pitch, double Q,
                                      double datum, const typename FvTypes<FX>::B* __restrict__ b,
                                      const typename FvTypes<FX>::H* __restrict__ h,
                                      double* __restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    const int r = r0 + i / nx_region, c = c0 + i % nx_region;
    out[i] = free_surface<FX>(b, h, (size_t)r * pitch + c, Q, datum);
  }
}

// Bilinear free-surface samples at fractional (row, col), clamped to the grid
// (reference order of the weighted sum).
template <bool FX>
__global__ void surface_bilinear_kernel(int ny, int nx, int pitch, double Q, double datum,
                                        const typename FvTypes<FX>::B* __restrict__ b,
                                        const typename FvTypes<FX>::H* __restrict__ h,
                                        const double* __restrict__ rows,
                                        const double* __restrict__ cols, int count,
                                        double* __restrict__ out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    const double row = fmin(fmax(rows[i], 0.0), (double)(ny - 1));
    const double col = fmin(fmax(cols[i], 0.0), (double)(nx - 1));
    const int r0 = (int)floor(row), c0 = (int)floor(col);
    const int r1 = min(r0 + 1, ny - 1), c1 = min(c0 + 1, nx - 1);
    const double fr = row - (double)r0, fc = col - (double)c0;
    const double v00 = free_surface<FX>(b, h, (size_t)r0 * pitch + c0, Q, datum);
    const double v01 = free_surface<FX>(b, h, (size_t)r0 * pitch + c1, Q, datum);
    const double v10 = free_surface<FX>(b, h, (size_t)r1 * pitch + c0, Q, datum);
    const double v11 = free_surface<FX>(b, h, (size_t)r1 * pitch + c1, Q, datum);
    out[i] = (1.0 - fr) * (1.0 - fc) * v00 + (1.0 - fr) * fc * v01 + fr * (1.0 - fc) * v10 +
             fr * fc * v11;
  }
}

}  // namespace sb
