// Resting <-> Mobile exchange primitives (reference
// runtime/bulk_state_authority.py:103-149, ``entrain`` / ``deposit``).
//
// Both keep b_eff + h invariant cell by cell.  Entrainment is donor-limited by
// max(b_eff - z_base, 0) and leaves momentum untouched; deposition is limited
// by the mobile thickness and removes the proportional momentum.  In the
// fixed-point precision the exchanged depth is a whole number of quanta, so
// the exchange volume sums are exact int64 (no compensation needed).
#pragma once

#include "sb_common.cuh"
#include "sb_fv.cuh"

namespace sb {

struct ExchangeOut {
  long long volume_w6_quanta;  // FX: sum depth_quanta * w6
  double volume_w_fp64;        // FP64: sum depth * w
  double momentum_w[2];        // deposition: sum removed q * w
  int bad_index;
  int pad;
};

// mode 0: requested depth; mode 1: requested target surface (depth = b - target).
template <bool FX>
__global__ void __launch_bounds__(kThreads)
    entrain_kernel(int ny, int nx, int pitch, double Q, double datum, double f,
                   typename FvTypes<FX>::B* __restrict__ b, const typename FvTypes<FX>::B* __restrict__ z,
                   typename FvTypes<FX>::H* __restrict__ h, const int32_t* __restrict__ idx,
                   const double* __restrict__ value, int count, int mode, ExchangeOut* out) {
  long long vq = 0;
  double vs = 0.0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x) {
    const int i = idx[k];
    if (i < 0 || i >= ny * nx) {
      atomicExch(&out->bad_index, 1);
      continue;
    }
    const int r = i / nx, c = i % nx;
    const size_t gi = (size_t)r * pitch + c;
    const int w6 = vertex_weight6(r, c, ny, nx);
    if constexpr (FX) {
      const long long avail = (long long)b[gi] - (long long)z[gi];
      long long req;
      if (mode == 0) {
        req = (long long)llrint(fmax(value[k], 0.0) / Q);
      } else {
        const double tq = rint((value[k] - datum) / Q);
        req = (long long)b[gi] - (long long)tq;
      }
      long long d = req < avail ? req : avail;
      if (d < 0) d = 0;
      b[gi] = (int32_t)(b[gi] - d);
      h[gi] = (int32_t)(h[gi] + d);
      vq += d * w6;
    } else {
      const double avail = fmax(b[gi] - z[gi], 0.0);
      const double req = mode == 0 ? fmax(value[k], 0.0) : fmax(b[gi] - value[k], 0.0);
      const double d = fmin(req, avail);
      b[gi] = b[gi] - d;
      h[gi] = h[gi] + d;
      vs += d * ((double)w6 * f);
    }
  }
  vq = (long long)warp_sum_u64((unsigned long long)vq);
  vs = warp_sum(vs);
  if ((threadIdx.x & 31) == 0) {
    if (vq) atomicAdd((unsigned long long*)&out->volume_w6_quanta, (unsigned long long)vq);
    if (vs != 0.0) atomicAdd(&out->volume_w_fp64, vs);
  }
}

template <bool FX>
__global__ void __launch_bounds__(kThreads)
    deposit_kernel(int ny, int nx, int pitch, double Q, double f,
                   typename FvTypes<FX>::B* __restrict__ b, typename FvTypes<FX>::H* __restrict__ h,
                   typename FvTypes<FX>::R* __restrict__ qx, typename FvTypes<FX>::R* __restrict__ qy,
                   const int32_t* __restrict__ idx, const double* __restrict__ depth, int count,
                   ExchangeOut* out) {
  long long vq = 0;
  double vs = 0.0, mx = 0.0, my = 0.0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x) {
    const int i = idx[k];
    if (i < 0 || i >= ny * nx) {
      atomicExch(&out->bad_index, 1);
      continue;
    }
    const int r = i / nx, c = i % nx;
    const size_t gi = (size_t)r * pitch + c;
    const double w = (double)vertex_weight6(r, c, ny, nx) * f;
    if constexpr (FX) {
      const long long before = h[gi] > 0 ? h[gi] : 0;
      long long d = (long long)llrint(fmax(depth[k], 0.0) / Q);
      if (d > before) d = before;
      const double frac = before > 0 ? (double)d / (double)before : 0.0;
      const float rx = (float)((double)qx[gi] * frac), ry = (float)((double)qy[gi] * frac);
      b[gi] = (int32_t)(b[gi] + d);
      h[gi] = (int32_t)(before - d);
      qx[gi] = qx[gi] - rx;
      qy[gi] = qy[gi] - ry;
      vq += d * vertex_weight6(r, c, ny, nx);
      mx += (double)rx * w;
      my += (double)ry * w;
    } else {
      const double before = fmax(h[gi], 0.0);
      const double d = fmin(fmax(depth[k], 0.0), before);
      const double frac = before > 0.0 ? d / before : 0.0;
      const double rx = qx[gi] * frac, ry = qy[gi] * frac;
      b[gi] = b[gi] + d;
      h[gi] = before - d;
      qx[gi] = qx[gi] - rx;
      qy[gi] = qy[gi] - ry;
      vs += d * w;
      mx += rx * w;
      my += ry * w;
    }
  }
  vq = (long long)warp_sum_u64((unsigned long long)vq);
  vs = warp_sum(vs);
  mx = warp_sum(mx);
  my = warp_sum(my);
  if ((threadIdx.x & 31) == 0) {
    if (vq) atomicAdd((unsigned long long*)&out->volume_w6_quanta, (unsigned long long)vq);
    if (vs != 0.0) atomicAdd(&out->volume_w_fp64, vs);
    if (mx != 0.0) atomicAdd(&out->momentum_w[0], mx);
    if (my != 0.0) atomicAdd(&out->momentum_w[1], my);
  }
}

}  // namespace sb
