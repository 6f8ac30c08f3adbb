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
  unsigned int arrive;         // blocks done with their partials (exchange_fold)
};

// Floating-point exchange sums in a fixed order: block partials (slot-major,
// NV x gridDim.x in part), folded by the last block into out[0..NV).  The
// result depends only on the grid and the command order, not on which block
// finishes first.  Every thread of a kThreads block calls it.
template <int NV>
__device__ __forceinline__ void exchange_fold(const double (&v)[NV], double* __restrict__ part,
                                              unsigned int* arrive, double* out) {
  __shared__ double fold[fold_words(NV)];
  __shared__ int last;
  const double* bt = block_fold<double, NV, NV>(v, fold);
  if (threadIdx.x < NV) part[(size_t)threadIdx.x * gridDim.x + blockIdx.x] = bt[threadIdx.x];
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(arrive, 1u) == gridDim.x - 1 ? 1 : 0;
  __syncthreads();
  if (!last) return;
  __threadfence();
  const double* tot = reduce_partials<NV, NV>(part, (int)gridDim.x, fold);
  if (threadIdx.x < NV) out[threadIdx.x] = tot[threadIdx.x];
  if (threadIdx.x == 0) *arrive = 0u;
}

// mode 0: requested depth; mode 1: requested target surface (depth = b - target).
template <bool FX>
__global__ void __launch_bounds__(kThreads)
    entrain_kernel(int ny, int nx, int pitch, double Q, double datum, double f,
                   typename FvTypes<FX>::B* __restrict__ b, const typename FvTypes<FX>::B* __restrict__ z,
                   typename FvTypes<FX>::H* __restrict__ h, const int32_t* __restrict__ idx,
                   const double* __restrict__ value, int count, int mode, ExchangeOut* out,
                   double* __restrict__ part) {
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
  if constexpr (FX) {
    vq = (long long)warp_sum_u64((unsigned long long)vq);
    if ((threadIdx.x & 31) == 0 && vq)
      atomicAdd((unsigned long long*)&out->volume_w6_quanta, (unsigned long long)vq);
  } else {
    const double v[1] = {vs};
    exchange_fold<1>(v, part, &out->arrive, &out->volume_w_fp64);
  }
}

template <bool FX>
__global__ void __launch_bounds__(kThreads)
    deposit_kernel(int ny, int nx, int pitch, double Q, double f,
                   typename FvTypes<FX>::B* __restrict__ b, typename FvTypes<FX>::H* __restrict__ h,
                   typename FvTypes<FX>::R* __restrict__ qx, typename FvTypes<FX>::R* __restrict__ qy,
                   const int32_t* __restrict__ idx, const double* __restrict__ depth, int count,
                   ExchangeOut* out, double* __restrict__ part) {
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
  if constexpr (FX) {
    vq = (long long)warp_sum_u64((unsigned long long)vq);
    if ((threadIdx.x & 31) == 0 && vq)
      atomicAdd((unsigned long long*)&out->volume_w6_quanta, (unsigned long long)vq);
    const double v[2] = {mx, my};
    exchange_fold<2>(v, part, &out->arrive, out->momentum_w);
  } else {
    // volume_w_fp64 and momentum_w[0..1] are consecutive
    const double v[3] = {vs, mx, my};
    exchange_fold<3>(v, part, &out->arrive, &out->volume_w_fp64);
  }
}

}  // namespace sb
