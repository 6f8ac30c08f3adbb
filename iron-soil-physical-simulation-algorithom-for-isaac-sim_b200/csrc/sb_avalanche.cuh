// Large-avalanche activation and lifecycle diagnostics (reference
// runtime/gpu_large_avalanche.py kernels ``mobilize`` :308-372 and
// ``reduce_persistence`` :374-451).
//
// mobilize: every unlatched cell of the selected component (the winner of the
// last labelling, read on the device) moves
//   transfer = min(max(b_eff - z_base, 0), mobilization_depth * severity)
// from Resting to Mobile at zero momentum (when above the dry tolerance),
// records its owned surface and export baseline, latches, and updates the
// per-cell activation history (count, first/last time, cumulative R->M).
// In the fixed-point state the transfer is a whole number of quanta (the
// same cap as the component's mobilizable volume), so it is exact.
//
// persistence: fixed-size lifecycle sums over the whole grid (activation
// history, current/moving mobile volume, net terrain change, activity tiles).
// Sums use block partials folded in a fixed order by the last block.
#pragma once

#include "sb_common.cuh"
#include "sb_fv.cuh"
#include "sb_labels.cuh"

namespace sb {

struct MobilizeConst {
  int ny, nx, pitch;
  double Q, datum, f;   // f = dx*dy/6 (weight unit)
  double mob_depth, dry, time_s;
};

constexpr int kMobilizeSums = 6;  // transferred, new vol, re vol, new area, re area, cells

struct MobilizeOut {
  double v[kMobilizeSums];
  long long transferred_w6_quanta;
};

template <bool FX>
__global__ void __launch_bounds__(kThreads)
    mobilize_kernel(const MobilizeConst c, const typename FvTypes<FX>::B* __restrict__ z,
                    typename FvTypes<FX>::B* __restrict__ b, typename FvTypes<FX>::H* __restrict__ h,
                    const int* __restrict__ parent, int* __restrict__ latch,
                    const typename FvTypes<FX>::R* __restrict__ severity,
                    double* __restrict__ owned_surface, double* __restrict__ export_base,
                    const double* __restrict__ export_cum, int* __restrict__ act_count,
                    double* __restrict__ act_first, double* __restrict__ act_last,
                    double* __restrict__ r2m, const LabelOut* lout, double* __restrict__ partials,
                    unsigned* arrive, MobilizeOut* out) {
  const int winner = lout->winner;
  const long long n = (long long)c.ny * c.nx;
  double s[kMobilizeSums] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  long long tq_sum = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n && winner >= 0;
       i += (long long)gridDim.x * blockDim.x) {
    if (parent[i] != winner || latch[i] != 0) continue;
    const int r = (int)(i / c.nx), col = (int)(i % c.nx);
    const size_t gi = (size_t)r * c.pitch + col;
    const int w6 = vertex_weight6(r, col, c.ny, c.nx);
    const double w = (double)w6 * c.f;
    double transfer;
    if constexpr (FX) {
      const long long avail = (long long)b[gi] - (long long)z[gi];
      const long long cap = (long long)floor(c.mob_depth * (double)severity[i] / c.Q);
      long long tq = avail < cap ? avail : cap;
      if (tq < 0) tq = 0;
      transfer = (double)tq * c.Q;
      if (!(transfer > c.dry)) continue;
      owned_surface[i] = ((double)b[gi] + (double)h[gi]) * c.Q + c.datum;
      b[gi] = (int32_t)((long long)b[gi] - tq);
      h[gi] = (int32_t)((long long)h[gi] + tq);
      tq_sum += tq * w6;
    } else {
      transfer = fmin(fmax(b[gi] - z[gi], 0.0), c.mob_depth * severity[i]);
      if (!(transfer > c.dry)) continue;
      owned_surface[i] = b[gi] + h[gi];
      b[gi] = b[gi] - transfer;
      h[gi] = h[gi] + transfer;
    }
    export_base[i] = export_cum[i];
    latch[i] = 1;
    const double weighted = transfer * w;
    const int prev = act_count[i];
    act_count[i] = prev + 1;
    if (prev == 0) {
      act_first[i] = c.time_s;
      s[1] += weighted;
      s[3] += w;
    } else {
      s[2] += weighted;
      s[4] += w;
    }
    act_last[i] = c.time_s;
    r2m[i] = r2m[i] + weighted;
    s[0] += weighted;
    s[5] += 1.0;
  }
  __shared__ double red[kThreads / 32 * (kMobilizeSums + 1)];
  __shared__ int last;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < kMobilizeSums; ++k) s[k] = warp_sum(s[k]);
  tq_sum = (long long)warp_sum_u64((unsigned long long)tq_sum);
  constexpr int NS = kMobilizeSums + 1;
  if (lane == 0) {
    for (int k = 0; k < kMobilizeSums; ++k) red[warp * NS + k] = s[k];
    red[warp * NS + kMobilizeSums] = __longlong_as_double(tq_sum);
  }
  __syncthreads();
  if (threadIdx.x < NS) {
    double a = 0.0;
    long long ai = 0;
    for (int w2 = 0; w2 < kThreads / 32; ++w2) {
      if (threadIdx.x == kMobilizeSums) ai += __double_as_longlong(red[w2 * NS + threadIdx.x]);
      else a += red[w2 * NS + threadIdx.x];
    }
    partials[(size_t)blockIdx.x * NS + threadIdx.x] =
        threadIdx.x == kMobilizeSums ? __longlong_as_double(ai) : a;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = (atomicAdd(arrive, 1u) == gridDim.x - 1) ? 1 : 0;
  __syncthreads();
  if (!last || threadIdx.x != 0) return;
  __threadfence();
  double t[kMobilizeSums] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  long long ti = 0;
  for (unsigned bk = 0; bk < gridDim.x; ++bk) {
    for (int k = 0; k < kMobilizeSums; ++k) t[k] += __ldcg(partials + (size_t)bk * NS + k);
    ti += __double_as_longlong(__ldcg(partials + (size_t)bk * NS + kMobilizeSums));
  }
  for (int k = 0; k < kMobilizeSums; ++k) out->v[k] = t[k];
  out->transferred_w6_quanta = ti;
  *arrive = 0;
}

struct PersistConst {
  int ny, nx, pitch, tile_size, tiles_x;
  double Q, datum, f, start_rad, stop_rad, dry, activity_speed;
};

// sums: 0 r2m, 1 m2r, 2 unique area, 3 reactivated area, 4 mobile volume,
// 5 max speed (max), 6 net change, 7 net transfer, 8 slope sum, 9 max slope
// (max), 10 slope - stop, 11 start - slope, 12 retired area, 13 moving volume;
// counts: 14 unique cells, 15 reactivated cells, 16 wet cells, 17 retired.
constexpr int kPersistSlots = 18;

template <bool FX>
__global__ void __launch_bounds__(kThreads)
    persistence_kernel(const PersistConst c, const typename FvTypes<FX>::B* __restrict__ b0,
                       const typename FvTypes<FX>::B* __restrict__ b,
                       const typename FvTypes<FX>::H* __restrict__ h,
                       const typename FvTypes<FX>::R* __restrict__ qx,
                       const typename FvTypes<FX>::R* __restrict__ qy,
                       const typename FvTypes<FX>::R* __restrict__ slope,
                       const int* __restrict__ parent, const int* __restrict__ latch,
                       const int* __restrict__ act_count, const double* __restrict__ r2m,
                       const double* __restrict__ m2r, int* __restrict__ tile_flags,
                       double* __restrict__ partials, unsigned* arrive, double* out) {
  const long long n = (long long)c.ny * c.nx;
  double s[kPersistSlots];
#pragma unroll
  for (int k = 0; k < kPersistSlots; ++k) s[k] = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(i / c.nx), col = (int)(i % c.nx);
    const size_t gi = (size_t)r * c.pitch + col;
    const double w = (double)vertex_weight6(r, col, c.ny, c.nx) * c.f;
    double hv, bv, b0v;
    if constexpr (FX) {
      hv = (double)h[gi] * c.Q;
      bv = (double)b[gi] * c.Q;
      b0v = (double)b0[gi] * c.Q;
    } else {
      hv = h[gi];
      bv = b[gi];
      b0v = b0[gi];
    }
    double speed = 0.0;
    if (hv > c.dry) {
      const double vx = (double)qx[gi] / hv, vy = (double)qy[gi] / hv;
      speed = sqrt(vx * vx + vy * vy);
      s[16] += 1.0;
      s[4] += hv * w;
      s[5] = fmax(s[5], speed);
      if (speed > c.activity_speed) s[13] += hv * w;
    }
    if (parent[i] >= 0 || (hv > c.dry && speed > c.activity_speed))
      tile_flags[(r / c.tile_size) * c.tiles_x + col / c.tile_size] = 1;
    const double delta = (bv + hv) - b0v;
    s[6] += delta * w;
    s[7] += fabs(delta) * w * 0.5;
    s[0] += r2m[i];
    s[1] += m2r[i];
    const int count = act_count[i];
    if (count <= 0) continue;
    const double sl = (double)slope[i];
    s[14] += 1.0;
    s[2] += w;
    s[8] += sl;
    s[9] = fmax(s[9], sl);
    s[10] += sl - c.stop_rad;
    s[11] += c.start_rad - sl;
    if (count > 1) {
      s[15] += 1.0;
      s[3] += w;
    }
    if (hv <= c.dry && sl <= c.stop_rad && latch[i] == 0) {
      s[17] += 1.0;
      s[12] += w;
    }
  }
  __shared__ double red[kThreads / 32 * kPersistSlots];
  __shared__ int last;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < kPersistSlots; ++k)
    s[k] = (k == 5 || k == 9) ? warp_max(s[k]) : warp_sum(s[k]);
  if (lane == 0)
    for (int k = 0; k < kPersistSlots; ++k) red[warp * kPersistSlots + k] = s[k];
  __syncthreads();
  if (threadIdx.x < kPersistSlots) {
    const int k = threadIdx.x;
    double a = 0.0;
    for (int w2 = 0; w2 < kThreads / 32; ++w2)
      a = (k == 5 || k == 9) ? fmax(a, red[w2 * kPersistSlots + k]) : a + red[w2 * kPersistSlots + k];
    partials[(size_t)blockIdx.x * kPersistSlots + k] = a;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = (atomicAdd(arrive, 1u) == gridDim.x - 1) ? 1 : 0;
  __syncthreads();
  if (!last) return;
  __threadfence();
  if (threadIdx.x < kPersistSlots) {
    const int k = threadIdx.x;
    double a = 0.0;
    for (unsigned bk = 0; bk < gridDim.x; ++bk) {
      const double x = __ldcg(partials + (size_t)bk * kPersistSlots + k);
      a = (k == 5 || k == 9) ? fmax(a, x) : a + x;
    }
    out[k] = a;
  }
  __syncthreads();
  if (threadIdx.x == 0) *arrive = 0;
}

}  // namespace sb
