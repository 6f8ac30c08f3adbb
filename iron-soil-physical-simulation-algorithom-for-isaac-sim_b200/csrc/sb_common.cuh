// Shared device helpers for the soilb200 kernels (sm_100a).
//
// The whole library is compiled with -fmad=false: every float/double
// expression is evaluated as individually rounded IEEE operations, which is
// what lets the FP64 kernels match the reference NumPy solver bit for bit and
// the fixed-point kernels match their CPU mirror.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace sb {

constexpr int kThreads = 256;
// Bounded device-side waits: a wait that exceeds this many polls records
// SB_ERR_WAIT_LIMIT in the control block and the kernel gives up the tile.
constexpr unsigned kSpinLimit = 1u << 24;

// ---------------------------------------------------------------------------
// Warp / block reductions (fixed shuffle tree => deterministic order).
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
template <typename T>
__device__ __forceinline__ T warp_max(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    T w = __shfl_xor_sync(0xffffffffu, v, o);
    v = w > v ? w : v;
  }
  return v;
}
template <typename T>
__device__ __forceinline__ T warp_min(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    T w = __shfl_xor_sync(0xffffffffu, v, o);
    v = w < v ? w : v;
  }
  return v;
}

// Block-wide sum of N doubles per thread; result valid in thread 0.
// ``scratch`` must hold kThreads/32 * N doubles.
template <int N>
__device__ __forceinline__ void block_sum(double (&v)[N], double* scratch) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < N; ++k) v[k] = warp_sum(v[k]);
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < N; ++k) scratch[warp * N + k] = v[k];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < N; ++k) {
      double s = 0.0;
      for (int w = 0; w < kThreads / 32; ++w) s += scratch[w * N + k];
      v[k] = s;
    }
  }
  __syncthreads();
}

// Fixed-order block reduction of NV values per thread through shared memory.
// A shuffle tree over NV doubles costs 10*NV shuffles per warp and the SM
// issues about one warp-shuffle per clock, so with many values per thread the
// shuffles, not the arithmetic, bound a block reduction; here each value is
// stored once and folded by NV*8 threads.  Slots [0, NSUM) are summed, slots
// [NSUM, NV) take the maximum.  Order: 32 consecutive threads in order, then
// the 8 groups in order.  ``scratch`` holds fold_words(NV) values of type T;
// the result is returned as a pointer to NV values in ``scratch``, valid for
// every thread of the block until the scratch is reused.
constexpr int kFoldStride = kThreads + kThreads / 32;  // one pad slot per 32 threads
__host__ __device__ constexpr int fold_words(int nv) { return nv * kFoldStride + nv * 8 + nv; }

__device__ __forceinline__ double fold_max(double a, double b) { return fmax(a, b); }
__device__ __forceinline__ long long fold_max(long long a, long long b) { return a > b ? a : b; }

template <typename T, int NV, int NSUM>
__device__ __forceinline__ const T* block_fold(const T* v, T* scratch) {
  static_assert(NV * 8 <= kThreads, "one pass of chunk folds");
  const int t = threadIdx.x;
  const int pos = t + (t >> 5);
#pragma unroll
  for (int k = 0; k < NV; ++k) scratch[k * kFoldStride + pos] = v[k];
  __syncthreads();
  T* part = scratch + NV * kFoldStride;
  T* out = part + NV * 8;
  if (t < NV * 8) {
    const int k = t >> 3, ch = t & 7;
    const T* src = scratch + k * kFoldStride + ch * 33;
    T s = src[0];
    if (k >= NSUM) {
#pragma unroll 8
      for (int j = 1; j < 32; ++j) s = fold_max(s, src[j]);
    } else {
#pragma unroll 8
      for (int j = 1; j < 32; ++j) s += src[j];
    }
    part[t] = s;
  }
  __syncthreads();
  if (t < NV) {
    const T* p = part + t * 8;
    T s = p[0];
#pragma unroll
    for (int ch = 1; ch < 8; ++ch) s = t >= NSUM ? fold_max(s, p[ch]) : s + p[ch];
    out[t] = s;
  }
  __syncthreads();
  return out;
}

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// ---------------------------------------------------------------------------
// TMA (cp.async.bulk.tensor) + mbarrier helpers.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

// Returns true when the phase completed, false after kSpinLimit polls.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity) {
  const uint32_t a = smem_u32(bar);
  for (unsigned i = 0; i < kSpinLimit; ++i) {
    uint32_t done;
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// 2-D tiled TMA load; x (innermost) must be a multiple of 16 bytes / element.
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
      "[%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void prefetch_tmap(const CUtensorMap* map) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(map) : "memory");
}

// Atomic max for non-negative floats / doubles via their integer images.
__device__ __forceinline__ void atomic_max_nonneg(float* addr, float v) {
  atomicMax(reinterpret_cast<int*>(addr), __float_as_int(v));
}
__device__ __forceinline__ void atomic_max_nonneg(double* addr, double v) {
  atomicMax(reinterpret_cast<unsigned long long*>(addr),
            static_cast<unsigned long long>(__double_as_longlong(v)));
}

// Triangle-A-C vertex weight of cell (r, c) in units of dx*dy/6
// (reference runtime/bulk_state_authority.py:612-621: 2f on [:-1,:-1],
// f on [:-1,1:], 2f on [1:,1:], f on [1:,:-1]).
__device__ __forceinline__ int vertex_weight6(int r, int c, int ny, int nx) {
  int w = 0;
  if (r < ny - 1 && c < nx - 1) w += 2;
  if (r < ny - 1 && c > 0) w += 1;
  if (r > 0 && c > 0) w += 2;
  if (r > 0 && c < nx - 1) w += 1;
  return w;
}

}  // namespace sb
