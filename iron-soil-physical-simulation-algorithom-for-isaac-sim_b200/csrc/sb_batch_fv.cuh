// Batched Mobile V2 runtime: patch table types and the substep kernel.
//
// Kept apart from sb_batch.cuh so that the production instantiation
// batch_fv_kernel<true> can be compiled in the FMA-contracted translation
// unit (sb_fv_fast.cu) without the other batch kernels.
#pragma once

#include "sb_fv.cuh"

namespace sb {

constexpr int kBandRows = 32;  // ledger band height (one CTA per band)

struct BatchPatch {
  FvConst c;          // geometry (ny, nx, pitch, strips in tiles_x, rows_per_warp) + constants
  long long base;     // element offset of the patch's row 0 in the field arenas
  double datum;       // support datum of the patch's b / z quanta
  double static_limit;
  int first_item, n_items;  // FV warps
  int first_band, n_bands;  // ledger CTAs
};

struct BatchCtl {  // per patch, device resident
  FvControl k;
  LedgerOut before;
  LedgerOut after;
};

struct BatchGlobal {
  unsigned arrive;
  int active;
};

struct BatchArena {
  const int32_t* b;
  const int32_t* z;
  int32_t* h[2];
  float* qx[2];
  float* qy[2];
};

// One substep of every active patch; a warp per work item.
template <bool FAST>
__global__ void __launch_bounds__(kThreads, 3)
    batch_fv_kernel(const BatchPatch* __restrict__ patches, const int* __restrict__ item_patch,
                    int nitems, BatchArena a, const BatchCtl* __restrict__ ctl,
                    double* __restrict__ item_partials) {
  const int gw = blockIdx.x * (kThreads / 32) + (threadIdx.x >> 5);
  if (gw >= nitems) return;  // warp-uniform
  const int p = item_patch[gw];
  if (ctl[p].k.done) return;
  const BatchPatch& P = patches[p];
  const FvConst& c = P.c;  // read through the read-only cache, not copied
  const long long base = P.base;
  const double sub_dt = ctl[p].k.sub_dt;
  const int parity = ctl[p].k.parity;
  const int local = gw - P.first_item;
  double acc[kFvDiag];
#pragma unroll
  for (int k = 0; k < kFvDiag; ++k) acc[k] = 0.0;
  double wave = 0.0;
  fx_strip_run<FAST>(c, a.b + base, a.h[parity] + base, a.qx[parity] + base, a.qy[parity] + base,
               a.h[parity ^ 1] + base, a.qx[parity ^ 1] + base, a.qy[parity ^ 1] + base, nullptr,
               nullptr, local % c.tiles_x, (local / c.tiles_x) * c.rows_per_warp,
               min((local / c.tiles_x + 1) * c.rows_per_warp, c.ny), sub_dt, acc, wave);
#pragma unroll
  for (int k = 0; k < kFvDiag; ++k) acc[k] = warp_sum(acc[k]);
  wave = warp_max(wave);
  if ((threadIdx.x & 31) == 0) {
    double* out = item_partials + (size_t)gw * (kFvDiag + 1);
    for (int k = 0; k < kFvDiag; ++k) out[k] = acc[k];
    out[kFvDiag] = wave;
  }
}

}  // namespace sb
