// Batched Mobile V2 runtime: many independent terrain patches (parallel dig
// environments of uneven sizes) advanced by the same launches.
//
// Every patch keeps its own quantisation, CFL substep dt, substep count and
// ping-pong parity (the per-patch loop of MobileV2ReferenceSolver.step,
// experimental/mobile_v2_reference.py:191-314).  A patch table drives the
// launches:
//   * FV work items are warps (one 30-column strip x rows_per_warp rows of one
//     patch, the same strip code as the single-grid kernel); item_patch maps
//     a global warp index to its patch, and rows_per_warp is chosen per patch
//     by the autotuner;
//   * ledger work items are CTAs over bands of kBandRows rows of one patch.
// Each substep round is two launches: all active patches' strips, then one
// warp per patch that reduces that patch's item partials in a fixed order,
// advances its loop control and plans its next dt; the last CTA of that
// launch sets the graph's while-condition to "some patch still active".
// The arithmetic is the single-grid FX32 kernel's, so every patch's fields
// are identical to stepping it alone.
#pragma once

#include "sb_batch_fv.cuh"
#include "sb_ledger.cuh"

namespace sb {

__global__ void batch_begin_kernel(int npatch, BatchCtl* ctl, const double* dt) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npatch) return;
  FvControl& k = ctl[p].k;
  k.remaining = *dt;
  k.sub_dt = 0.0;
  k.max_cfl = 0.0;
  k.wave = 0.0;
  for (int i = 0; i < kFvDiag; ++i) k.diag[i] = 0.0;
  k.substeps = 0;
  k.done = 0;
  k.status = 0;
  k.cfl_limited = 0;
  k.static_skip = 0;
  k.arrive = 0;
  k.wait_fail = 0;
}

// One CTA per ledger band.
__global__ void __launch_bounds__(kThreads)
    batch_ledger_kernel(const BatchPatch* __restrict__ patches, const int* __restrict__ band_patch,
                        int nbands, BatchArena a, const BatchCtl* __restrict__ ctl,
                        double* __restrict__ partials, long long* __restrict__ ipartials) {
  __shared__ double fold[fold_words(L_NP)];
  const int band = blockIdx.x;
  if (band >= nbands) return;
  const int p = band_patch[band];
  const BatchPatch& P = patches[p];
  const FvConst c = P.c;
  const int parity = ctl[p].k.parity;
  const long long base = P.base;
  const int r0 = (band - P.first_band) * kBandRows;
  const int r1 = min(r0 + kBandRows, c.ny);
  double v[L_NP];
#pragma unroll
  for (int k = 0; k < L_NP; ++k) v[k] = 0.0;
  v[L_NEGMINH] = -1.0e300;
  long long iq0 = 0, iq1 = 0, iq2 = 0;
  const int n = (r1 - r0) * c.nx;
  for (int i = threadIdx.x; i < n; i += kThreads)
    ledger_cell<true>(c, a.b + base, a.z + base, a.h[parity] + base, a.qx[parity] + base,
                      a.qy[parity] + base, nullptr, nullptr, P.datum, r0 + i / c.nx, i % c.nx, v,
                      iq0, iq1, iq2);
  ledger_block_store(v, iq0, iq1, iq2, fold, partials + (size_t)band * L_NP,
                     ipartials + (size_t)band * kLedgerI64, 1);
}

// One warp per patch: fixed-order fold of the patch's band partials into its
// ledger; mode 0 also runs the prologue (static check, first dt) and counts
// the patches that have substeps to run.
__global__ void __launch_bounds__(kThreads)
    batch_ledger_finish_kernel(int npatch, const BatchPatch* __restrict__ patches,
                               BatchCtl* ctl, const double* __restrict__ partials,
                               const long long* __restrict__ ipartials, int mode, BatchGlobal* g,
                               cudaGraphConditionalHandle handle, int use_handle) {
  __shared__ int last;
  const int lane = threadIdx.x & 31;
  const int p = blockIdx.x * (kThreads / 32) + (threadIdx.x >> 5);
  if (p < npatch) {
    const BatchPatch& P = patches[p];
    double v[L_NP];
#pragma unroll
    for (int k = 0; k < L_NP; ++k) v[k] = 0.0;
    v[L_NEGMINH] = -1.0e300;
    long long iq[kLedgerI64] = {0, 0, 0};
    for (int j = lane; j < P.n_bands; j += 32) {
      const size_t bidx = (size_t)(P.first_band + j);
#pragma unroll
      for (int k = 0; k < L_NP; ++k) {
        const double x = partials[bidx * L_NP + k];
        v[k] = k < L_NSUM ? v[k] + x : fmax(v[k], x);
      }
      for (int k = 0; k < kLedgerI64; ++k) iq[k] += ipartials[bidx * kLedgerI64 + k];
    }
#pragma unroll
    for (int k = 0; k < L_NP; ++k) v[k] = k < L_NSUM ? warp_sum(v[k]) : warp_max(v[k]);
    for (int k = 0; k < kLedgerI64; ++k) iq[k] = (long long)warp_sum_u64((unsigned long long)iq[k]);
    if (lane == 0) {
      LedgerOut* out = mode == 0 ? &ctl[p].before : &ctl[p].after;
      for (int k = 0; k < L_NP; ++k) out->v[k] = ledger_final_value<true>(k, v[k]);
      for (int k = 0; k < kLedgerI64; ++k) out->iq[k] = iq[k];
      if (mode == 0) {
        ledger_prologue(P.c, out, P.static_limit, &ctl[p].k);
        if (!ctl[p].k.done) atomicAdd(&g->active, 1);
      }
    }
  }
  if (mode != 0) return;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = (atomicAdd(&g->arrive, 1u) == gridDim.x - 1) ? 1 : 0;
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    const int active = *(volatile int*)&g->active;
    g->arrive = 0;
    g->active = 0;
    __threadfence();
    if (use_handle) cudaGraphSetConditional(handle, active > 0 ? 1u : 0u);
  }
}

// End of a substep round: one warp per still-active patch folds its item
// partials (fixed order) and advances the patch's loop control exactly as
// the single-grid last-block finalisation does.
__global__ void __launch_bounds__(kThreads)
    batch_round_kernel(int npatch, const BatchPatch* __restrict__ patches, BatchCtl* ctl,
                       const double* __restrict__ item_partials, BatchGlobal* g,
                       cudaGraphConditionalHandle handle, int use_handle) {
  __shared__ int last;
  const int lane = threadIdx.x & 31;
  const int p = blockIdx.x * (kThreads / 32) + (threadIdx.x >> 5);
  // the warp's lanes agree on the patch's state before lane 0 updates it
  int run = 0;
  if (p < npatch) run = __shfl_sync(0xffffffffu, lane == 0 ? !ctl[p].k.done : 0, 0);
  if (run) {
    const BatchPatch& P = patches[p];
    double v[kFvDiag + 1];
#pragma unroll
    for (int k = 0; k <= kFvDiag; ++k) v[k] = 0.0;
    for (int j = lane; j < P.n_items; j += 32) {
      const double* in = item_partials + (size_t)(P.first_item + j) * (kFvDiag + 1);
#pragma unroll
      for (int k = 0; k < kFvDiag; ++k) v[k] += in[k];
      v[kFvDiag] = fmax(v[kFvDiag], in[kFvDiag]);
    }
#pragma unroll
    for (int k = 0; k < kFvDiag; ++k) v[k] = warp_sum(v[k]);
    v[kFvDiag] = warp_max(v[kFvDiag]);
    if (lane == 0) {
      FvControl* k = &ctl[p].k;
      for (int i = 0; i < kFvDiag; ++i) k->diag[i] += v[i];
      k->substeps += 1;
      k->remaining -= k->sub_dt;
      k->parity ^= 1;
      k->wave = v[kFvDiag];
      if (!(k->remaining > 1.0e-14)) {
        k->done = 1;
      } else if (k->substeps >= P.c.max_substeps) {
        k->status = 2;  // SB_ERR_SUBSTEP_CAP
        k->done = 1;
      } else {
        plan_substep(P.c, k);
      }
      if (!k->done) atomicAdd(&g->active, 1);
    }
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = (atomicAdd(&g->arrive, 1u) == gridDim.x - 1) ? 1 : 0;
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    const int active = *(volatile int*)&g->active;
    g->arrive = 0;
    g->active = 0;
    __threadfence();
    if (use_handle) cudaGraphSetConditional(handle, active > 0 ? 1u : 0u);
  }
}

}  // namespace sb
