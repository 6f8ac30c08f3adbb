// Kernels that glue the plain terrain step into one CUDA graph.
//
// The reference takes every decision of the step on the host between blocking
// synchronisations (runtime/v2_physics_core.py:708-1003,
// runtime/gpu_large_avalanche.py:620-676).  Here the same decisions run in a
// single-thread device kernel between the graph's kernels: the large-avalanche
// classification and persistence, the frontier seeding flags and the
// residual-MiniSlope gate.
#pragma once

#include "sb_exchange.cuh"
#include "sb_labels.cuh"
#include "sb_ledger.cuh"
#include "sb_relax.cuh"

namespace sb {

struct PathConst {
  double dt;                  // unused in kernels (dt comes from the device copy)
  double f;                   // weight unit dx*dy/6
  double Q;
  double dx, dy;
  int min_cells;
  double min_area, min_volume, min_mean_excess_deg, persistence_time;
  double settled_volume, settled_speed, dry_tol;
  int residual_mode;          // 0 off, 1 gated as the reference, 2 always
  int fx;
};

// Device-resident state of the step pipeline (persistence across steps).
struct PathState {
  double persistence_s;
  double entrained_m3;
  double mean_excess_start_deg;
  double area_m2;
  double volume_m3;
  int has_previous;
  int candidate;
  int ready;
  int classification;         // 0 NO_LARGE_EVENT, 1 LOCAL_STATIC, 2 PERSISTING, 3 MOBILE_PATH
  int keep_candidate;
  int seed_frontier;
  int residual_enable;
  int pad;
};

// Per-step inputs of the fused step, written by the host into mapped pinned
// memory before each graph launch and read by the graph's first kernels over
// the host link (no copy-engine operations between steps).
struct alignas(16) PathInput {
  double dt;
  int count;  // cut command length
  int pad;
};

// Step start: dt and the cut command length from the host-mapped inputs into
// device copies, the Mobile V2 loop control for dt (fv_begin) and cleared
// exchange and labelling records.  One block.
__global__ void path_begin_kernel(FvControl* ctl, const PathInput* in, double* dt_dev,
                                  int* count_dev, ExchangeOut* xout, LabelOut* lout) {
  if (threadIdx.x == 0) {
    // one 16-byte read over the host link (each read there is a round trip
    // of about a microsecond): dt in the first word, the count in the low
    // half of the second
    const double2 v = __ldcv(reinterpret_cast<const double2*>(in));
    *dt_dev = v.x;
    *count_dev = (int)(unsigned)(__double_as_longlong(v.y) & 0xffffffffll);
    fv_begin_body(ctl, dt_dev);
  }
  unsigned* xw = reinterpret_cast<unsigned*>(xout);
  unsigned* lw = reinterpret_cast<unsigned*>(lout);
  for (int k = threadIdx.x; k < (int)(sizeof(ExchangeOut) / 4); k += blockDim.x) xw[k] = 0u;
  for (int k = threadIdx.x; k < (int)(sizeof(LabelOut) / 4); k += blockDim.x) lw[k] = 0u;
}

// Bucket-cut entrainment to target surfaces; the command length is read on
// the device so the graph is independent of it (mode 1 of entrain_kernel).
// idx / target are the host-mapped command (read once each, uncached).
template <bool FX>
__global__ void __launch_bounds__(kThreads)
    path_entrain_kernel(int ny, int nx, int pitch, double Q, double datum, double f,
                        typename FvTypes<FX>::B* __restrict__ b,
                        const typename FvTypes<FX>::B* __restrict__ z,
                        typename FvTypes<FX>::H* __restrict__ h0,
                        typename FvTypes<FX>::H* __restrict__ h1,
                        const FvControl* ctl, const int32_t* __restrict__ idx,
                        const double* __restrict__ target, const int* count_dev,
                        ExchangeOut* out, double* __restrict__ part) {
  const int count = *count_dev;
  typename FvTypes<FX>::H* h = ctl->parity ? h1 : h0;
  long long vq = 0;
  double vs = 0.0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x) {
    const int i = __ldcv(idx + k);
    const double tk = __ldcv(target + k);
    if (i < 0 || i >= ny * nx) {
      atomicExch(&out->bad_index, 1);
      continue;
    }
    const int r = i / nx, c = i % nx;
    const size_t gi = (size_t)r * pitch + c;
    const int w6 = vertex_weight6(r, c, ny, nx);
    if constexpr (FX) {
      const long long avail = (long long)b[gi] - (long long)z[gi];
      const long long req = (long long)b[gi] - (long long)rint((tk - datum) / Q);
      long long d = req < avail ? req : avail;
      if (d < 0) d = 0;
      b[gi] = (int32_t)(b[gi] - d);
      h[gi] = (int32_t)(h[gi] + d);
      vq += d * w6;
    } else {
      const double avail = fmax(b[gi] - z[gi], 0.0);
      const double d = fmin(fmax(b[gi] - tk, 0.0), avail);
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

// Step start and bucket-cut entrainment in one block, for commands of up to
// kPathStartCells cells: one thread reads dt and the command length from
// the host-mapped inputs (one 16-byte read), starts the Mobile V2 loop
// control and clears the labelling record; the block then entrains the
// command (four host-link loads in flight per thread) and writes the
// exchange record whole (block sums in a fixed order), so it needs no
// clearing beforehand.  The command's first kThreads * 4 entries are read
// together with the length (the buffers hold ``cap`` entries; those past the
// length are not used), so a command of up to 1024 cells costs one host-link
// round trip.  Same per-cell arithmetic as path_entrain_kernel.
constexpr int kPathStartCells = 4096;

template <bool FX>
__global__ void __launch_bounds__(kThreads)
    path_start_kernel(int ny, int nx, int pitch, double Q, double datum, double f,
                      typename FvTypes<FX>::B* __restrict__ b,
                      const typename FvTypes<FX>::B* __restrict__ z,
                      typename FvTypes<FX>::H* __restrict__ h0,
                      typename FvTypes<FX>::H* __restrict__ h1, FvControl* ctl,
                      const PathInput* in, double* dt_dev, const int32_t* __restrict__ idx,
                      const double* __restrict__ target, int cap, ExchangeOut* out,
                      LabelOut* lout) {
  __shared__ int s_count;
  __shared__ double fold[fold_words(1)];
  __shared__ long long ifold[fold_words(1)];
  constexpr int kInFlight = 4;
  int iv0[kInFlight];
  double tv0[kInFlight];
#pragma unroll
  for (int u = 0; u < kInFlight; ++u) {
    const int k = u * kThreads + threadIdx.x;
    iv0[u] = k < cap ? __ldcv(idx + k) : 0;
    tv0[u] = k < cap ? __ldcv(target + k) : 0.0;
  }
  if (threadIdx.x == 0) {
    const double2 v = __ldcv(reinterpret_cast<const double2*>(in));
    *dt_dev = v.x;
    s_count = (int)(unsigned)(__double_as_longlong(v.y) & 0xffffffffll);
    fv_begin_body(ctl, dt_dev);
  }
  unsigned* lw = reinterpret_cast<unsigned*>(lout);
  for (int k = threadIdx.x; k < (int)(sizeof(LabelOut) / 4); k += blockDim.x) lw[k] = 0u;
  __syncthreads();
  const int count = min(s_count, kPathStartCells);
  typename FvTypes<FX>::H* h = ctl->parity ? h1 : h0;
  long long vq = 0;
  double vs = 0.0;
  int bad = 0;
  for (int base = 0; base < count; base += kThreads * kInFlight) {
    int iv[kInFlight];
    double tv[kInFlight];
#pragma unroll
    for (int u = 0; u < kInFlight; ++u) {
      const int k = base + u * kThreads + threadIdx.x;
      if (base == 0) {
        iv[u] = iv0[u];
        tv[u] = tv0[u];
      } else {
        iv[u] = k < count ? __ldcv(idx + k) : 0;
        tv[u] = k < count ? __ldcv(target + k) : 0.0;
      }
    }
#pragma unroll
    for (int u = 0; u < kInFlight; ++u) {
      const int k = base + u * kThreads + threadIdx.x;
      if (k >= count) continue;
      const int i = iv[u];
      const double tk = tv[u];
      if (i < 0 || i >= ny * nx) {
        bad = 1;
        continue;
      }
      const int r = i / nx, c = i % nx;
      const size_t gi = (size_t)r * pitch + c;
      const int w6 = vertex_weight6(r, c, ny, nx);
      if constexpr (FX) {
        const long long avail = (long long)b[gi] - (long long)z[gi];
        const long long req = (long long)b[gi] - (long long)rint((tk - datum) / Q);
        long long d = req < avail ? req : avail;
        if (d < 0) d = 0;
        b[gi] = (int32_t)(b[gi] - d);
        h[gi] = (int32_t)(h[gi] + d);
        vq += d * w6;
      } else {
        const double avail = fmax(b[gi] - z[gi], 0.0);
        const double d = fmin(fmax(b[gi] - tk, 0.0), avail);
        b[gi] = b[gi] - d;
        h[gi] = h[gi] + d;
        vs += d * ((double)w6 * f);
      }
    }
  }
  const int any_bad = __syncthreads_or(bad);
  const long long iv1[1] = {vq};
  const double v1[1] = {vs};
  const long long* qt = block_fold<long long, 1, 1>(iv1, ifold);
  const double* st = block_fold<double, 1, 1>(v1, fold);
  if (threadIdx.x == 0) {
    out->volume_w6_quanta = qt[0];
    out->volume_w_fp64 = st[0];
    out->momentum_w[0] = 0.0;
    out->momentum_w[1] = 0.0;
    out->bad_index = any_bad ? 1 : 0;
    out->arrive = 0u;
  }
}

// Classification, persistence and gating (reference gpu_large_avalanche.py
// :620-676 and the residual gate of v2_physics_core.py:930-1003).
// One thread.
__device__ __forceinline__ void path_classify_body(const PathConst& c, const LabelOut* lo,
                                                   const StepIO* io, const ExchangeOut* xo,
                                                   PathState* ps, const double* dt_dev,
                                                   RelaxControl* rctl) {
  const double dt = *dt_dev;
  const int largest = lo->winner >= 0 ? lo->largest : 0;
  const double area = (double)lo->area6 * c.f;
  const double volume = c.fx ? (double)lo->volume * c.Q * c.f : (double)lo->volume / kVolumeScaleFp64 * c.f;
  const double mean_start =
      largest ? ((double)lo->exc_start / kExcessScale / (double)largest) * (180.0 / 3.141592653589793)
              : 0.0;
  const bool extent = largest >= c.min_cells && area >= c.min_area;
  const bool vol_pass = volume >= c.min_volume;
  const bool exc_pass = mean_start >= c.min_mean_excess_deg;
  const bool candidate = extent && vol_pass && exc_pass;
  const bool overlap = lo->prev_overlap > 0;
  if (candidate)
    ps->persistence_s = (overlap || !ps->has_previous) ? ps->persistence_s + dt : dt;
  else
    ps->persistence_s = 0.0;
  const bool ready = candidate && ps->persistence_s >= c.persistence_time;
  int cls = 0;
  if (ready) cls = 3;
  else if (candidate) cls = 2;
  else if (lo->total_unstable > 0) cls = 1;
  ps->candidate = candidate;
  ps->ready = ready;
  ps->classification = cls;
  ps->keep_candidate = candidate;
  ps->seed_frontier = cls == 1;
  ps->has_previous = candidate;
  ps->mean_excess_start_deg = mean_start;
  ps->area_m2 = area;
  ps->volume_m3 = volume;
  ps->entrained_m3 = c.fx ? (double)xo->volume_w6_quanta * c.Q * c.f : xo->volume_w_fp64;
  const LedgerOut& a = io->after;
  const double mobile_volume = c.fx ? (double)a.iq[1] * c.Q * c.f : a.v[L_HSUM_W] * c.f;
  const bool quiet = mobile_volume <= c.settled_volume && a.v[L_MAXSPEED] <= c.settled_speed;
  const bool yield_present = lo->total_unstable > 0 && volume > c.dry_tol * c.dx * c.dy;
  ps->residual_enable = c.residual_mode == 2 || (c.residual_mode == 1 && quiet && !yield_present);
  // frontier loop control for this step: a disabled residual leaves the
  // pending tile flags untouched for a later step (the reference keeps them queued)
  rctl->iterations = 0;
  rctl->done = ps->residual_enable ? 0 : 1;
  rctl->converged = 0;
  rctl->status = 0;
  rctl->max_excess_bits = 0;
  rctl->arrive = 0;
  rctl->parity = 0;
  rctl->n_active = 0;
  rctl->rounds = 0;
  rctl->moved_edges = 0;
  rctl->list_len = 0;
  rctl->sub_len = 0;
}

// The component reduction and, in the thread that finishes it, the
// classification: one node of the step graph instead of two.
__global__ void __launch_bounds__(kThreads)
    path_reduce_classify_kernel(LabelRoots roots, const int* __restrict__ root_list, LabelOut* lo,
                                unsigned int* arrive, const PathConst c, const StepIO* io,
                                const ExchangeOut* xo, PathState* ps, const double* dt_dev,
                                RelaxControl* rctl) {
  if (label_reduce_body(roots, root_list, lo, arrive)) {
    __threadfence();
    path_classify_body(c, lo, io, xo, ps, dt_dev, rctl);
  }
}

// Previous-candidate mask and frontier seeds of the winner; the last block
// to finish then opens the residual frontier loop (frontier_begin).
__global__ void __launch_bounds__(kThreads)
    path_update_previous_kernel(const LabelConst c, const int* __restrict__ parent,
                                int* __restrict__ previous, int* __restrict__ reached,
                                int* __restrict__ tile_flags, const LabelOut* out,
                                const PathState* ps, const RelaxConst rc, int* __restrict__ phase0,
                                int* __restrict__ phase1, RelaxControl* rctl,
                                cudaGraphConditionalHandle handle) {
  __shared__ int last;
  const int n = c.ny * c.nx;
  const int winner = out->winner;
  const int keep = ps->keep_candidate, seed = ps->seed_frontier;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const bool belongs = winner >= 0 && parent[i] == winner;
    previous[i] = (belongs && keep) ? 1 : 0;
    if (belongs && seed) {
      const int r = i / c.nx, col = i % c.nx;
      reached[(size_t)r * c.pitch + col] = 1;
      tile_flags[(r / c.tile_size) * c.frontier_tiles_x + col / c.tile_size] = 1;
    }
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = (atomicAdd(&rctl->arrive, 1u) == gridDim.x - 1) ? 1 : 0;
  __syncthreads();
  if (!last) return;
  __threadfence();
  if (threadIdx.x == 0) rctl->arrive = 0;
  frontier_begin_body(rc, tile_flags, phase0, phase1, rctl, handle);
}

// Step end: the step's records into the caller-visible pinned host copies
// (device-mapped pointers, one launch instead of one copy per record), and the
// reached mask cleared after a converged residual (frontier_finish).
struct PathRecordPtrs {
  const void* src[6];
  void* dst[6];
  int bytes[6];
};

__global__ void __launch_bounds__(kThreads)
    path_records_kernel(const PathRecordPtrs p, const RelaxConst rc, int* __restrict__ reached,
                        const RelaxControl* rctl) {
  if (blockIdx.x == 0) {
    for (int k = 0; k < 6; ++k) {
      const unsigned* s = static_cast<const unsigned*>(p.src[k]);
      unsigned* d = static_cast<unsigned*>(p.dst[k]);
      for (int w = threadIdx.x; w < p.bytes[k] / 4; w += blockDim.x) d[w] = __ldcg(s + w);
    }
    __threadfence_system();
  }
  if (!rctl->converged) return;
  const long long n = (long long)rc.n0 * rc.pitch;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    reached[i] = 0;
}

// The standalone Mobile V2 step graph's ends: dt from the host-mapped input
// into the device copy + loop control (one thread), and the step records to
// mapped host memory (one block), so a step issues no copy-engine operation.
__global__ void fv_begin_mapped_kernel(FvControl* ctl, const double* dt_mapped, double* dt_dev) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    *dt_dev = __ldcv(dt_mapped);
    fv_begin_body(ctl, dt_dev);
  }
}

__global__ void records_copy_kernel(const PathRecordPtrs p, int n) {
  for (int k = 0; k < n; ++k) {
    const unsigned* s = static_cast<const unsigned*>(p.src[k]);
    unsigned* d = static_cast<unsigned*>(p.dst[k]);
    for (int w = threadIdx.x; w < p.bytes[k] / 4; w += blockDim.x) d[w] = __ldcg(s + w);
  }
  __threadfence_system();
}

}  // namespace sb
