// Repose (MiniSlope) relaxation kernels.
//
// Arrays are generic 2-D fields whose axis 0 (rows) uses spacing s0 and axis 1
// (columns) spacing s1, the convention of the reference's
// ``relax_critical_slope(height, grid_spacing)`` (slope_model.py:273-343).
// Direction order and parity rule follow ``_neighbor_pairs`` (:744-750): for
// (d0, d1) in ((1,0,s0), (0,1,s1), (1,1,hyp), (1,-1,hyp)), parity on the
// axis-0 coordinate of endpoint a when d0 != 0, else on its axis-1 coordinate.
//
// relax_full_kernel      -- one full-domain iteration (8 colour sub-phases) per
//                           launch with temporal blocking: a (T+2*8)^2 halo
//                           box is TMA-loaded into shared memory, all eight
//                           sub-phases run there (the exact region shrinks by
//                           one cell per sub-phase), the T^2 interior is
//                           written back; the iteration's max excess (over all
//                           pairs of each sub-phase, before its update) feeds
//                           the convergence test on the device.
// frontier_*_kernel      -- production compact-frontier rounds
//                           (runtime/v2_physics_core.py:1172-1254 over
//                           solvers/warp_compact_frontier.py:56-130): the
//                           round's active tiles compacted into a list with
//                           warp ballots, a fixed grid striding over the list,
//                           reached-gated weighted transfers, tile activation
//                           of the 3x3 cell stencil around moved endpoints
//                           (appended to the list), final scan -> next active
//                           tiles.
#pragma once

#include <climits>

#include "sb_common.cuh"
#include "sb_fv.cuh"

namespace sb {

constexpr int kRelaxTile = 32;
constexpr int kRelaxHalo = 8;
constexpr int kRelaxBox = kRelaxTile + 2 * kRelaxHalo;  // 48

struct RelaxConst {
  int n0, n1, pitch, tiles1, ntiles;
  double s0, s1;
  double crit[4];       // tan(angle) * L per direction
  double crit_q[4];     // FX: crit / Q
  double tol, tol_q;
  int max_iterations;
  int weighted;         // frontier: Triangle-A-C vertex weights (else uniform)
  int ftile;            // frontier tile size
  double f;             // weight unit s0*s1/6
};

struct RelaxControl {
  int iterations;
  int done;
  int converged;
  int status;
  unsigned long long max_excess_bits;  // double bits of this iteration's max excess
  unsigned int arrive;
  int parity;        // buffer holding the current field (full relax)
  int n_active;      // frontier: active tiles at the start of the last round
  int rounds;
  int moved_edges;
  int confirm;       // reached-gated sweep: 1 while the confirming scan is pending
  int bb[4];         // reached-gated sweep: bounding box of reached cells (min0, max0, min1, max1)
  int list_len;      // frontier: tiles in this round's compacted phase-tile list
  int sub_len;       // frontier: list entries the current sub-phase / scan processes
};

__device__ __forceinline__ void dir_of(int d, int& d0, int& d1) {
  d0 = d == 1 ? 0 : 1;
  d1 = d == 0 ? 0 : (d == 3 ? -1 : 1);
}

// ------------------------------------------------------------------------
// Full-domain relaxation (one iteration per launch).
// ------------------------------------------------------------------------
template <bool FX>
__global__ void __launch_bounds__(kThreads)
    relax_full_kernel(const RelaxConst c, const __grid_constant__ CUtensorMap tm0,
                      const __grid_constant__ CUtensorMap tm1,
                      typename FvTypes<FX>::H* __restrict__ f0,
                      typename FvTypes<FX>::H* __restrict__ f1, RelaxControl* ctl,
                      cudaGraphConditionalHandle handle, int use_handle) {
  using H = typename FvTypes<FX>::H;
  __shared__ alignas(128) H s[kRelaxBox * kRelaxBox];
  __shared__ alignas(8) uint64_t bar;
  __shared__ double red[kThreads / 32];
  __shared__ int last;
  if (*(volatile int*)&ctl->done) return;
  const int parity_buf = ctl->parity;
  const int t1 = blockIdx.x % c.tiles1, t0 = blockIdx.x / c.tiles1;
  const int g0 = t0 * kRelaxTile - kRelaxHalo, g1 = t1 * kRelaxTile - kRelaxHalo;
  if (threadIdx.x == 0) mbar_init(&bar, 1);
  __syncthreads();
  if (threadIdx.x == 0) {
    mbar_expect_tx(&bar, kRelaxBox * kRelaxBox * (unsigned)sizeof(H));
    tma_load_2d(s, parity_buf ? &tm1 : &tm0, g1, g0, &bar);
  }
  const bool loaded = mbar_wait(&bar, 0);
  // a box wholly inside the domain needs no domain checks
  const bool inner = g0 >= 0 && g1 >= 0 && g0 + kRelaxBox <= c.n0 && g1 + kRelaxBox <= c.n1;
  double worst = 0.0;
  for (int d = 0; d < 4; ++d) {
    int d0, d1;
    dir_of(d, d0, d1);
    for (int par = 0; par < 2; ++par) {
      // (1) max excess, before this sub-phase's update, over the pairs owned by
      // the interior whose endpoint a has the inactive parity (those of the
      // active parity are taken in (2) as they are read, before their update)
      constexpr int kHalfTile = kRelaxTile / 2;
      const int ifirst = d0 ? ((1 - par - g0) & 1) : ((1 - par - g1) & 1);
      for (int k = threadIdx.x; k < kHalfTile * kRelaxTile; k += kThreads) {
        const int la0 = kRelaxHalo + (d0 ? ifirst + 2 * (k / kRelaxTile) : k / kHalfTile);
        const int la1 = kRelaxHalo + (d0 ? k % kRelaxTile : ifirst + 2 * (k % kHalfTile));
        const int a0 = g0 + la0, a1 = g1 + la1, b0 = a0 + d0, b1 = a1 + d1;
        if (a0 >= c.n0 || a1 >= c.n1 || b0 >= c.n0 || b1 < 0 || b1 >= c.n1) continue;
        const int ia = la0 * kRelaxBox + la1, ib = (la0 + d0) * kRelaxBox + la1 + d1;
        double ex;
        if constexpr (FX) {
          const long long df = (long long)s[ia] - (long long)s[ib];
          ex = (double)(df < 0 ? -df : df) - c.crit_q[d];  // in quanta
        } else {
          ex = fmax(fabs(s[ia] - s[ib]) - c.crit[d], 0.0);
        }
        worst = fmax(worst, ex);
      }
      __syncthreads();
      // (2) Jacobi update of the active-parity pairs inside the box: only the
      // rows (d0 != 0) or columns (d0 == 0) whose global index has parity
      // par hold an active endpoint a.  Sub-phase i (0-7) only needs pairs
      // with endpoint a in [i, kRelaxBox - i) on both axes: every pair that
      // touches a cell still exact after it (distance > i from the box edge)
      // has a there, and its inputs are exact (distance >= i).
      if (loaded) {
        const int lo = d * 2 + par, hi = kRelaxBox - lo, span = hi - lo;
        const int first = d0 ? ((par - g0) & 1) : ((par - g1) & 1);
        const int start = lo + ((first - lo) & 1);  // first line of the parity in [lo, hi)
        const int lines = (hi - start + 1) >> 1;
        // k / ncol by a multiply and shift (exact for k < 2^20 / 48)
        const int ncol = d0 ? span : lines;
        const unsigned inv = ((1u << 20) + (unsigned)ncol - 1u) / (unsigned)ncol;
        for (int k = threadIdx.x; k < lines * span; k += kThreads) {
          const int q = (int)(((unsigned)k * inv) >> 20), rem = k - q * ncol;
          int la0, la1;
          if (d0) {
            la0 = start + 2 * q;
            la1 = lo + rem;
          } else {
            la0 = lo + q;
            la1 = start + 2 * rem;
          }
          const int lb0 = la0 + d0, lb1 = la1 + d1;
          if (lb0 >= kRelaxBox || lb1 < 0 || lb1 >= kRelaxBox) continue;
          const int a0 = g0 + la0, a1 = g1 + la1, b0 = a0 + d0, b1 = a1 + d1;
          if (!inner) {
            if (a0 < 0 || a1 < 0 || a0 >= c.n0 || a1 >= c.n1) continue;
            if (b0 >= c.n0 || b1 < 0 || b1 >= c.n1) continue;
          }
          const int ia = la0 * kRelaxBox + la1, ib = lb0 * kRelaxBox + lb1;
          const bool owned = la0 >= kRelaxHalo && la0 < kRelaxHalo + kRelaxTile &&
                             la1 >= kRelaxHalo && la1 < kRelaxHalo + kRelaxTile;
          if constexpr (FX) {
            const long long df = (long long)s[ia] - (long long)s[ib];
            const double ex = (double)(df < 0 ? -df : df) - c.crit_q[d];
            if (owned) worst = fmax(worst, ex);
            if (ex > 0.0) {
              const long long t = (long long)ceil(ex * 0.5);
              const long long st = df < 0 ? -t : t;
              s[ia] = (H)(s[ia] - st);
              s[ib] = (H)(s[ib] + st);
            }
          } else {
            const double diff = s[ia] - s[ib];
            const double ex = fmax(fabs(diff) - c.crit[d], 0.0);
            if (owned) worst = fmax(worst, ex);
            const double sg = diff > 0.0 ? 1.0 : (diff < 0.0 ? -1.0 : 0.0);
            const double t = 0.5 * ex * sg;
            s[ia] = s[ia] - t;
            s[ib] = s[ib] + t;
          }
        }
      }
      __syncthreads();
    }
  }
  // write back the interior into the other buffer
  H* dst = parity_buf ? f0 : f1;
  for (int k = threadIdx.x; k < kRelaxTile * kRelaxTile; k += kThreads) {
    const int la0 = kRelaxHalo + k / kRelaxTile, la1 = kRelaxHalo + k % kRelaxTile;
    const int a0 = g0 + la0, a1 = g1 + la1;
    if (a0 < c.n0 && a1 < c.n1 && loaded) dst[(size_t)a0 * c.pitch + a1] = s[la0 * kRelaxBox + la1];
  }
  worst = warp_max(worst);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = worst;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0.0;
    for (int w = 0; w < kThreads / 32; ++w) m = fmax(m, red[w]);
    if (!loaded) atomicExch(&ctl->status, 6);
    atomicMax(&ctl->max_excess_bits, (unsigned long long)__double_as_longlong(m));
    __threadfence();
    last = atomicAdd(&ctl->arrive, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last || threadIdx.x != 0) return;
  __threadfence();
  const double m = __longlong_as_double((long long)ctl->max_excess_bits);
  ctl->arrive = 0;
  ctl->max_excess_bits = 0;
  ctl->iterations += 1;
  ctl->parity = parity_buf ^ 1;
  if (ctl->status) {
    ctl->done = 1;
  } else if (m <= (FX ? c.tol_q : c.tol)) {
    ctl->converged = 1;
    ctl->done = 1;
  } else if (ctl->iterations >= c.max_iterations) {
    ctl->done = 1;
  }
  __threadfence();
  if (use_handle) cudaGraphSetConditional(handle, ctl->done ? 0u : 1u);
}

// ------------------------------------------------------------------------
// Reached-gated full-domain iteration: the event-driven reached-bbox
// MiniSlope backend (EventDrivenMinimumSlopeAdapter._relax_dynamic_frontier,
// solvers/event_driven_slope.py:166-302).
//
// Same temporal blocking as relax_full_kernel (48^2 box, 8 sub-phases in
// shared memory, 32^2 interior written back), plus the reached mask staged
// in a second TMA box: a pair moves only if one endpoint is reached, both
// endpoints of a moved pair become reached (the mask can spread one cell per
// sub-phase, so the 8-cell halo stays exact), and the iteration maximum takes
// only reachable pairs.  A box that holds no reached cell when its CTA starts
// cannot change its interior within one iteration, so CTAs whose box misses
// the reached bounding box (grown with atomics, never shrunk) skip the
// iteration; both ping-pong buffers hold the same values for such tiles
// (begin kernel), so nothing needs writing.  An iteration whose maximum is
// <= tolerance is followed by a confirming scan of all reachable pairs on the
// post-iteration state (no update, not counted); the solve ends when that
// scan is <= tolerance too, otherwise the iterations continue.
// ------------------------------------------------------------------------
template <bool FX>
__global__ void __launch_bounds__(kThreads)
    relax_reached_kernel(const RelaxConst c, const __grid_constant__ CUtensorMap tm0,
                         const __grid_constant__ CUtensorMap tm1,
                         const __grid_constant__ CUtensorMap tr0,
                         const __grid_constant__ CUtensorMap tr1,
                         typename FvTypes<FX>::H* __restrict__ f0,
                         typename FvTypes<FX>::H* __restrict__ f1, int* __restrict__ r0,
                         int* __restrict__ r1, RelaxControl* ctl,
                         cudaGraphConditionalHandle handle, int use_handle) {
  using H = typename FvTypes<FX>::H;
  __shared__ alignas(128) H s[kRelaxBox * kRelaxBox];
  __shared__ alignas(128) int rs[kRelaxBox * kRelaxBox];
  __shared__ alignas(8) uint64_t bar;
  __shared__ double red[kThreads / 32];
  __shared__ int bbs[4];
  __shared__ int last;
  if (*(volatile int*)&ctl->done) return;
  const int parity_buf = ctl->parity;
  const int confirm = ctl->confirm;
  const int t1 = blockIdx.x % c.tiles1, t0 = blockIdx.x / c.tiles1;
  const int g0 = t0 * kRelaxTile - kRelaxHalo, g1 = t1 * kRelaxTile - kRelaxHalo;
  const volatile int* vb = ctl->bb;
  const int bmin0 = vb[0], bmax0 = vb[1], bmin1 = vb[2], bmax1 = vb[3];
  const bool work = bmin0 <= bmax0 && bmax0 >= g0 && bmin0 < g0 + kRelaxBox && bmax1 >= g1 &&
                    bmin1 < g1 + kRelaxBox;  // block-uniform
  double worst = 0.0;
  bool loaded = true;
  if (work) {
    if (threadIdx.x == 0) {
      mbar_init(&bar, 1);
      bbs[0] = INT_MAX;
      bbs[1] = INT_MIN;
      bbs[2] = INT_MAX;
      bbs[3] = INT_MIN;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      mbar_expect_tx(&bar, kRelaxBox * kRelaxBox * (unsigned)(sizeof(H) + sizeof(int)));
      tma_load_2d(s, parity_buf ? &tm1 : &tm0, g1, g0, &bar);
      tma_load_2d(rs, parity_buf ? &tr1 : &tr0, g1, g0, &bar);
    }
    loaded = mbar_wait(&bar, 0);
    if (confirm) {
      // all reachable pairs owned by the interior, every direction, no update
      for (int d = 0; d < 4 && loaded; ++d) {
        int d0, d1;
        dir_of(d, d0, d1);
        for (int k = threadIdx.x; k < kRelaxTile * kRelaxTile; k += kThreads) {
          const int la0 = kRelaxHalo + k / kRelaxTile, la1 = kRelaxHalo + k % kRelaxTile;
          const int a0 = g0 + la0, a1 = g1 + la1, b0 = a0 + d0, b1 = a1 + d1;
          if (a0 >= c.n0 || a1 >= c.n1 || b0 >= c.n0 || b1 < 0 || b1 >= c.n1) continue;
          const int ia = la0 * kRelaxBox + la1, ib = (la0 + d0) * kRelaxBox + la1 + d1;
          if (!(rs[ia] | rs[ib])) continue;
          double ex;
          if constexpr (FX) {
            const long long df = (long long)s[ia] - (long long)s[ib];
            ex = (double)(df < 0 ? -df : df) - c.crit_q[d];
          } else {
            ex = fabs(s[ia] - s[ib]) - c.crit[d];
          }
          worst = fmax(worst, ex);
        }
      }
    } else {
      for (int d = 0; d < 4; ++d) {
        int d0, d1;
        dir_of(d, d0, d1);
        for (int par = 0; par < 2; ++par) {
          // (1) reachable inactive-parity pairs owned by the interior, before
          // this sub-phase's update
          constexpr int kHalfTile = kRelaxTile / 2;
          const int ifirst = d0 ? ((1 - par - g0) & 1) : ((1 - par - g1) & 1);
          for (int k = threadIdx.x; k < kHalfTile * kRelaxTile; k += kThreads) {
            const int la0 = kRelaxHalo + (d0 ? ifirst + 2 * (k / kRelaxTile) : k / kHalfTile);
            const int la1 = kRelaxHalo + (d0 ? k % kRelaxTile : ifirst + 2 * (k % kHalfTile));
            const int a0 = g0 + la0, a1 = g1 + la1, b0 = a0 + d0, b1 = a1 + d1;
            if (a0 >= c.n0 || a1 >= c.n1 || b0 >= c.n0 || b1 < 0 || b1 >= c.n1) continue;
            const int ia = la0 * kRelaxBox + la1, ib = (la0 + d0) * kRelaxBox + la1 + d1;
            if (!(rs[ia] | rs[ib])) continue;
            double ex;
            if constexpr (FX) {
              const long long df = (long long)s[ia] - (long long)s[ib];
              ex = (double)(df < 0 ? -df : df) - c.crit_q[d];
            } else {
              ex = fmax(fabs(s[ia] - s[ib]) - c.crit[d], 0.0);
            }
            worst = fmax(worst, ex);
          }
          __syncthreads();
          // (2) gated Jacobi update of the active-parity pairs inside the box
          if (loaded) {
            constexpr int kHalf = kRelaxBox / 2;
            const int first = d0 ? ((par - g0) & 1) : ((par - g1) & 1);
            for (int k = threadIdx.x; k < kHalf * kRelaxBox; k += kThreads) {
              int la0, la1;
              if (d0) {
                la0 = first + 2 * (k / kRelaxBox);
                la1 = k % kRelaxBox;
              } else {
                la0 = k / kHalf;
                la1 = first + 2 * (k % kHalf);
              }
              const int lb0 = la0 + d0, lb1 = la1 + d1;
              if (lb0 >= kRelaxBox || lb1 < 0 || lb1 >= kRelaxBox) continue;
              const int a0 = g0 + la0, a1 = g1 + la1, b0 = a0 + d0, b1 = a1 + d1;
              if (a0 < 0 || a1 < 0 || a0 >= c.n0 || a1 >= c.n1) continue;
              if (b0 >= c.n0 || b1 < 0 || b1 >= c.n1) continue;
              const int ia = la0 * kRelaxBox + la1, ib = lb0 * kRelaxBox + lb1;
              if (!(rs[ia] | rs[ib])) continue;
              const bool owned = la0 >= kRelaxHalo && la0 < kRelaxHalo + kRelaxTile &&
                                 la1 >= kRelaxHalo && la1 < kRelaxHalo + kRelaxTile;
              if constexpr (FX) {
                const long long df = (long long)s[ia] - (long long)s[ib];
                const double ex = (double)(df < 0 ? -df : df) - c.crit_q[d];
                if (owned) worst = fmax(worst, ex);
                if (ex > 0.0) {
                  const long long t = (long long)ceil(ex * 0.5);
                  const long long st = df < 0 ? -t : t;
                  s[ia] = (H)(s[ia] - st);
                  s[ib] = (H)(s[ib] + st);
                  rs[ia] = 1;
                  rs[ib] = 1;
                }
              } else {
                const double diff = s[ia] - s[ib];
                const double ex = fmax(fabs(diff) - c.crit[d], 0.0);
                if (owned) worst = fmax(worst, ex);
                if (ex > 0.0) {
                  const double sg = diff > 0.0 ? 1.0 : (diff < 0.0 ? -1.0 : 0.0);
                  const double t = 0.5 * ex * sg;
                  s[ia] = s[ia] - t;
                  s[ib] = s[ib] + t;
                  rs[ia] = 1;
                  rs[ib] = 1;
                }
              }
            }
          }
          __syncthreads();
        }
      }
      // write back the interior (heights and reached) into the other buffers,
      // and grow the reached bounding box by the interior's reached cells
      H* dst = parity_buf ? f0 : f1;
      int* rdst = parity_buf ? r0 : r1;
      int lo0 = INT_MAX, hi0 = INT_MIN, lo1 = INT_MAX, hi1 = INT_MIN;
      for (int k = threadIdx.x; k < kRelaxTile * kRelaxTile; k += kThreads) {
        const int la0 = kRelaxHalo + k / kRelaxTile, la1 = kRelaxHalo + k % kRelaxTile;
        const int a0 = g0 + la0, a1 = g1 + la1;
        if (a0 < c.n0 && a1 < c.n1 && loaded) {
          const int li = la0 * kRelaxBox + la1;
          dst[(size_t)a0 * c.pitch + a1] = s[li];
          rdst[(size_t)a0 * c.pitch + a1] = rs[li];
          if (rs[li]) {
            lo0 = min(lo0, a0);
            hi0 = max(hi0, a0);
            lo1 = min(lo1, a1);
            hi1 = max(hi1, a1);
          }
        }
      }
      if (lo0 <= hi0) {
        atomicMin(&bbs[0], lo0);
        atomicMax(&bbs[1], hi0);
        atomicMin(&bbs[2], lo1);
        atomicMax(&bbs[3], hi1);
      }
      __syncthreads();
      if (threadIdx.x == 0 && bbs[0] <= bbs[1]) {
        atomicMin(&ctl->bb[0], bbs[0]);
        atomicMax(&ctl->bb[1], bbs[1]);
        atomicMin(&ctl->bb[2], bbs[2]);
        atomicMax(&ctl->bb[3], bbs[3]);
      }
    }
  }
  worst = warp_max(worst);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = worst;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0.0;
    for (int w = 0; w < kThreads / 32; ++w) m = fmax(m, red[w]);
    if (!loaded) atomicExch(&ctl->status, 6);
    atomicMax(&ctl->max_excess_bits, (unsigned long long)__double_as_longlong(m));
    __threadfence();
    last = atomicAdd(&ctl->arrive, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last || threadIdx.x != 0) return;
  __threadfence();
  const double m = __longlong_as_double((long long)ctl->max_excess_bits);
  const double tol = FX ? c.tol_q : c.tol;
  ctl->arrive = 0;
  ctl->max_excess_bits = 0;
  if (ctl->status) {
    ctl->done = 1;
  } else if (confirm) {
    if (m <= tol) {
      ctl->converged = 1;
      ctl->done = 1;
    }
    ctl->confirm = 0;
  } else {
    ctl->iterations += 1;
    ctl->parity = parity_buf ^ 1;
    if (m <= tol) ctl->confirm = 1;
  }
  // the safety cap: a next iteration beyond max_iterations is an error
  if (!ctl->done && !ctl->confirm && ctl->iterations >= c.max_iterations) {
    ctl->status = 4;  // SB_ERR_NONCONVERGENCE
    ctl->done = 1;
  }
  __threadfence();
  if (use_handle) cudaGraphSetConditional(handle, ctl->done ? 0u : 1u);
}

// Start of a reached-gated solve: loop control reset, both ping-pong buffers
// made equal (heights and reached) and the reached bounding box from the seeds.
template <bool FX>
__global__ void __launch_bounds__(kThreads)
    relax_reached_begin_kernel(const RelaxConst c, const typename FvTypes<FX>::H* __restrict__ f0,
                               typename FvTypes<FX>::H* __restrict__ f1,
                               const int* __restrict__ r0, int* __restrict__ r1,
                               RelaxControl* ctl) {
  __shared__ int bbs[4];
  if (threadIdx.x == 0) {
    bbs[0] = INT_MAX;
    bbs[1] = INT_MIN;
    bbs[2] = INT_MAX;
    bbs[3] = INT_MIN;
  }
  __syncthreads();
  int lo0 = INT_MAX, hi0 = INT_MIN, lo1 = INT_MAX, hi1 = INT_MIN;
  const long long n = (long long)c.n0 * c.n1;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int a0 = (int)(i / c.n1), a1 = (int)(i % c.n1);
    const size_t gi = (size_t)a0 * c.pitch + a1;
    f1[gi] = f0[gi];
    const int r = r0[gi] != 0;
    r1[gi] = r;
    if (r) {
      lo0 = min(lo0, a0);
      hi0 = max(hi0, a0);
      lo1 = min(lo1, a1);
      hi1 = max(hi1, a1);
    }
  }
  if (lo0 <= hi0) {
    atomicMin(&bbs[0], lo0);
    atomicMax(&bbs[1], hi0);
    atomicMin(&bbs[2], lo1);
    atomicMax(&bbs[3], hi1);
  }
  __syncthreads();
  if (threadIdx.x == 0 && bbs[0] <= bbs[1]) {
    atomicMin(&ctl->bb[0], bbs[0]);
    atomicMax(&ctl->bb[1], bbs[1]);
    atomicMin(&ctl->bb[2], bbs[2]);
    atomicMax(&ctl->bb[3], bbs[3]);
  }
}

// ------------------------------------------------------------------------
// Compact frontier rounds (production schedule).
// ------------------------------------------------------------------------
__device__ __forceinline__ double vertex_weight_fp64(int r, int col, int n0, int n1, double f) {
  double w = 0.0;
  if (r < n0 - 1 && col < n1 - 1) w += 2.0 * f;
  if (r < n0 - 1 && col > 0) w += f;
  if (r > 0 && col > 0) w += 2.0 * f;
  if (r > 0 && col < n1 - 1) w += f;
  return w;
}

__device__ __forceinline__ long long gcd_ll(long long a, long long b) {
  while (b) {
    const long long t = a % b;
    a = b;
    b = t;
  }
  return a;
}

// Round start: the pending tile flags (scan results and seeds) are compacted
// into this round's tile list with warp ballots -- one atomicAdd per warp on a
// shared counter, each active lane writing its tile at the warp's base plus the
// count of active lanes below it -- and become the round's membership flags;
// the flags are cleared for the next round.  Decides termination.  Body for
// one block of kThreads threads (the list order is irrelevant: tiles of one
// sub-phase never share a pair endpoint).
__device__ __forceinline__ void frontier_begin_body(const RelaxConst& c, int* __restrict__ unstable,
                                                    int* __restrict__ member,
                                                    int* __restrict__ list, RelaxControl* ctl,
                                                    cudaGraphConditionalHandle handle) {
  __shared__ int count;
  if (*(volatile int*)&ctl->done) {  // loop disabled before it started: keep the flags
    if (threadIdx.x == 0) cudaGraphSetConditional(handle, 0u);
    return;
  }
  if (threadIdx.x == 0) count = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  for (int base = 0; base < c.ntiles; base += blockDim.x) {  // uniform trip count
    const int t = base + threadIdx.x;
    int a = 0;
    if (t < c.ntiles) {
      a = unstable[t] != 0;
      member[t] = a;
      unstable[t] = 0;
    }
    const unsigned mask = __ballot_sync(0xffffffffu, a);
    int off = 0;
    if (lane == 0 && mask) off = atomicAdd(&count, __popc(mask));
    off = __shfl_sync(0xffffffffu, off, 0);
    if (a) list[off + __popc(mask & ((1u << lane) - 1u))] = t;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int tot = count;
    ctl->n_active = tot;
    ctl->list_len = tot;
    ctl->sub_len = tot;
    if (tot == 0) {
      ctl->converged = 1;
      ctl->done = 1;
    } else if (ctl->rounds >= c.max_iterations) {
      ctl->status = 4;  // NONCONVERGENCE
      ctl->done = 1;
    } else {
      ctl->rounds += 1;
    }
    __threadfence();
    cudaGraphSetConditional(handle, ctl->done ? 0u : 1u);
  }
}

__global__ void frontier_begin_kernel(const RelaxConst c, int* __restrict__ unstable,
                                      int* __restrict__ member, int* __restrict__ list,
                                      RelaxControl* ctl, cudaGraphConditionalHandle handle) {
  frontier_begin_body(c, unstable, member, list, ctl, handle);
}

// One colour sub-phase over the round's compacted tile list: a fixed grid of
// CTAs strides over the first ctl->sub_len entries (the tiles active when the
// sub-phase starts), one 32 x T tile per entry.  Tiles of the 3x3 cell stencil
// around moved endpoints join the list (membership flag taken by atomicExch,
// so each tile is appended once per round) and are processed from the next
// sub-phase on; the last CTA publishes the new length.
template <bool FX>
__global__ void __launch_bounds__(kThreads)
    frontier_subphase_kernel(const RelaxConst c, int dir, int par,
                             typename FvTypes<FX>::H* __restrict__ hfield,
                             int* __restrict__ reached, int* __restrict__ member,
                             int* __restrict__ list, RelaxControl* ctl) {
  using H = typename FvTypes<FX>::H;
  __shared__ int trig[9];
  __shared__ int moved_count;
  __shared__ int last;
  if (*(volatile int*)&ctl->done) return;  // uniform across the grid
  const int len = *(volatile int*)&ctl->sub_len;
  const int T = c.ftile;
  int d0, d1;
  dir_of(dir, d0, d1);
  int moved_total = 0;
  for (int e = blockIdx.x; e < len; e += gridDim.x) {
    const int t = list[e];
    const int tr = t / c.tiles1, tc = t % c.tiles1;
    if (threadIdx.x < 9) trig[threadIdx.x] = 0;
    __syncthreads();
    int moved = 0;
    // only the tile's rows (d0 != 0) or columns (d0 == 0) of parity par hold an
    // active endpoint a: enumerate those lines alone
    const int first = d0 ? ((par - tr * T) & 1) : ((par - tc * T) & 1);
    const int half = (T - first + 1) / 2;
    for (int k = threadIdx.x; k < half * T; k += kThreads) {
      int la0, la1;
      if (d0) {
        la0 = first + 2 * (k / T);
        la1 = k % T;
      } else {
        la0 = k / half;
        la1 = first + 2 * (k % half);
      }
      const int a0 = tr * T + la0, a1 = tc * T + la1;
      const int b0 = a0 + d0, b1 = a1 + d1;
      if (a0 >= c.n0 || a1 >= c.n1 || b0 >= c.n0 || b1 < 0 || b1 >= c.n1) continue;
      const size_t ia = (size_t)a0 * c.pitch + a1, ib = (size_t)b0 * c.pitch + b1;
      if (!reached[ia] && !reached[ib]) continue;
      bool did = false;
      if constexpr (FX) {
        const long long df = (long long)hfield[ia] - (long long)hfield[ib];
        const double ex = (double)(df < 0 ? -df : df) - c.crit_q[dir];
        if (ex > 0.0) {
          long long ua = 1, ub = 1;
          if (c.weighted) {
            const long long wa = vertex_weight6(a0, a1, c.n0, c.n1);
            const long long wb = vertex_weight6(b0, b1, c.n0, c.n1);
            const long long g = gcd_ll(wa, wb);
            ua = wb / g;
            ub = wa / g;
          }
          const long long kk = (long long)ceil(ex / (double)(ua + ub));
          const long long sg = df < 0 ? -1 : 1;
          hfield[ia] = (H)(hfield[ia] - sg * kk * ua);
          hfield[ib] = (H)(hfield[ib] + sg * kk * ub);
          did = true;
        }
      } else {
        const double diff = hfield[ia] - hfield[ib];
        const double ex = fabs(diff) - c.crit[dir];
        if (ex > 0.0) {
          const double signed_ex = diff < 0.0 ? -ex : ex;
          double wa = 1.0, wb = 1.0;
          if (c.weighted) {
            wa = vertex_weight_fp64(a0, a1, c.n0, c.n1, c.f);
            wb = vertex_weight_fp64(b0, b1, c.n0, c.n1, c.f);
          }
          const double ws = wa + wb;
          const double ta = signed_ex * wb / ws, tb = signed_ex * wa / ws;
          hfield[ia] = hfield[ia] - ta;
          hfield[ib] = hfield[ib] + tb;
          did = true;
        }
      }
      if (did) {
        reached[ia] = 1;
        reached[ib] = 1;
        ++moved;
        // tiles of the 3x3 cell stencil around both endpoints (within the 3x3 tile block)
        const int ends[4] = {a0, a1, b0, b1};
        for (int q = 0; q < 2; ++q) {
          const int p0 = ends[2 * q], p1 = ends[2 * q + 1];
          for (int o0 = -1; o0 <= 1; ++o0)
            for (int o1 = -1; o1 <= 1; ++o1) {
              const int q0 = p0 + o0, q1 = p1 + o1;
              if (q0 < 0 || q1 < 0 || q0 >= c.n0 || q1 >= c.n1) continue;
              const int rt = q0 / T - tr, ct = q1 / T - tc;  // in [-1, 1]
              trig[(rt + 1) * 3 + ct + 1] = 1;
            }
        }
      }
    }
    moved_total += moved;
    __syncthreads();
    if (threadIdx.x < 9 && trig[threadIdx.x]) {
      const int rt = tr + threadIdx.x / 3 - 1, ct = tc + threadIdx.x % 3 - 1;
      const int nt = rt * c.tiles1 + ct;
      if (atomicExch(&member[nt], 1) == 0) list[atomicAdd(&ctl->list_len, 1)] = nt;
    }
    __syncthreads();  // trig is reset by the next entry
  }
  moved_total = warp_sum(moved_total);
  if (threadIdx.x == 0) moved_count = 0;
  __syncthreads();
  if ((threadIdx.x & 31) == 0 && moved_total) atomicAdd(&moved_count, moved_total);
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    if (moved_count) atomicAdd(&ctl->moved_edges, moved_count);
    __threadfence();
    last = atomicAdd(&ctl->arrive, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last || threadIdx.x != 0) return;
  __threadfence();
  ctl->arrive = 0;
  ctl->sub_len = *(volatile int*)&ctl->list_len;  // appended tiles join the next sub-phase
}

// Final scan of a round over the compacted list: tiles owning a reachable
// pair whose excess is above the tolerance become pending for the next round.
template <bool FX>
__global__ void __launch_bounds__(kThreads)
    frontier_scan_kernel(const RelaxConst c, const typename FvTypes<FX>::H* __restrict__ hfield,
                         const int* __restrict__ reached, const int* __restrict__ list,
                         int* __restrict__ unstable, RelaxControl* ctl) {
  __shared__ int bad;
  if (*(volatile int*)&ctl->done) return;
  const int len = *(volatile int*)&ctl->sub_len;
  const int T = c.ftile;
  for (int e = blockIdx.x; e < len; e += gridDim.x) {
    const int t = list[e];
    if (threadIdx.x == 0) bad = 0;
    __syncthreads();
    const int tr = t / c.tiles1, tc = t % c.tiles1;
    int found = 0;
    for (int k = threadIdx.x; k < T * T && !found; k += kThreads) {
      const int a0 = tr * T + k / T, a1 = tc * T + k % T;
      if (a0 >= c.n0 || a1 >= c.n1) continue;
      for (int d = 0; d < 4 && !found; ++d) {
        int d0, d1;
        dir_of(d, d0, d1);
        const int b0 = a0 + d0, b1 = a1 + d1;
        if (b0 >= c.n0 || b1 < 0 || b1 >= c.n1) continue;
        const size_t ia = (size_t)a0 * c.pitch + a1, ib = (size_t)b0 * c.pitch + b1;
        if (!reached[ia] && !reached[ib]) continue;
        if constexpr (FX) {
          const long long df = (long long)hfield[ia] - (long long)hfield[ib];
          if ((double)(df < 0 ? -df : df) - c.crit_q[d] > c.tol_q) found = 1;
        } else {
          if (fabs(hfield[ia] - hfield[ib]) - c.crit[d] > c.tol) found = 1;
        }
      }
    }
    if (found) bad = 1;
    __syncthreads();
    if (threadIdx.x == 0 && bad) unstable[t] = 1;
    __syncthreads();
  }
}

__global__ void frontier_finish_kernel(const RelaxConst c, int* __restrict__ reached,
                                       const RelaxControl* ctl) {
  if (!ctl->converged) return;
  const long long n = (long long)c.n0 * c.pitch;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    reached[i] = 0;
}

// sum, min and max 8-neighbour slope of a support field (RelaxationStats:
// volume_before/after and max_slope = slope_model.max_neighbor_slope :261-270).
template <bool FX>
__global__ void __launch_bounds__(kThreads)
    field_stats_kernel(int n0, int n1, int pitch, double s0, double s1, double Q, double datum,
                       const typename FvTypes<FX>::H* __restrict__ f, double* __restrict__ partials,
                       long long* __restrict__ ipartials, unsigned int* arrive, double* out) {
  const double diag = hypot(s0, s1);
  double sum = 0.0, mx = 0.0, mn = 1.0e300;
  long long isum = 0;
  const long long n = (long long)n0 * n1;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int a0 = (int)(i / n1), a1 = (int)(i % n1);
    const size_t ia = (size_t)a0 * pitch + a1;
    double va;
    if constexpr (FX) {
      isum += f[ia];
      va = (double)f[ia] * Q + datum;
    } else {
      va = f[ia];
      sum += va;
    }
    mn = fmin(mn, va);
    for (int d = 0; d < 4; ++d) {
      int d0, d1;
      dir_of(d, d0, d1);
      const int b0 = a0 + d0, b1 = a1 + d1;
      if (b0 >= n0 || b1 < 0 || b1 >= n1) continue;
      const size_t ib = (size_t)b0 * pitch + b1;
      const double dist = d == 0 ? s0 : (d == 1 ? s1 : diag);
      double diff;
      if constexpr (FX) diff = (double)((long long)f[ia] - (long long)f[ib]) * Q;
      else diff = f[ia] - f[ib];
      mx = fmax(mx, fabs(diff) / dist);
    }
  }
  sum = warp_sum(sum);
  isum = (long long)warp_sum_u64((unsigned long long)isum);
  mx = warp_max(mx);
  mn = warp_min(mn);
  __shared__ double r[kThreads / 32][3];
  __shared__ long long ri[kThreads / 32];
  __shared__ int last;
  if ((threadIdx.x & 31) == 0) {
    r[threadIdx.x >> 5][0] = sum;
    r[threadIdx.x >> 5][1] = mx;
    r[threadIdx.x >> 5][2] = mn;
    ri[threadIdx.x >> 5] = isum;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0, cmin = 1.0e300;
    long long ia = 0;
    for (int w = 0; w < kThreads / 32; ++w) {
      a += r[w][0];
      b = fmax(b, r[w][1]);
      cmin = fmin(cmin, r[w][2]);
      ia += ri[w];
    }
    partials[blockIdx.x * 3 + 0] = a;
    partials[blockIdx.x * 3 + 1] = b;
    partials[blockIdx.x * 3 + 2] = cmin;
    ipartials[blockIdx.x] = ia;
    __threadfence();
    last = atomicAdd(arrive, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last || threadIdx.x != 0) return;
  __threadfence();
  double a = 0.0, b = 0.0, cmin = 1.0e300;
  long long ia = 0;
  for (unsigned k = 0; k < gridDim.x; ++k) {
    a += __ldcg(partials + k * 3);
    b = fmax(b, __ldcg(partials + k * 3 + 1));
    cmin = fmin(cmin, __ldcg(partials + k * 3 + 2));
    ia += __ldcg(ipartials + k);
  }
  *arrive = 0;
  out[0] = FX ? (double)ia * Q + datum * (double)n : a;
  out[1] = b;
  out[2] = cmin;
  out[3] = (double)ia;
}

// The ping-pong relaxation may end in the alternate buffer: copy it back
// (every block reads the same flag), then clear the flag in a second launch.
template <bool FX>
__global__ void relax_copyback_kernel(const typename FvTypes<FX>::B* __restrict__ src,
                                      typename FvTypes<FX>::B* __restrict__ dst, long long count,
                                      const RelaxControl* ctl) {
  if (!ctl->parity) return;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
       i += (long long)gridDim.x * blockDim.x)
    dst[i] = src[i];
}

// reached mask back into the caller-visible field after a reached-gated solve
__global__ void reached_copyback_kernel(const int* __restrict__ src, int* __restrict__ dst,
                                        long long count, const RelaxControl* ctl) {
  if (!ctl->parity) return;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
       i += (long long)gridDim.x * blockDim.x)
    dst[i] = src[i];
}

__global__ void relax_parity_clear_kernel(RelaxControl* ctl) {
  if (threadIdx.x == 0 && blockIdx.x == 0) ctl->parity = 0;
}

}  // namespace sb
