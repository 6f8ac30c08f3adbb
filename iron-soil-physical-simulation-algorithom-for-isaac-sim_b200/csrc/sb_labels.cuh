// Large-avalanche (FailureZone) labelling: cohesive yield + connected components.
//
// Semantics of the reference device bridge (runtime/gpu_large_avalanche.py):
//   initialize            (:58-162)  -> label_init_local_kernel (fused)
//   union_pass + compress (:164-198, host loop :576-599)
//                                    -> block-local union-find in shared memory,
//                                       label_merge_kernel across tile borders,
//                                       label_compress_kernel
//   aggregate/reduce/select_winner/winner_diagnostics (:200-275)
//                                    -> per-root integer accumulators filled in
//                                       the compress pass, label_reduce_kernel
//   update_previous_and_tiles (:277-306) -> label_update_previous_kernel
//
// Final labels are canonical: every unstable cell holds the minimum flat index
// of its component (roots only ever hook under smaller roots), so the result
// does not depend on scheduling.  The reference needs up to max(ny, nx)
// host-synchronised union passes; here one local pass, one border merge and
// one compression suffice because the lock-free union retries until both
// roots are joined.
//
// Component sums are exact integers (area in units of dx*dy/6, mobilizable
// volume in height quanta * area units, slope excesses in 2^-32 rad), so the
// statistics are deterministic as well.
//
// Yield arithmetic: FP64 in the parity path (the reference's); float32 in the
// fixed-point path (integer height differences, IEEE divisions and roots, the
// slope angle by a published polynomial), restated bit for bit on the CPU.
#pragma once

#include "sb_common.cuh"
#include "sb_fv.cuh"

namespace sb {

constexpr int kLabelTile = 32;
// Threads of the yield/labelling tile kernel: 16 warps per 32x32 tile (two
// cells per thread) and 3 tiles per SM; measured with the FP64 yield (now the
// parity path only; the fixed-point path's yield is float32), 12 warps per
// tile (4 tiles per SM) were 1.3 % slower on the whole 701^2 step, 8 warps
// 0.1 % slower still.
constexpr int kLabelInitThreads = 512;
// Fixed-point units of the per-root sums.  2^32 keeps the int64 sums free of
// overflow up to 2^24 cells with slopes < pi/2 rad and failure depths < 8 m
// (1.7e7 * 8 * 6 * 2^32 < 2^63), at a resolution of 2.3e-10.
constexpr double kExcessScale = 4294967296.0;     // 2^32 per radian
constexpr double kVolumeScaleFp64 = 4294967296.0;  // 2^32 per (m * w6)

struct LabelConst {
  int ny, nx, pitch, tiles_x, connectivity;
  double dx, dy, tan_start, tan_stop, density, gravity, cohesion, mob_depth, dry;
  double activity_speed, start_rad, stop_rad;
  double Q, datum;
  int release_latches;
  int tile_size, frontier_tiles_x;  // frontier tile geometry for seeding
};

// Per-root accumulators (flat index = root).
struct LabelRoots {
  int* count;
  long long* area6;
  long long* volume;      // FX: quanta*w6; FP64: round(transfer*w6 * 2^32)
  long long* exc_start;   // 2^-32 rad
  long long* exc_stop;
  long long* max_exc_start;
  long long* max_exc_stop;
  int* prev_overlap;
};

struct LabelOut {
  int regions;
  int largest;
  int winner;
  int total_unstable;
  int status;
  int root_count;
  unsigned long long best_key;
  long long area6, volume, exc_start, exc_stop, max_exc_start, max_exc_stop;
  int prev_overlap;
  int pad;
};

template <bool FX>
__device__ __forceinline__ double free_surface_diff(const typename FvTypes<FX>::B* b,
                                                    const typename FvTypes<FX>::H* h, size_t ir,
                                                    size_t il, double Q) {
  if constexpr (FX) {
    const long long d = ((long long)b[ir] + h[ir]) - ((long long)b[il] + h[il]);
    return (double)d * Q;
  } else {
    // reference device order: ((r[R] + m[R]) - r[L]) - m[L]
    return ((b[ir] + h[ir]) - b[il]) - h[il];
  }
}

// Fixed-point yield constants in float32, each one rounding of its double
// expression: gradient scales {Q / (2 dx), Q / dx} and {Q / (2 dy), Q / dy},
// the quantum, the mobilization depth, density * gravity, cohesion, the start
// and stop tangents, their difference and the dry tolerance.
struct YieldF {
  float sx[2], sy[2];
  float Q, depth, rg, coh, ts, tp, dts, dry;
};

__device__ __forceinline__ YieldF yield_constants(const LabelConst& c) {
  YieldF y;
  y.sx[0] = (float)(c.Q / (2.0 * c.dx));
  y.sx[1] = (float)(c.Q / c.dx);
  y.sy[0] = (float)(c.Q / (2.0 * c.dy));
  y.sy[1] = (float)(c.Q / c.dy);
  y.Q = (float)c.Q;
  y.depth = (float)c.mob_depth;
  y.rg = (float)(c.density * c.gravity);
  y.coh = (float)c.cohesion;
  y.ts = (float)c.tan_start;
  y.tp = (float)c.tan_stop;
  y.dts = (float)(c.tan_start - c.tan_stop);
  y.dry = (float)c.dry;
  return y;
}

// Arc tangent of x >= 0 in float32 by the polynomial of Abramowitz & Stegun,
// Handbook of Mathematical Functions, 4.4.49 (Hastings): on [0, 1]
// atan(x) = x (1 + a2 x^2 + ... + a16 x^16) with |error| <= 2e-8; for x > 1,
// pi/2 - atan(1/x).  Evaluated in float32 with separate multiplies and adds
// (Horner), so a NumPy float32 restatement gives the same bits; error against
// the exact value <= 2e-7 rad.
__device__ __forceinline__ float atan_as4449(float x) {
  const bool inv = x > 1.0f;
  const float t = inv ? 1.0f / x : x;
  const float t2 = t * t;
  float p = 0.0028662257f;
  p = -0.0161657367f + t2 * p;
  p = 0.0429096138f + t2 * p;
  p = -0.0752896400f + t2 * p;
  p = 0.1065626393f + t2 * p;
  p = -0.1420889944f + t2 * p;
  p = 0.1999355085f + t2 * p;
  p = -0.3333314528f + t2 * p;
  p = 1.0f + t2 * p;
  const float r = t * p;
  return inv ? 1.5707963267948966f - r : r;
}

__device__ __forceinline__ int lfind(const int* lab, int x) {
  for (int i = 0; i < kLabelTile * kLabelTile && lab[x] != x; ++i) x = lab[x];
  return x;
}

__device__ __forceinline__ void lunion(int* lab, int a, int b) {
  for (int it = 0; it < 4 * kLabelTile * kLabelTile; ++it) {
    a = lfind(lab, a);
    b = lfind(lab, b);
    if (a == b) return;
    if (a > b) {
      const int t = a;
      a = b;
      b = t;
    }
    const int old = atomicMin(&lab[b], a);
    if (old == b) return;
    b = old;
  }
}

// Block-local union-find over one kLabelTile^2 tile held in shared memory,
// then global root ids (the tile's min member in row-major order is also its
// min flat index) written to ``parent``.
__device__ __forceinline__ void local_ccl(int* lab, int connectivity, int gy0, int gx0, int nx,
                                          int* __restrict__ parent) {
  __syncthreads();
  // block-local union over the backward neighbours W, N (and NW, NE for 8-conn)
  for (int li = threadIdx.x; li < kLabelTile * kLabelTile; li += blockDim.x) {
    if (lab[li] < 0) continue;
    const int ly = li / kLabelTile, lx = li % kLabelTile;
    if (lx > 0 && lab[li - 1] >= 0) lunion(lab, li, li - 1);
    if (ly > 0) {
      if (lab[li - kLabelTile] >= 0) lunion(lab, li, li - kLabelTile);
      if (connectivity == 8) {
        if (lx > 0 && lab[li - kLabelTile - 1] >= 0) lunion(lab, li, li - kLabelTile - 1);
        if (lx + 1 < kLabelTile && lab[li - kLabelTile + 1] >= 0)
          lunion(lab, li, li - kLabelTile + 1);
      }
    }
  }
  __syncthreads();
  for (int li = threadIdx.x; li < kLabelTile * kLabelTile; li += blockDim.x) {
    if (lab[li] < 0) continue;
    const int root = lfind(lab, li);
    const int ly = li / kLabelTile, lx = li % kLabelTile;
    const int rr = root / kLabelTile, rc = root % kLabelTile;
    parent[(long long)(gy0 + ly) * nx + gx0 + lx] = (gy0 + rr) * nx + gx0 + rc;
  }
}


template <bool FX>
__global__ void __launch_bounds__(kLabelInitThreads, 3)
    label_init_local_kernel(const LabelConst c, const typename FvTypes<FX>::B* __restrict__ b,
                            const typename FvTypes<FX>::B* __restrict__ z,
                            const typename FvTypes<FX>::H* __restrict__ h0,
                            const typename FvTypes<FX>::H* __restrict__ h1,
                            const typename FvTypes<FX>::R* __restrict__ qx0,
                            const typename FvTypes<FX>::R* __restrict__ qx1,
                            const typename FvTypes<FX>::R* __restrict__ qy0,
                            const typename FvTypes<FX>::R* __restrict__ qy1, const FvControl* ctl,
                            int* __restrict__ parent, typename FvTypes<FX>::R* __restrict__ slope_out,
                            typename FvTypes<FX>::R* __restrict__ severity_out,
                            int* __restrict__ latch, const double* __restrict__ export_cum,
                            const double* __restrict__ export_base, LabelRoots roots) {
  __shared__ int lab[kLabelTile * kLabelTile];
  const int tx = blockIdx.x % c.tiles_x, ty = blockIdx.x / c.tiles_x;
  const int gx0 = tx * kLabelTile, gy0 = ty * kLabelTile;
  const int P = ctl->parity;  // buffer holding the current mobile state
  const typename FvTypes<FX>::H* h = P ? h1 : h0;
  const typename FvTypes<FX>::R* qx = P ? qx1 : qx0;
  const typename FvTypes<FX>::R* qy = P ? qy1 : qy0;
  const YieldF yf = yield_constants(c);
  for (int li = threadIdx.x; li < kLabelTile * kLabelTile; li += kLabelInitThreads) {
    const int ly = li / kLabelTile, lx = li % kLabelTile;
    const int r = gy0 + ly, col = gx0 + lx;
    int u = 0;
    if (r < c.ny && col < c.nx) {
      const size_t gi = (size_t)r * c.pitch + col;
      const long long flat = (long long)r * c.nx + col;
      const int cl = col > 0 ? col - 1 : col, cr = col + 1 < c.nx ? col + 1 : col;
      const int rd = r > 0 ? r - 1 : r, ru = r + 1 < c.ny ? r + 1 : r;
      const bool inx = col > 0 && col + 1 < c.nx, iny = r > 0 && r + 1 < c.ny;
      double mob;
      bool settled;  // stop margin <= 0
      if constexpr (FX) {
        // float32 throughout (the ledger and the exchange sums are the only
        // FP64 work of the fixed-point path)
        const long long dxq = ((long long)b[(size_t)r * c.pitch + cr] + h[(size_t)r * c.pitch + cr]) -
                              ((long long)b[(size_t)r * c.pitch + cl] + h[(size_t)r * c.pitch + cl]);
        const long long dyq = ((long long)b[(size_t)ru * c.pitch + col] + h[(size_t)ru * c.pitch + col]) -
                              ((long long)b[(size_t)rd * c.pitch + col] + h[(size_t)rd * c.pitch + col]);
        const float gx = (float)dxq * (inx ? yf.sx[0] : yf.sx[1]);
        const float gy = (float)dyq * (iny ? yf.sy[0] : yf.sy[1]);
        const float mag = sqrtf(gx * gx + gy * gy);
        const long long dq = (long long)b[gi] - (long long)z[gi];
        const float layer = fminf((float)(dq > 0 ? dq : 0) * yf.Q, yf.depth);
        mob = (double)h[gi] * c.Q;
        const float norm = sqrtf(1.0f + mag * mag);
        const float drive = yf.rg * layer * mag / norm;
        const float normal = yf.rg * layer / norm;
        const float start_margin = drive - (yf.coh + normal * yf.ts);
        const float stop_margin = drive - (yf.coh + normal * yf.tp);
        const float sev = fminf(fmaxf(stop_margin / fmaxf(normal * yf.dts, 1.0e-12f), 0.f), 1.f);
        slope_out[flat] = atan_as4449(mag);
        severity_out[flat] = sev;
        u = (layer > yf.dry && start_margin > 0.f) ? 1 : 0;
        settled = stop_margin <= 0.f;
      } else {
        const double denx = inx ? 2.0 * c.dx : c.dx;
        const double deny = iny ? 2.0 * c.dy : c.dy;
        const double gx = free_surface_diff<FX>(b, h, (size_t)r * c.pitch + cr,
                                                (size_t)r * c.pitch + cl, c.Q) / denx;
        const double gy = free_surface_diff<FX>(b, h, (size_t)ru * c.pitch + col,
                                                (size_t)rd * c.pitch + col, c.Q) / deny;
        const double mag = sqrt(gx * gx + gy * gy);
        const double layer = fmin(fmax(b[gi] - z[gi], 0.0), c.mob_depth);
        mob = h[gi];
        const double norm = sqrt(1.0 + mag * mag);
        const double drive = c.density * c.gravity * layer * mag / norm;
        const double normal = c.density * c.gravity * layer / norm;
        const double start_margin = drive - (c.cohesion + normal * c.tan_start);
        const double stop_margin = drive - (c.cohesion + normal * c.tan_stop);
        const double sev = fmin(fmax(stop_margin / fmax(normal * (c.tan_start - c.tan_stop), 1.0e-12), 0.0), 1.0);
        slope_out[flat] = atan(mag);
        severity_out[flat] = sev;
        u = (layer > c.dry && start_margin > 0.0) ? 1 : 0;
        settled = stop_margin <= 0.0;
      }
      parent[flat] = u ? (int)flat : -1;
      if (u) {
        roots.count[flat] = 0;
        roots.area6[flat] = 0;
        roots.volume[flat] = 0;
        roots.exc_start[flat] = 0;
        roots.exc_stop[flat] = 0;
        roots.max_exc_start[flat] = 0;
        roots.max_exc_stop[flat] = 0;
        roots.prev_overlap[flat] = 0;
      }
      // a latch that is already released stays released: only set latches
      // need the speed and export test
      if (c.release_latches && latch[flat] != 0) {
        double speed = 0.0;
        if (mob > c.dry) {
          const double vx = (double)qx[gi] / mob, vy = (double)qy[gi] / mob;
          speed = sqrt(vx * vx + vy * vy);
        }
        const double w = (double)vertex_weight6(r, col, c.ny, c.nx) * (c.dx * c.dy / 6.0);
        const bool resolved = (export_cum[flat] - export_base[flat]) > c.dry * w;
        if (speed <= c.activity_speed && (resolved || settled)) latch[flat] = 0;
      }
    }
    lab[li] = u ? li : -1;
  }
  local_ccl(lab, c.connectivity, gy0, gx0, c.nx, parent);
}

// Labels a caller-provided mask (reference ``_largest_connected_region``).
__global__ void __launch_bounds__(kThreads)
    label_mask_local_kernel(const LabelConst c, const int* __restrict__ mask,
                            int* __restrict__ parent, LabelRoots roots) {
  __shared__ int lab[kLabelTile * kLabelTile];
  const int tx = blockIdx.x % c.tiles_x, ty = blockIdx.x / c.tiles_x;
  const int gx0 = tx * kLabelTile, gy0 = ty * kLabelTile;
  for (int li = threadIdx.x; li < kLabelTile * kLabelTile; li += kThreads) {
    const int ly = li / kLabelTile, lx = li % kLabelTile;
    const int r = gy0 + ly, col = gx0 + lx;
    int u = 0;
    if (r < c.ny && col < c.nx) {
      const long long flat = (long long)r * c.nx + col;
      u = mask[flat] != 0;
      parent[flat] = u ? (int)flat : -1;
      if (u) {
        roots.count[flat] = 0;
        roots.area6[flat] = 0;
        roots.volume[flat] = 0;
        roots.exc_start[flat] = 0;
        roots.exc_stop[flat] = 0;
        roots.max_exc_start[flat] = 0;
        roots.max_exc_stop[flat] = 0;
        roots.prev_overlap[flat] = 0;
      }
    }
    lab[li] = u ? li : -1;
  }
  local_ccl(lab, c.connectivity, gy0, gx0, c.nx, parent);
}

__device__ __forceinline__ int gfind(const int* parent, int x, int n) {
  for (int i = 0; i < n; ++i) {
    const int p = __ldcg(parent + x);
    if (p == x) return x;
    x = p;
  }
  return x;
}

__device__ __forceinline__ bool gunion(int* parent, int a, int b, int n) {
  for (int it = 0; it < n; ++it) {
    a = gfind(parent, a, n);
    b = gfind(parent, b, n);
    if (a == b) return true;
    if (a > b) {
      const int t = a;
      a = b;
      b = t;
    }
    const int old = atomicMin(&parent[b], a);
    if (old == b) return true;
    b = old;
  }
  return false;
}

// Joins components across tile borders (backward neighbours in other tiles).
__global__ void __launch_bounds__(kThreads)
    label_merge_kernel(const LabelConst c, int* __restrict__ parent, LabelOut* out) {
  const int tx = blockIdx.x % c.tiles_x, ty = blockIdx.x / c.tiles_x;
  const int gx0 = tx * kLabelTile, gy0 = ty * kLabelTile;
  const int n = c.ny * c.nx;
  // border cells: first row (ly == 0), first column (lx == 0), last column (lx == T-1)
  for (int k = threadIdx.x; k < 3 * kLabelTile; k += kThreads) {
    int ly, lx;
    if (k < kLabelTile) {
      ly = 0;
      lx = k;
    } else if (k < 2 * kLabelTile) {
      ly = k - kLabelTile;
      lx = 0;
    } else {
      ly = k - 2 * kLabelTile;
      lx = kLabelTile - 1;
    }
    const int r = gy0 + ly, col = gx0 + lx;
    if (r >= c.ny || col >= c.nx) continue;
    const int i = r * c.nx + col;
    if (__ldcg(parent + i) < 0) continue;
    bool ok = true;
    // W (other tile iff lx == 0)
    if (lx == 0 && col > 0 && __ldcg(parent + i - 1) >= 0) ok &= gunion(parent, i, i - 1, n);
    if (r > 0) {
      // N (other tile iff ly == 0)
      if (ly == 0 && __ldcg(parent + i - c.nx) >= 0) ok &= gunion(parent, i, i - c.nx, n);
      if (c.connectivity == 8) {
        // NW: other tile iff ly == 0 or lx == 0
        if ((ly == 0 || lx == 0) && col > 0 && __ldcg(parent + i - c.nx - 1) >= 0)
          ok &= gunion(parent, i, i - c.nx - 1, n);
        // NE: other tile iff ly == 0 or lx == T-1
        if ((ly == 0 || lx == kLabelTile - 1) && col + 1 < c.nx &&
            __ldcg(parent + i - c.nx + 1) >= 0)
          ok &= gunion(parent, i, i - c.nx + 1, n);
      }
    }
    if (!ok) atomicExch(&out->status, 4);
  }
}

// Full path compression + per-root statistics; roots are appended to a list.
template <bool FX>
__global__ void __launch_bounds__(kThreads)
    label_compress_kernel(const LabelConst c, int* __restrict__ parent,
                          const typename FvTypes<FX>::B* __restrict__ b,
                          const typename FvTypes<FX>::B* __restrict__ z,
                          const typename FvTypes<FX>::R* __restrict__ slope,
                          const typename FvTypes<FX>::R* __restrict__ severity,
                          const int* __restrict__ latch, const int* __restrict__ previous,
                          LabelRoots roots, int* __restrict__ root_list, LabelOut* out,
                          int mask_only) {
  const int n = c.ny * c.nx;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int p = __ldcg(parent + i);
    if (p < 0) continue;
    const int root = gfind(parent, i, n);
    if (root != p) parent[i] = root;
    const int r = i / c.nx, col = i % c.nx;
    const size_t gi = (size_t)r * c.pitch + col;
    const int w6 = vertex_weight6(r, col, c.ny, c.nx);
    long long vol = 0;
    if (mask_only) {
      atomicAdd(&roots.count[root], 1);
      atomicAdd((unsigned long long*)&roots.area6[root], (unsigned long long)w6);
      if (root == i) root_list[atomicAdd(&out->root_count, 1)] = i;
      continue;
    }
    if (latch[i] == 0) {
      if constexpr (FX) {
        const long long avail = (long long)b[gi] - (long long)z[gi];
        const long long cap = (long long)floor(c.mob_depth * (double)severity[i] / c.Q);
        vol = (avail > 0 ? (avail < cap ? avail : cap) : 0) * w6;
      } else {
        const double t = fmin(fmax(b[gi] - z[gi], 0.0), c.mob_depth * severity[i]);
        vol = llrint(t * (double)w6 * kVolumeScaleFp64);
      }
    }
    const double s = (double)slope[i];
    const long long es = llrint(fmax(s - c.start_rad, 0.0) * kExcessScale);
    const long long et = llrint(fmax(s - c.stop_rad, 0.0) * kExcessScale);
    atomicAdd(&roots.count[root], 1);
    atomicAdd((unsigned long long*)&roots.area6[root], (unsigned long long)w6);
    if (vol) atomicAdd((unsigned long long*)&roots.volume[root], (unsigned long long)vol);
    if (es) {
      atomicAdd((unsigned long long*)&roots.exc_start[root], (unsigned long long)es);
      atomicMax(&roots.max_exc_start[root], es);
    }
    if (et) {
      atomicAdd((unsigned long long*)&roots.exc_stop[root], (unsigned long long)et);
      atomicMax(&roots.max_exc_stop[root], et);
    }
    if (previous[i]) atomicAdd(&roots.prev_overlap[root], 1);
    if (root == i) {
      const int slot = atomicAdd(&out->root_count, 1);
      root_list[slot] = i;
    }
  }
}

// Region count, total, largest (ties -> smallest root) in one pass over roots;
// the last block copies the winner's accumulators into the output record.
// Returns true in the one thread (thread 0 of the last block) that wrote the
// final record.
__device__ __forceinline__ bool label_reduce_body(const LabelRoots& roots,
                                                  const int* __restrict__ root_list, LabelOut* out,
                                                  unsigned int* arrive) {
  const int nroots = out->root_count;
  unsigned long long best = 0;
  int total = 0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nroots; k += gridDim.x * blockDim.x) {
    const int root = root_list[k];
    const int cnt = roots.count[root];
    total += cnt;
    const unsigned long long key =
        ((unsigned long long)(unsigned)cnt << 32) | (unsigned long long)(0x7fffffffu - (unsigned)root);
    best = key > best ? key : best;
  }
  total = warp_sum(total);
  best = warp_max(best);
  if ((threadIdx.x & 31) == 0) {
    if (total) atomicAdd(&out->total_unstable, total);
    if (best) atomicMax(&out->best_key, best);
  }
  __threadfence();
  __syncthreads();
  __shared__ int last;
  if (threadIdx.x == 0) last = atomicAdd(arrive, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last || threadIdx.x != 0) return false;
  __threadfence();
  *arrive = 0;
  out->regions = nroots;
  const unsigned long long key = *(volatile unsigned long long*)&out->best_key;
  if (key == 0) {
    out->largest = 0;
    out->winner = -1;
    return true;
  }
  const int winner = (int)(0x7fffffffu - (unsigned)(key & 0xffffffffu));
  out->largest = (int)(key >> 32);
  out->winner = winner;
  out->area6 = roots.area6[winner];
  out->volume = roots.volume[winner];
  out->exc_start = roots.exc_start[winner];
  out->exc_stop = roots.exc_stop[winner];
  out->max_exc_start = roots.max_exc_start[winner];
  out->max_exc_stop = roots.max_exc_stop[winner];
  out->prev_overlap = roots.prev_overlap[winner];
  return true;
}

__global__ void __launch_bounds__(kThreads)
    label_reduce_kernel(LabelRoots roots, const int* __restrict__ root_list, LabelOut* out,
                        unsigned int* arrive) {
  label_reduce_body(roots, root_list, out, arrive);
}

// previous-component mask and residual frontier seeding (reference :277-306).
__global__ void __launch_bounds__(kThreads)
    label_update_previous_kernel(const LabelConst c, const int* __restrict__ parent,
                                 int* __restrict__ previous, int* __restrict__ reached,
                                 int* __restrict__ tile_flags, const LabelOut* out,
                                 int keep_candidate, int seed_frontier) {
  const int n = c.ny * c.nx;
  const int winner = out->winner;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const bool belongs = winner >= 0 && parent[i] == winner;
    previous[i] = (belongs && keep_candidate) ? 1 : 0;
    if (belongs && seed_frontier) {
      const int r = i / c.nx, col = i % c.nx;
      reached[(size_t)r * c.pitch + col] = 1;
      tile_flags[(r / c.tile_size) * c.frontier_tiles_x + col / c.tile_size] = 1;
    }
  }
}

}  // namespace sb
