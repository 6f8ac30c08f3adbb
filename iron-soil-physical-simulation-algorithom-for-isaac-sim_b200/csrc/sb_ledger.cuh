// Per-step ledger / prologue reduction and field conversion kernels.
//
// One pass over the state computes, with a deterministic two-level reduction:
//   * the FP64 ledger of MobileV2ReferenceSolver.mass/momentum/energy_terms
//     (experimental/mobile_v2_reference.py:104-127) and of the production
//     ``summarize`` kernel (bulk_interaction/warp_mobile_v2.py:28-54); in the
//     fixed-point path mass and Triangle-A-C volume are exact int64 sums;
//   * the static short-circuit of ``_globally_static_below_start`` (:353-363);
//   * the wave speed that sets the first substep's dt (:239-253).
#pragma once

#include "sb_fv.cuh"

namespace sb {

// FX: squared free-surface gradient of cell (r, col) (np.gradient,
// edge_order 1) from integer b + h differences, scaled by Q / (2 dx) inside
// and Q / dx on the edges (c.gsx / c.gsy, computed on the host).
__device__ __forceinline__ double fx_grad2(const FvConst& c, const int32_t* __restrict__ b,
                                           const int32_t* __restrict__ h, int r, int col) {
  const bool inx = col > 0 && col + 1 < c.nx, iny = r > 0 && r + 1 < c.ny;
  const int cl = col > 0 ? col - 1 : col, cr = col + 1 < c.nx ? col + 1 : col;
  const int rd = r > 0 ? r - 1 : r, ru = r + 1 < c.ny ? r + 1 : r;
  const size_t il = (size_t)r * c.pitch + cl, ir = (size_t)r * c.pitch + cr;
  const size_t idn = (size_t)rd * c.pitch + col, iup = (size_t)ru * c.pitch + col;
  const long long Hl = (long long)b[il] + h[il], Hr = (long long)b[ir] + h[ir];
  const long long Hd = (long long)b[idn] + h[idn], Hu = (long long)b[iup] + h[iup];
  const double gx = (double)(Hr - Hl) * (inx ? c.gsx[0] : c.gsx[1]);
  const double gy = (double)(Hu - Hd) * (iny ? c.gsy[0] : c.gsy[1]);
  return gx * gx + gy * gy;
}

// FX ledger contributions of cell (r, col).  Every load of the cell is
// issued before any branch (one memory round trip per cell).  A cell with no
// mobile material and no momentum (most of a terrain) contributes an exact
// zero to every sum and to every maximum other than the resting volume, the
// gradient, the external forcing and the depth minimum; adding a zero leaves
// a sum that starts at +0 bit for bit unchanged, so only those are evaluated.
__device__ __forceinline__ void ledger_cell_fx(const FvConst& c, const int32_t* __restrict__ b,
                                               const int32_t* __restrict__ z,
                                               const int32_t* __restrict__ h,
                                               const float* __restrict__ qx,
                                               const float* __restrict__ qy,
                                               const float* __restrict__ ext_x,
                                               const float* __restrict__ ext_y, double datum,
                                               int r, int col, double* v, long long& iq0,
                                               long long& iq1, long long& iq2) {
  const size_t gi = (size_t)r * c.pitch + col;
  const int w6 = vertex_weight6(r, col, c.ny, c.nx);
  const int hq = h[gi], bq = b[gi], zq = z[gi];
  const float qxf = qx[gi], qyf = qy[gi];
  const double grad = fx_grad2(c, b, h, r, col);  // squared; sqrt after the max
  const long long rest = (long long)bq - (long long)zq;
  iq2 += (rest > 0 ? rest : 0) * w6;
  v[L_MAXGRAD] = fmax(v[L_MAXGRAD], grad);
  if (c.has_external)
    v[L_MAXEXT] = fmax(v[L_MAXEXT], fmax(fabs((double)ext_x[gi]), fabs((double)ext_y[gi])));
  const double hv = (double)hq * c.Q;
  v[L_NEGMINH] = fmax(v[L_NEGMINH], -hv);
  if (hq == 0 && qxf == 0.f && qyf == 0.f) return;
  const double bv = (double)bq * c.Q + datum;
  const double qxv = (double)qxf, qyv = (double)qyf;
  iq0 += hq;
  iq1 += (long long)hq * w6;
  double s2 = 0.0, e = 0.0, wave = 0.0;  // empty cell: no velocity, no celerity
  if (hq != 0) {
    const float hn = (float)hq * c.Qf;
    float vx = 0.f, vy = 0.f;
    if (hn > c.dryf) {
      const float inv = 1.0f / hn;
      vx = qxf * inv;
      vy = qyf * inv;
    }
    wave = (double)(sqrtf(vx * vx + vy * vy) + sqrtf(c.KGf * hn));
  }
  if (hv > c.dry) {  // one reciprocal: e = |q|^2 / h (= h |u|^2), s2 = e / h
    const double inv = 1.0 / hv;
    e = (qxv * qxv + qyv * qyv) * inv;
    s2 = e * inv;
  }
  v[L_QX] += qxv;
  v[L_QY] += qyv;
  v[L_QX_W] += qxv * w6;
  v[L_QY_W] += qyv * w6;
  v[L_HS2] += e;
  v[L_HS2_W] += e * w6;
  v[L_HB] += hv * bv;
  v[L_HB_W] += hv * bv * w6;
  v[L_HH] += hv * hv;
  v[L_HH_W] += hv * hv * w6;
  v[L_MAXSPEED] = fmax(v[L_MAXSPEED], s2);  // squared speed; sqrt after the max
  v[L_MAXQ] = fmax(v[L_MAXQ], fmax(fabs(qxv), fabs(qyv)));
  v[L_MAXWAVE] = fmax(v[L_MAXWAVE], wave);
}

// Ledger contributions of cell (r, col): sums into v[0 .. L_NSUM), maxima
// into v[L_NSUM .. L_NP), exact quanta sums into iq0..iq2 (FX: ledger_cell_fx).
template <bool FX>
__device__ __forceinline__ void ledger_cell(const FvConst& c,
                                            const typename FvTypes<FX>::B* __restrict__ b,
                                            const typename FvTypes<FX>::B* __restrict__ z,
                                            const typename FvTypes<FX>::H* __restrict__ h,
                                            const typename FvTypes<FX>::R* __restrict__ qx,
                                            const typename FvTypes<FX>::R* __restrict__ qy,
                                            const typename FvTypes<FX>::R* __restrict__ ext_x,
                                            const typename FvTypes<FX>::R* __restrict__ ext_y,
                                            double datum, int r, int col, double* v,
                                            long long& iq0, long long& iq1, long long& iq2) {
  if constexpr (FX) {
    ledger_cell_fx(c, b, z, h, qx, qy, ext_x, ext_y, datum, r, col, v, iq0, iq1, iq2);
  } else {
    const size_t gi = (size_t)r * c.pitch + col;
    const int w6 = vertex_weight6(r, col, c.ny, c.nx);
    const double qxv = (double)qx[gi], qyv = (double)qy[gi];
    // gradient of the free surface b + h (np.gradient, edge_order 1)
    const int cl = col > 0 ? col - 1 : col, cr = col + 1 < c.nx ? col + 1 : col;
    const int rd = r > 0 ? r - 1 : r, ru = r + 1 < c.ny ? r + 1 : r;
    const double denx = (col > 0 && col + 1 < c.nx) ? 2.0 * c.dx : c.dx;
    const double deny = (r > 0 && r + 1 < c.ny) ? 2.0 * c.dy : c.dy;
    const size_t il = (size_t)r * c.pitch + cl, ir = (size_t)r * c.pitch + cr;
    const size_t idn = (size_t)rd * c.pitch + col, iup = (size_t)ru * c.pitch + col;
    const double hv = h[gi];
    const double bv = b[gi];
    v[L_HSUM] += hv;
    v[L_HSUM_W] += hv * w6;
    v[L_REST_W] += fmax(b[gi] - z[gi], 0.0) * w6;
    const double gx = ((b[ir] + h[ir]) - (b[il] + h[il])) / denx;
    const double gy = ((b[iup] + h[iup]) - (b[idn] + h[idn])) / deny;
    const double grad = hypot(gx, gy);
    const bool wet = hv > c.dry;
    double s2 = 0.0, spd = 0.0, e = 0.0;
    double vx = 0.0, vy = 0.0;
    if (wet) {
      vx = qxv / hv;
      vy = qyv / hv;
    }
    const double wave = sqrt(vx * vx + vy * vy) + sqrt(c.kg * fmax(hv, 0.0));
    if (wet) {
      s2 = (qxv * qxv + qyv * qyv) / (hv * hv);
      spd = sqrt(s2);
      e = hv * s2;
    }
    v[L_QX] += qxv;
    v[L_QY] += qyv;
    v[L_QX_W] += qxv * w6;
    v[L_QY_W] += qyv * w6;
    v[L_HS2] += e;
    v[L_HS2_W] += e * w6;
    v[L_HB] += hv * bv;
    v[L_HB_W] += hv * bv * w6;
    v[L_HH] += hv * hv;
    v[L_HH_W] += hv * hv * w6;
    v[L_MAXSPEED] = fmax(v[L_MAXSPEED], spd);
    v[L_NEGMINH] = fmax(v[L_NEGMINH], -hv);
    v[L_MAXQ] = fmax(v[L_MAXQ], fmax(fabs(qxv), fabs(qyv)));
    v[L_MAXGRAD] = fmax(v[L_MAXGRAD], grad);
    v[L_MAXWAVE] = fmax(v[L_MAXWAVE], wave);
    if (c.has_external)
      v[L_MAXEXT] = fmax(v[L_MAXEXT], fmax(fabs((double)ext_x[gi]), fabs((double)ext_y[gi])));
  }
}

// Block reduction of per-thread ledger values into one block's partials, in a
// fixed order: slot k to part[k * stride], integer slot k to ipart[k * stride].
// fold: fold_words(L_NP) doubles of shared memory.
__device__ __forceinline__ void ledger_block_store(const double* v, long long iq0, long long iq1,
                                                   long long iq2, double* fold, double* part,
                                                   long long* ipart, int stride) {
  const double* bt = block_fold<double, L_NP, L_NSUM>(v, fold);
  const double mine = threadIdx.x < L_NP ? bt[threadIdx.x] : 0.0;
  __syncthreads();  // the integer fold reuses the scratch
  const long long iv[kLedgerI64] = {iq0, iq1, iq2};
  const long long* it =
      block_fold<long long, kLedgerI64, kLedgerI64>(iv, reinterpret_cast<long long*>(fold));
  if (threadIdx.x < L_NP) part[(size_t)threadIdx.x * stride] = mine;
  if (threadIdx.x < kLedgerI64) ipart[(size_t)threadIdx.x * stride] = it[threadIdx.x];
}

// Final value of ledger slot k: the FX path accumulates squared gradient and
// squared speed maxima and takes the (monotone) square root after the max.
template <bool FX>
__device__ __forceinline__ double ledger_final_value(int k, double val) {
  if (FX && (k == L_MAXGRAD || k == L_MAXSPEED)) return sqrt(val);
  return val;
}

// Fixed-order fold of a ledger's slot-major block partials (nb blocks) into
// out.  Every thread of the block calls it; scratch: fold_words(L_NP) doubles.
template <bool FX>
__device__ void ledger_final_fold(const double* partials, const long long* ipartials, int nb,
                                  double* fold, LedgerOut* out) {
  const double* tot = reduce_partials<L_NP, L_NSUM>(partials, nb, fold);
  const double mine = threadIdx.x < L_NP ? tot[threadIdx.x] : 0.0;
  __syncthreads();  // the integer fold reuses the scratch
  long long a[kLedgerI64] = {0, 0, 0};
  for (int bk = threadIdx.x; bk < nb; bk += kThreads)
#pragma unroll
    for (int k = 0; k < kLedgerI64; ++k) a[k] += __ldcg(ipartials + (size_t)k * nb + bk);
  const long long* itot =
      block_fold<long long, kLedgerI64, kLedgerI64>(a, reinterpret_cast<long long*>(fold));
  if (threadIdx.x < L_NP) out->v[threadIdx.x] = ledger_final_value<FX>(threadIdx.x, mine);
  if (threadIdx.x < kLedgerI64) out->iq[threadIdx.x] = itot[threadIdx.x];
  __syncthreads();
}

// Static short-circuit and the first substep's dt from a "before" ledger
// (reference step :199-205, :239-253).  One thread.
__device__ __forceinline__ void ledger_prologue(const FvConst& c, const LedgerOut* out,
                                                double static_limit, FvControl* ctl) {
  const bool no_ext = !c.has_external || out->v[L_MAXEXT] <= 1.0e-14;
  const bool is_static = no_ext && out->v[L_MAXQ] <= 1.0e-14 && out->v[L_MAXGRAD] <= static_limit;
  ctl->wave = out->v[L_MAXWAVE];
  if (is_static) {
    ctl->static_skip = 1;
    ctl->done = 1;
  } else if (!(ctl->remaining > 1.0e-14)) {
    ctl->done = 1;
  } else if (c.max_substeps <= 0) {
    ctl->status = 2;
    ctl->done = 1;
  } else {
    plan_substep(c, ctl);
  }
}

// mode 0: "before" ledger of a step + prologue (static short-circuit, first
// dt, loop condition).  The prologue only needs four maxima, which the blocks
// send by atomicMax (order-free), so the last block plans the first substep
// at once; the before ledger's sums stay as block partials (part_before).
// mode 1: "after" ledger.  mode 2: "after" ledger, then the folds that the
// step deferred: the before ledger's partials into io->before and the step's
// substep impulse/energy sums (diag_acc, c.nblocks FV blocks) into ctl->diag.
template <bool FX>
__global__ void __launch_bounds__(kThreads, 3)
    ledger_kernel(const FvConst c, const typename FvTypes<FX>::B* __restrict__ b,
                  const typename FvTypes<FX>::B* __restrict__ z,
                  const typename FvTypes<FX>::H* __restrict__ h0,
                  const typename FvTypes<FX>::H* __restrict__ h1,
                  const typename FvTypes<FX>::R* __restrict__ qx0,
                  const typename FvTypes<FX>::R* __restrict__ qx1,
                  const typename FvTypes<FX>::R* __restrict__ qy0,
                  const typename FvTypes<FX>::R* __restrict__ qy1,
                  const typename FvTypes<FX>::R* __restrict__ ext_x,
                  const typename FvTypes<FX>::R* __restrict__ ext_y, double datum,
                  double static_limit, int mode, FvControl* ctl, StepIO* io,
                  double* __restrict__ partials, long long* __restrict__ ipartials,
                  unsigned int* arrive, double* __restrict__ diag_acc,
                  double* __restrict__ part_before, long long* __restrict__ ipart_before,
                  cudaGraphConditionalHandle loop_handle, int use_handle) {
  using T = FvTypes<FX>;
  const int parity = ctl->parity;
  const typename T::H* h = parity ? h1 : h0;
  const typename T::R* qx = parity ? qx1 : qx0;
  const typename T::R* qy = parity ? qy1 : qy0;
  double v[L_NP];
#pragma unroll
  for (int k = 0; k < L_NP; ++k) v[k] = 0.0;
  v[L_NEGMINH] = -1.0e300;
  long long iq0 = 0, iq1 = 0, iq2 = 0;
  {
    // warp items = 32-column segments of one row; a lane owns one column
    const int strips = (c.nx + 31) >> 5;
    const int items = strips * c.ny;
    const int nwarps = gridDim.x * (kThreads / 32);
    const int lane = threadIdx.x & 31;
    int it = blockIdx.x * (kThreads / 32) + (threadIdx.x >> 5);
    int r = it / strips, s = it - r * strips;
    const int dr = nwarps / strips, ds = nwarps - dr * strips;
#pragma unroll 2
    for (; it < items; it += nwarps) {
      const int col = (s << 5) + lane;
      if (col < c.nx)
        ledger_cell<FX>(c, b, z, h, qx, qy, ext_x, ext_y, datum, r, col, v, iq0, iq1, iq2);
      r += dr;
      s += ds;
      if (s >= strips) {
        s -= strips;
        ++r;
      }
    }
  }
  __shared__ double fold[fold_words(L_NP)];
  __shared__ int last;
  // block partials slot-major: partials[k * gridDim.x + block]
  double* part = mode == 0 ? part_before : partials;
  long long* ipart = mode == 0 ? ipart_before : ipartials;
  ledger_block_store(v, iq0, iq1, iq2, fold, part + blockIdx.x, ipart + blockIdx.x, gridDim.x);
  __syncthreads();
  if (mode == 0 && threadIdx.x < 4) {  // the prologue's maxima (all >= 0: bits order like values)
    const int slot = threadIdx.x == 0 ? L_MAXEXT
                     : threadIdx.x == 1 ? L_MAXQ
                     : threadIdx.x == 2 ? L_MAXGRAD
                                        : L_MAXWAVE;
    const double m = part[(size_t)slot * gridDim.x + blockIdx.x];
    atomicMax(&ctl->pmax[threadIdx.x], (unsigned long long)__double_as_longlong(m));
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = (atomicAdd(arrive, 1u) == gridDim.x - 1) ? 1 : 0;
  __syncthreads();
  if (!last) return;
  __threadfence();
  if (mode == 0) {
    if (threadIdx.x == 0) {
      // prologue: static short-circuit and the first substep's dt
      LedgerOut pro;
      pro.v[L_MAXEXT] = __longlong_as_double((long long)atomicExch(&ctl->pmax[0], 0ull));
      pro.v[L_MAXQ] = __longlong_as_double((long long)atomicExch(&ctl->pmax[1], 0ull));
      pro.v[L_MAXGRAD] = ledger_final_value<FX>(
          L_MAXGRAD, __longlong_as_double((long long)atomicExch(&ctl->pmax[2], 0ull)));
      pro.v[L_MAXWAVE] = __longlong_as_double((long long)atomicExch(&ctl->pmax[3], 0ull));
      *arrive = 0;
      ledger_prologue(c, &pro, static_limit, ctl);
      __threadfence();
      if (use_handle) cudaGraphSetConditional(loop_handle, ctl->done ? 0u : 1u);
    }
    return;
  }
  ledger_final_fold<FX>(partials, ipartials, gridDim.x, fold, &io->after);
  if (mode == 2) {
    ledger_final_fold<FX>(part_before, ipart_before, gridDim.x, fold, &io->before);
    // the step's impulse/energy sums: fold the FV blocks' accumulators in a
    // fixed order and clear them for the next step
    const int nb = c.nblocks;
    double d[kFvDiag];
#pragma unroll
    for (int k = 0; k < kFvDiag; ++k) d[k] = 0.0;
    for (int bk = threadIdx.x; bk < nb; bk += kThreads) {
#pragma unroll
      for (int k = 0; k < kFvDiag; ++k) {
        double* a = diag_acc + (size_t)k * nb + bk;
        d[k] += __ldcg(a);
        *a = 0.0;
      }
    }
    const double* dt = block_fold<double, kFvDiag, kFvDiag>(d, fold);
    if (threadIdx.x < kFvDiag) ctl->diag[threadIdx.x] = dt[threadIdx.x];
    __syncthreads();
  }
  if (threadIdx.x == 0) *arrive = 0;
}

// Resets the loop control block for a new physics step of dt seconds (one thread).
__device__ __forceinline__ void fv_begin_body(FvControl* ctl, const double* dt) {
  {
    ctl->remaining = *dt;
    ctl->sub_dt = 0.0;
    ctl->max_cfl = 0.0;
    ctl->wave = 0.0;
    for (int k = 0; k < kFvDiag; ++k) ctl->diag[k] = 0.0;
    ctl->substeps = 0;
    ctl->done = 0;
    ctl->status = 0;
    ctl->cfl_limited = 0;
    ctl->static_skip = 0;
    ctl->arrive = 0;
    ctl->wait_fail = 0;
    for (int k = 0; k < 3; ++k) ctl->wave3[k] = 0ull;
  }
}

__global__ void fv_begin_kernel(FvControl* ctl, const double* dt) {
  if (threadIdx.x == 0 && blockIdx.x == 0) fv_begin_body(ctl, dt);
}

// ---------------------------------------------------------------------------
// Field conversion (host float64 layout <-> device storage).
// ---------------------------------------------------------------------------
__global__ void to_fixed_kernel(const double* __restrict__ src, int32_t* __restrict__ dst, int ny,
                                int nx, int pitch, double datum, double scale, int* range_error) {
  const long long n = (long long)ny * nx;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(i / nx), c = (int)(i % nx);
    const double x = rint((src[i] - datum) * scale);
    if (!(fabs(x) < 2147483647.0)) {
      atomicExch(range_error, 1);
      dst[(size_t)r * pitch + c] = 0;
    } else {
      dst[(size_t)r * pitch + c] = (int32_t)x;
    }
  }
}

__global__ void from_fixed_kernel(const int32_t* __restrict__ src, double* __restrict__ dst,
                                  int ny, int nx, int pitch, double datum, double quantum) {
  const long long n = (long long)ny * nx;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(i / nx), c = (int)(i % nx);
    dst[i] = (double)src[(size_t)r * pitch + c] * quantum + datum;
  }
}

__global__ void to_float_kernel(const double* __restrict__ src, float* __restrict__ dst, int ny,
                                int nx, int pitch) {
  const long long n = (long long)ny * nx;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(i / nx), c = (int)(i % nx);
    dst[(size_t)r * pitch + c] = (float)src[i];
  }
}

__global__ void from_float_kernel(const float* __restrict__ src, double* __restrict__ dst, int ny,
                                  int nx, int pitch) {
  const long long n = (long long)ny * nx;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(i / nx), c = (int)(i % nx);
    dst[i] = (double)src[(size_t)r * pitch + c];
  }
}

}  // namespace sb
