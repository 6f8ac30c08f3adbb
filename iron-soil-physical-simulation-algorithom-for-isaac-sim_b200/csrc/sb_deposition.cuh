// Incremental Mobile -> Resting deposition (reference
// bulk_interaction/warp_deposition.py:23-130 kernel ``deposit`` and
// ``weighted_sum``, driven by WarpDepositionOperator.step_resident :183-238).
//
// Per cell with mobile material h > 0 and no tool forcing:
//   * sub-cell tail (the whole mobile volume is below one dx*dy*min(dx,dy)
//     voxel): everything settles, momentum removed;
//   * otherwise, if |q/h| <= speed threshold and the free-surface slope is
//     below the cohesive stop yield (drive = rho g h tan/sqrt(1+tan^2) not
//     above cohesion + rho g h tan(stop)/sqrt(1+tan^2)), min(h, rate*dt)
//     settles and the momentum shrinks in proportion.
// The free surface b + h does not change when material settles, but a cell
// must read its neighbours' pre-step surface: the reference reads them while
// other threads write (a race it tolerates); here a first pass decides every
// cell's amount from the unmodified state and a second pass applies it.
#pragma once

#include "sb_common.cuh"
#include "sb_fv.cuh"

namespace sb {

struct DepositionConst {
  int ny, nx, pitch;
  double dx, dy, dt, rate, speed_threshold, density, gravity, cohesion, stop_tan;
  int settle_tail;
  double Q;            // FX quantum
  long long rate_q;    // FX: rate * dt in whole quanta
  float Qf;
};

struct DepositionOut {
  long long volume_w6_quanta;  // FX: sum settled quanta * w6
  double volume_w;             // sum settled * w (m^3)
  double momentum_w[2];        // density * sum removed q * w
  int cells;
  int pad;
};

// Pass 1: settled amount per cell (FX: quanta, FP64: metres) into amount[flat].
template <bool FX>
__global__ void __launch_bounds__(kThreads)
    deposition_decide_kernel(const DepositionConst c, const typename FvTypes<FX>::B* __restrict__ b,
                             const typename FvTypes<FX>::H* __restrict__ h,
                             const typename FvTypes<FX>::R* __restrict__ qx,
                             const typename FvTypes<FX>::R* __restrict__ qy,
                             const int32_t* __restrict__ forcing, double* __restrict__ amount) {
  const long long n = (long long)c.ny * c.nx;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(i / c.nx), col = (int)(i % c.nx);
    const size_t gi = (size_t)r * c.pitch + col;
    double a = 0.0;
    const bool forced = forcing && forcing[i] != 0;
    if constexpr (FX) {
      const int hq = h[gi];
      if (hq > 0 && !forced) {
        if (c.settle_tail) {
          a = (double)hq;
        } else {
          const float hf = (float)hq * c.Qf;
          const float inv = 1.0f / hf;
          const float vx = qx[gi] * inv, vy = qy[gi] * inv;
          if (!(sqrtf(vx * vx + vy * vy) > (float)c.speed_threshold)) {
            const int cl = col > 0 ? col - 1 : col, cr = col + 1 < c.nx ? col + 1 : col;
            const int rd = r > 0 ? r - 1 : r, ru = r + 1 < c.ny ? r + 1 : r;
            const double hx = (col == 0 || col + 1 == c.nx) ? c.dx : 2.0 * c.dx;
            const double hy = (r == 0 || r + 1 == c.ny) ? c.dy : 2.0 * c.dy;
            const size_t il = (size_t)r * c.pitch + cl, ir = (size_t)r * c.pitch + cr;
            const size_t id = (size_t)rd * c.pitch + col, iu = (size_t)ru * c.pitch + col;
            const long long dxq = ((long long)b[ir] + h[ir]) - ((long long)b[il] + h[il]);
            const long long dyq = ((long long)b[iu] + h[iu]) - ((long long)b[id] + h[id]);
            const double sx = (double)dxq * c.Q / hx, sy = (double)dyq * c.Q / hy;
            const double t = sqrt(sx * sx + sy * sy);
            const double norm = sqrt(1.0 + t * t);
            const double hm = (double)hq * c.Q;
            const double drive = c.density * c.gravity * hm * t / norm;
            const double resist = c.cohesion + c.density * c.gravity * hm * c.stop_tan / norm;
            if (!(drive > resist)) a = (double)(hq < c.rate_q ? (long long)hq : c.rate_q);
          }
        }
      }
    } else {
      const double hv = h[gi];
      if (hv > 0.0 && !forced) {
        if (c.settle_tail) {
          a = hv;
        } else {
          const double vx = qx[gi] / hv, vy = qy[gi] / hv;
          if (!(sqrt(vx * vx + vy * vy) > c.speed_threshold)) {
            const int cl = col > 0 ? col - 1 : col, cr = col + 1 < c.nx ? col + 1 : col;
            const int rd = r > 0 ? r - 1 : r, ru = r + 1 < c.ny ? r + 1 : r;
            const double hx = (col == 0 || col + 1 == c.nx) ? c.dx : 2.0 * c.dx;
            const double hy = (r == 0 || r + 1 == c.ny) ? c.dy : 2.0 * c.dy;
            const size_t il = (size_t)r * c.pitch + cl, ir = (size_t)r * c.pitch + cr;
            const size_t id = (size_t)rd * c.pitch + col, iu = (size_t)ru * c.pitch + col;
            // reference order: b[R] + m[R] - b[L] - m[L], left to right
            const double sx = (((b[ir] + h[ir]) - b[il]) - h[il]) / hx;
            const double sy = (((b[iu] + h[iu]) - b[id]) - h[id]) / hy;
            const double t = sqrt(sx * sx + sy * sy);
            const double norm = sqrt(1.0 + t * t);
            const double drive = c.density * c.gravity * hv * t / norm;
            const double resist = c.cohesion + c.density * c.gravity * hv * c.stop_tan / norm;
            if (!(drive > resist)) a = fmin(hv, c.rate * c.dt);
          }
        }
      }
    }
    amount[i] = a;
  }
}

// Pass 2: apply, accumulate the reference's weighted sums (fixed-order block
// partials, last block folds), and add settled volume to the per-cell
// mobile-to-resting record.
template <bool FX>
__global__ void __launch_bounds__(kThreads)
    deposition_apply_kernel(const DepositionConst c, typename FvTypes<FX>::B* __restrict__ b,
                            typename FvTypes<FX>::H* __restrict__ h,
                            typename FvTypes<FX>::R* __restrict__ qx,
                            typename FvTypes<FX>::R* __restrict__ qy,
                            const double* __restrict__ amount, double* __restrict__ m2r_cum,
                            double* __restrict__ partials, unsigned* arrive, DepositionOut* out) {
  const long long n = (long long)c.ny * c.nx;
  const double f = c.dx * c.dy / 6.0;
  long long vq = 0;
  double vw = 0.0, mx = 0.0, my = 0.0;
  int cells = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double a = amount[i];
    if (a == 0.0) continue;
    const int r = (int)(i / c.nx), col = (int)(i % c.nx);
    const size_t gi = (size_t)r * c.pitch + col;
    const int w6 = vertex_weight6(r, col, c.ny, c.nx);
    const double w = (double)w6 * f;
    double rx, ry, settled;
    if constexpr (FX) {
      const int hq = h[gi];
      const int aq = (int)a;
      const float qxo = qx[gi], qyo = qy[gi];
      if (c.settle_tail) {
        rx = qxo;
        ry = qyo;
        qx[gi] = 0.f;
        qy[gi] = 0.f;
      } else {
        const float frac_removed = (float)aq / (float)hq;
        const float fraction = (float)(hq - aq) / (float)hq;
        rx = (double)(qxo * frac_removed);
        ry = (double)(qyo * frac_removed);
        qx[gi] = qxo * fraction;
        qy[gi] = qyo * fraction;
      }
      b[gi] = b[gi] + aq;
      h[gi] = hq - aq;
      vq += (long long)aq * w6;
      settled = (double)aq * c.Q;
    } else {
      const double hv = h[gi];
      if (c.settle_tail) {
        rx = qx[gi];
        ry = qy[gi];
        b[gi] = b[gi] + hv;
        h[gi] = 0.0;
        qx[gi] = 0.0;
        qy[gi] = 0.0;
      } else {
        const double frac_removed = a / hv;
        rx = qx[gi] * frac_removed;
        ry = qy[gi] * frac_removed;
        b[gi] = b[gi] + a;
        h[gi] = hv - a;
        const double fraction = (hv - a) / hv;
        qx[gi] = qx[gi] * fraction;
        qy[gi] = qy[gi] * fraction;
      }
      settled = a;
    }
    if (m2r_cum) m2r_cum[i] = m2r_cum[i] + settled * w;
    vw += settled * w;
    mx += c.density * rx * w;
    my += c.density * ry * w;
    ++cells;
  }
  __shared__ double red[kThreads / 32 * 5];
  __shared__ int last;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double v[5] = {vw, mx, my, (double)cells, 0.0};
  vq = (long long)warp_sum_u64((unsigned long long)vq);
#pragma unroll
  for (int k = 0; k < 4; ++k) v[k] = warp_sum(v[k]);
  if (lane == 0) {
    for (int k = 0; k < 4; ++k) red[warp * 5 + k] = v[k];
    red[warp * 5 + 4] = __longlong_as_double(vq);
  }
  __syncthreads();
  if (threadIdx.x < 5) {
    double s = 0.0;
    long long si = 0;
    for (int w2 = 0; w2 < kThreads / 32; ++w2) {
      if (threadIdx.x == 4) si += __double_as_longlong(red[w2 * 5 + 4]);
      else s += red[w2 * 5 + threadIdx.x];
    }
    partials[(size_t)blockIdx.x * 5 + threadIdx.x] = threadIdx.x == 4 ? __longlong_as_double(si) : s;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = (atomicAdd(arrive, 1u) == gridDim.x - 1) ? 1 : 0;
  __syncthreads();
  if (!last || threadIdx.x != 0) return;
  __threadfence();
  double s[4] = {0.0, 0.0, 0.0, 0.0};
  long long si = 0;
  for (unsigned bk = 0; bk < gridDim.x; ++bk) {
    for (int k = 0; k < 4; ++k) s[k] += __ldcg(partials + (size_t)bk * 5 + k);
    si += __double_as_longlong(__ldcg(partials + (size_t)bk * 5 + 4));
  }
  out->volume_w = s[0];
  out->momentum_w[0] = s[1];
  out->momentum_w[1] = s[2];
  out->cells = (int)s[3];
  out->volume_w6_quanta = si;
  *arrive = 0;
}

}  // namespace sb
