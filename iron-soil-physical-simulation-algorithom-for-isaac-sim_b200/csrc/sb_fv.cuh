// Mobile V2 finite-volume substep kernels.
//
// Equations: reference experimental/mobile_v2_reference.py, ``_face_updates``
// (:365-431), ``_physical_flux`` (:433-449) and the substep body of ``step``
// (:236-307).  One launch = one CFL substep over the whole grid:
//
//   TMA loads a (64 + 2*HX) x (16 + 2) halo tile of b, h, qx, qy into shared
//   memory -> every face touching the tile is evaluated exactly once into
//   shared memory (so both cells of a face see the identical flux) -> each
//   cell gathers its four faces, applies positivity handling, dry zeroing,
//   the external source and Coulomb friction, and writes the other buffer of
//   the ping-pong pair -> the block reduces the next wave-speed maximum and
//   the impulse/energy diagnostics -> the last block to finish reduces all
//   block partials in a fixed order and computes the next substep's dt on the
//   device, so the substep loop never returns to the host.
//
// Precision instantiations:
//   FX = false : double everywhere, operation order identical to the
//                reference NumPy code (bit-identical fields).
//   FX = true  : int32 height quanta (b relative to a datum), float momentum;
//                face mass fluxes are rounded to whole quanta and capped at
//                floor(h_donor/4) per face => exact mass, h >= 0 always.
#pragma once

#include "sb_common.cuh"

namespace sb {

constexpr int kTileX = 64;
constexpr int kTileY = 16;
constexpr int kEastFaces = kTileY * (kTileX + 1);
constexpr int kNorthFaces = (kTileY + 1) * kTileX;
constexpr int kFvDiag = 8;      // cons x,y | ext x,y | fric x,y | fdiss | ework
constexpr int kFvPartial = 10;  // kFvDiag + wave max + positivity flag

struct FvConst {
  int ny, nx, pitch, tiles_x, nblocks;  // FX: tiles_x = column strips, nblocks = launch grid
  int rows_per_warp;                    // batched strips: rows of one warp's strip
  int row_chunks;                       // FX streaming kernel: row chunks per strip
  double dx, dy, K, g, cfl, dry, mu_g, c_half, kg, min_spacing;
  // fixed-point constants
  double Q;
  double gsx[2], gsy[2];  // ledger gradient scales: {Q / (2 dx), Q / dx}, {Q / (2 dy), Q / dy}
  float Kf, KGf, HKGf, Qf, invQf, dryf, QKf;  // QKf = float(Q / K)
  int max_substeps;
  int has_external;
};

// Device-resident loop control block (one per context).
struct FvControl {
  double remaining;
  double sub_dt;
  double max_cfl;
  double wave;
  double diag[kFvDiag];
  int substeps;
  int parity;       // buffer index holding the current state
  int done;         // 1 => substep kernels return immediately
  int status;       // sb_status
  int cfl_limited;
  int static_skip;
  unsigned int arrive;
  int wait_fail;
  unsigned long long wave_bits;  // this substep's wave-speed maximum (atomicMax of the bits)
  int neg_flag;                  // this substep's positivity failure (atomicOr)
  int pad;
  unsigned long long pmax[4];    // "before" ledger maxima for the prologue: external, |q|, grad, wave
  unsigned int gen;              // persistent substep loop: barrier generation
  int pad2;
  // persistent substep loop: substep k's wave-speed maximum goes to slot
  // k % 3 (cleared two substeps ahead by the barrier)
  unsigned long long wave3[3];
};

// Ledger record layout (filled by the ledger kernels of sb_ledger.cuh).
enum LedgerSlot {
  L_HSUM = 0, L_HSUM_W, L_QX, L_QY, L_QX_W, L_QY_W, L_HS2, L_HS2_W, L_HB, L_HB_W, L_HH, L_HH_W,
  L_REST_W,  // FP64: sum max(b - z, 0) * w6
  L_NSUM,
  L_MAXSPEED = L_NSUM, L_NEGMINH, L_MAXQ, L_MAXGRAD, L_MAXWAVE, L_MAXEXT,
  L_NP
};
constexpr int kLedgerI64 = 3;  // h quanta, h quanta * w6, max(b - z, 0) quanta * w6

struct LedgerOut {
  double v[L_NP];
  long long iq[kLedgerI64];
};

struct StepIO {  // per-step device record: ledgers before/after + loop control
  LedgerOut before;
  LedgerOut after;
};

template <bool FX>
struct FvTypes;
template <>
struct FvTypes<true> {
  using H = int32_t;  // height quanta
  using B = int32_t;  // support quanta (datum relative)
  using R = float;    // momentum / arithmetic
};
template <>
struct FvTypes<false> {
  using H = double;
  using B = double;
  using R = double;
};

template <bool FX>
struct FvTile {
  static constexpr int HX = 16 / sizeof(typename FvTypes<FX>::R);  // TMA x alignment
  static constexpr int BW = kTileX + 2 * HX;                        // box width
  static constexpr int BH = kTileY + 2;                             // box height
  static constexpr int BOX = BW * BH;
  static constexpr int BOX_BYTES = BOX * (int)sizeof(typename FvTypes<FX>::R);
  __device__ static int cell(int ly, int lx) { return (ly + 1) * BW + lx + HX; }
};

template <bool FX>
struct FvSmem {
  using T = FvTypes<FX>;
  using Tl = FvTile<FX>;
  using M = typename std::conditional<FX, int32_t, double>::type;  // mass flux type
  alignas(128) typename T::B b[Tl::BOX];
  alignas(128) typename T::H h[Tl::BOX];
  alignas(128) typename T::R qx[Tl::BOX];
  alignas(128) typename T::R qy[Tl::BOX];
  // FX only: per-cell velocity q/h and celerity sqrt(K g h) of the loaded tile
  typename T::R u[Tl::BOX], v[Tl::BOX], cel[Tl::BOX];
  M em[kEastFaces];
  typename T::R enm[kEastFaces], enp[kEastFaces], et[kEastFaces];
  M nm[kNorthFaces];
  typename T::R nnm[kNorthFaces], nnp[kNorthFaces], nt[kNorthFaces];
  uint64_t bar;
  int flag;
};

// --------------------------------------------------------------------------
// Float arithmetic of the FX32 kernels.  FAST = false: IEEE round-to-nearest
// reciprocal, square root and division (the CPU mirror's arithmetic, bit for
// bit, in a translation unit compiled without FMA contraction).  FAST = true
// (production): the PTX approximate instructions rcp.approx.ftz.f32 and
// sqrt.approx.ftz.f32 (relative error ~2^-23) in a translation unit compiled
// with FMA contraction.  Mass stays exact either way: every face mass flux is
// rounded to whole quanta and applied with opposite signs to its two cells.
// --------------------------------------------------------------------------
template <bool FAST>
__device__ __forceinline__ float fx_rcp(float x) {
  if constexpr (FAST) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
  } else {
    return __frcp_rn(x);
  }
}

template <bool FAST>
__device__ __forceinline__ float fx_sqrt(float x) {
  if constexpr (FAST) {
    float r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
  } else {
    return sqrtf(x);
  }
}

// Coulomb friction factor max(0, 1 - dec / max(spd, 1e-15)).
template <bool FAST>
__device__ __forceinline__ float fx_friction(float dec, float spd) {
  if constexpr (FAST) {
    return fmaxf(0.f, 1.f - dec * fx_rcp<true>(fmaxf(spd, 1.0e-15f)));
  } else {
    return fmaxf(0.f, 1.f - dec / fmaxf(spd, 1.0e-15f));
  }
}

// --------------------------------------------------------------------------
// Face fluxes.  (L, R) = (west, east) or (south, north) cell; n/t = normal and
// tangential momentum components.  Outputs: mass flux (quanta or raw),
// normal-momentum flux seen by L (minus) and by R (plus), tangential flux.
// --------------------------------------------------------------------------
// FX face: un/ut are the cells' velocity components q/h (0 for empty cells), cl/cr
// their celerities sqrt(K g h).  The hydrostatic depth only differs from h on
// the lower side of a face (d > 0): it and its celerity are computed once, for
// whichever side is lower, and selected (on a flat face the same expressions
// reproduce h and the prepared celerity exactly), so the face has no branch
// other than the early return for a face between two empty cells (all of a
// terrain away from the mobile layer), whose fluxes are all zero.
// Reconstructed discharge is u * hs (= q * hs / h of the reference).  Roots
// and reciprocals go through fx_sqrt / fx_rcp (IEEE when FAST is false).
template <bool FAST = false>
__device__ __forceinline__ void face_fx(const FvConst& c, float lam, int bl, int br, int hlq,
                                        int hrq, float unl, float utl, float unr, float utr,
                                        float cl, float cr, int& m, float& fnm, float& fnp,
                                        float& ft) {
  if ((hlq | hrq) == 0) {
    // both cells empty: every flux below is a (signed) zero; return +0 (the
    // sign of a zero flux never changes a field value)
    m = 0;
    fnm = fnp = ft = 0.f;
    return;
  }
  const int bface = max(bl, br);
  const int dl = bface - bl;
  const int dr = bface - br;
  const float hl = (float)hlq * c.Qf;
  const float hr = (float)hrq * c.Qf;
  // only the lower side of a face can have a hydrostatic depth below h
  const bool llow = dl != 0;
  const float hlow = llow ? hl : hr;
  const float hs_low = fmaxf(hlow - (float)(dl + dr) * c.QKf, 0.f);
  const float cs_low = fx_sqrt<FAST>(c.KGf * hs_low);
  const float cor_low = (c.HKGf * hlow) * hlow - (c.HKGf * hs_low) * hs_low;
  const float hsl = llow ? hs_low : hl, csl = llow ? cs_low : cl, corl = llow ? cor_low : 0.f;
  const float hsr = llow ? hr : hs_low, csr = llow ? cr : cs_low, corr = llow ? 0.f : cor_low;
  const float qnsl = unl * hsl, qtsl = utl * hsl;
  const float qnsr = unr * hsr, qtsr = utr * hsr;
  const bool wl = hsl > c.dryf, wr = hsr > c.dryf;
  const float vnl = wl ? unl : 0.f, vtl = wl ? utl : 0.f;
  const float vnr = wr ? unr : 0.f, vtr = wr ? utr : 0.f;
  const float fnl = qnsl * vnl + (c.HKGf * hsl) * hsl;
  const float fnr = qnsr * vnr + (c.HKGf * hsr) * hsr;
  const float ftl = qnsl * vtl, ftr = qnsr * vtr;
  const float spd = fmaxf(fabsf(vnl) + csl, fabsf(vnr) + csr);
  const float half = 0.5f * spd;
  const float fh = 0.5f * (qnsl + qnsr) - half * (hsr - hsl);
  const float fn = 0.5f * (fnl + fnr) - half * (qnsr - qnsl);
  ft = 0.5f * (ftl + ftr) - half * (qtsr - qtsl);
  float mf = rintf((lam * fh) * c.invQf);
  mf = fminf(fmaxf(mf, -1073741824.f), 1073741824.f);
  int mi = (int)mf;
  mi = mi > 0 ? min(mi, hlq >> 2) : max(mi, -(hrq >> 2));
  m = mi;
  fnm = fn + corl;
  fnp = fn + corr;
}

__device__ __forceinline__ void face_fp64(const FvConst& c, double bl, double br, double hl,
                                          double hr, double qnl, double qtl, double qnr,
                                          double qtr, double& fh, double& fnm, double& fnp,
                                          double& ft) {
  const double bface = fmax(bl, br);
  const double hsl = fmax(((bl + c.K * hl) - bface) / c.K, 0.0);
  const double hsr = fmax(((br + c.K * hr) - bface) / c.K, 0.0);
  const double sl = hl > c.dry ? hsl / hl : 0.0;
  const double sr = hr > c.dry ? hsr / hr : 0.0;
  const double qnsl = qnl * sl, qtsl = qtl * sl;
  const double qnsr = qnr * sr, qtsr = qtr * sr;
  const bool wl = hsl > c.dry, wr = hsr > c.dry;
  const double unl = wl ? qnsl / hsl : 0.0, utl = wl ? qtsl / hsl : 0.0;
  const double unr = wr ? qnsr / hsr : 0.0, utr = wr ? qtsr / hsr : 0.0;
  const double fnl = qnsl * unl + (c.c_half * hsl) * hsl;
  const double fnr = qnsr * unr + (c.c_half * hsr) * hsr;
  const double ftl = qnsl * utl, ftr = qnsr * utr;
  const double spd = fmax(fabs(unl) + sqrt(c.kg * hsl), fabs(unr) + sqrt(c.kg * hsr));
  const double half = 0.5 * spd;
  fh = 0.5 * (qnsl + qnsr) - half * (hsr - hsl);
  const double fn = 0.5 * (fnl + fnr) - half * (qnsr - qnsl);
  ft = 0.5 * (ftl + ftr) - half * (qtsr - qtsl);
  fnm = fn + ((c.c_half * hl) * hl - (c.c_half * hsl) * hsl);
  fnp = fn + ((c.c_half * hr) * hr - (c.c_half * hsr) * hsr);
}

// --------------------------------------------------------------------------
// Finalisation of one substep by the last block: fixed-order reduction of the
// block partials, loop control, next dt.
// --------------------------------------------------------------------------
// Grid reduction of block partials stored slot-major (partials[k * nblocks +
// block]): thread t folds blocks t, t + kThreads, ... in order (coalesced
// loads), then the block folds the threads in a fixed order.  Slots [0, NSUM)
// are sums, [NSUM, NP) maxima (0 is the identity of both: every maximum here is
// of non-negative values or only tested against 0).  Returns a pointer into
// scratch (fold_words(NP) doubles).
template <int NP, int NSUM>
__device__ const double* reduce_partials(const double* partials, int nblocks, double* scratch) {
  double v[NP];
#pragma unroll
  for (int k = 0; k < NP; ++k) v[k] = 0.0;
  for (int b = threadIdx.x; b < nblocks; b += kThreads) {
#pragma unroll
    for (int k = 0; k < NP; ++k) {
      const double x = __ldcg(partials + (size_t)k * nblocks + b);
      v[k] = k >= NSUM ? fmax(v[k], x) : v[k] + x;
    }
  }
  return block_fold<double, NP, NSUM>(v, scratch);
}

// Computes sub_dt/max_cfl for the next substep from ctl->wave (CPU: reference
// step :247-257).  Called by one thread.
__device__ __forceinline__ void plan_substep(const FvConst& c, FvControl* ctl) {
  const double w = ctl->wave;
  const double rem = ctl->remaining;
  const double stable = w <= 1.0e-14 ? rem : c.cfl * c.min_spacing / w;
  const double sub = fmin(rem, stable);
  if (sub < rem - 1.0e-14) ctl->cfl_limited = 1;
  ctl->max_cfl = fmax(ctl->max_cfl, w * sub / c.min_spacing);
  ctl->sub_dt = sub;
}

// Loop control after the last block of a substep has arrived (one thread):
// substep count, remaining time, ping-pong parity, error status and the next
// substep's dt from this substep's wave-speed maximum.
__device__ __forceinline__ void fv_advance(const FvConst& c, FvControl* ctl, double sub_dt,
                                           int parity) {
  const double w = __longlong_as_double((long long)atomicExch(&ctl->wave_bits, 0ull));
  const int failed = atomicExch(&ctl->neg_flag, 0);
  ctl->substeps += 1;
  ctl->remaining -= sub_dt;
  ctl->parity = parity ^ 1;
  ctl->wave = w;
  ctl->arrive = 0;
  if (ctl->wait_fail) {
    ctl->status = 6;  // SB_ERR_WAIT_LIMIT
    ctl->done = 1;
  } else if (failed) {
    ctl->status = 3;  // SB_ERR_POSITIVITY
    ctl->done = 1;
  } else if (!(ctl->remaining > 1.0e-14)) {
    ctl->done = 1;
  } else if (ctl->substeps >= c.max_substeps) {
    ctl->status = 2;  // SB_ERR_SUBSTEP_CAP
    ctl->done = 1;
  } else {
    plan_substep(c, ctl);
  }
}

// End of one substep.  Every block folds its impulse/energy sums, wave
// maximum and positivity flag (fixed order); the sums are added to the block's
// own accumulators (diag_acc[k * nblocks + block], summed over the step's
// substeps and folded by the after-step ledger), the maximum and the flag go
// to the control block by atomicMax / atomicOr (order-free, so deterministic).
// The last block to arrive then only reads those two words: substep count,
// remaining time, ping-pong parity, error status and the next substep's dt;
// the graph's while-condition is set from here.
__device__ __forceinline__ void fv_finish(const FvConst& c, FvControl* ctl, double* diag_acc,
                                          const double* acc, double wave, int neg, int* flag,
                                          double sub_dt, int parity,
                                          cudaGraphConditionalHandle loop_handle, int use_handle) {
  __shared__ double fold[fold_words(kFvPartial)];
  double v[kFvPartial];
#pragma unroll
  for (int k = 0; k < kFvDiag; ++k) v[k] = acc[k];
  v[kFvDiag] = wave;
  v[kFvDiag + 1] = neg ? 1.0 : 0.0;
  const double* bt = block_fold<double, kFvPartial, kFvDiag>(v, fold);
  if (threadIdx.x < kFvDiag) {
    double* a = diag_acc + (size_t)threadIdx.x * c.nblocks + blockIdx.x;
    *a = *a + bt[threadIdx.x];
  } else if (threadIdx.x == kFvDiag) {  // wave >= 0: its bits order like the values
    atomicMax(&ctl->wave_bits, (unsigned long long)__double_as_longlong(bt[kFvDiag]));
  } else if (threadIdx.x == kFvDiag + 1 && bt[kFvDiag + 1] != 0.0) {
    atomicOr(&ctl->neg_flag, 1);
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned prev = atomicAdd(&ctl->arrive, 1u);
    *flag = (prev == (unsigned)c.nblocks - 1) ? 1 : 0;
  }
  __syncthreads();
  if (!*flag || threadIdx.x != 0) return;
  __threadfence();
  fv_advance(c, ctl, sub_dt, parity);
  __threadfence();
  if (use_handle) cudaGraphSetConditional(loop_handle, ctl->done ? 0u : 1u);
}

template <bool FX>
__global__ void __launch_bounds__(kThreads)
    fv_substep_kernel(const FvConst c, const __grid_constant__ CUtensorMap tm_b,
                      const __grid_constant__ CUtensorMap tm_h0,
                      const __grid_constant__ CUtensorMap tm_h1,
                      const __grid_constant__ CUtensorMap tm_qx0,
                      const __grid_constant__ CUtensorMap tm_qx1,
                      const __grid_constant__ CUtensorMap tm_qy0,
                      const __grid_constant__ CUtensorMap tm_qy1,
                      typename FvTypes<FX>::H* __restrict__ h0,
                      typename FvTypes<FX>::H* __restrict__ h1,
                      typename FvTypes<FX>::R* __restrict__ qx0,
                      typename FvTypes<FX>::R* __restrict__ qx1,
                      typename FvTypes<FX>::R* __restrict__ qy0,
                      typename FvTypes<FX>::R* __restrict__ qy1,
                      const typename FvTypes<FX>::R* __restrict__ ext_x,
                      const typename FvTypes<FX>::R* __restrict__ ext_y, FvControl* ctl,
                      double* __restrict__ diag_acc, cudaGraphConditionalHandle loop_handle,
                      int use_handle) {
  using T = FvTypes<FX>;
  using Tl = FvTile<FX>;
  using R = typename T::R;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  // TMA destinations need 128-byte alignment; the launch reserves 128 spare bytes.
  unsigned char* smem_base = smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u);
  FvSmem<FX>& s = *reinterpret_cast<FvSmem<FX>*>(smem_base);

  if (*(volatile int*)&ctl->done) return;  // uniform across the grid
  const double sub_dt = ctl->sub_dt;
  const int parity = ctl->parity;
  const int tile_x = blockIdx.x % c.tiles_x;
  const int tile_y = blockIdx.x / c.tiles_x;
  const int gx0 = tile_x * kTileX, gy0 = tile_y * kTileY;

  // ---- TMA: halo tile of the four fields -------------------------------
  if (threadIdx.x == 0) {
    mbar_init(&s.bar, 1);
    s.flag = 0;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const CUtensorMap* mh = parity ? &tm_h1 : &tm_h0;
    const CUtensorMap* mx = parity ? &tm_qx1 : &tm_qx0;
    const CUtensorMap* my = parity ? &tm_qy1 : &tm_qy0;
    mbar_expect_tx(&s.bar, 4 * Tl::BOX_BYTES);
    const int x0 = gx0 - Tl::HX, y0 = gy0 - 1;
    tma_load_2d(s.b, &tm_b, x0, y0, &s.bar);
    tma_load_2d(s.h, mh, x0, y0, &s.bar);
    tma_load_2d(s.qx, mx, x0, y0, &s.bar);
    tma_load_2d(s.qy, my, x0, y0, &s.bar);
  }
  const bool loaded = mbar_wait(&s.bar, 0);
  if (!loaded) {
    if (threadIdx.x == 0) atomicExch(&ctl->wait_fail, 1);
  }
  if constexpr (FX) {
    // per-cell velocity and celerity of the whole halo box
    for (int j = threadIdx.x; j < Tl::BOX; j += kThreads) {
      const float hf = (float)s.h[j] * c.Qf;
      const float inv = s.h[j] > 0 ? __frcp_rn(hf) : 0.f;
      s.u[j] = s.qx[j] * inv;
      s.v[j] = s.qy[j] * inv;
      s.cel[j] = sqrtf(c.KGf * hf);
    }
    __syncthreads();
  }
  const float lamx_f = (float)(sub_dt / c.dx);
  const float lamy_f = (float)(sub_dt / c.dy);
  const double lamx = sub_dt / c.dx;
  const double lamy = sub_dt / c.dy;

  // ---- Faces --------------------------------------------------------------
  for (int f = threadIdx.x; f < kEastFaces + kNorthFaces; f += kThreads) {
    const bool east = f < kEastFaces;
    int ly, lx, la, lb;
    bool valid;
    if (east) {
      ly = f / (kTileX + 1);
      lx = f % (kTileX + 1) - 1;
      const int gx = gx0 + lx, gy = gy0 + ly;
      valid = loaded && gx >= 0 && gx + 1 < c.nx && gy < c.ny;
      la = Tl::cell(ly, lx);
      lb = la + 1;
    } else {
      const int g = f - kEastFaces;
      ly = g / kTileX - 1;
      lx = g % kTileX;
      const int gx = gx0 + lx, gy = gy0 + ly;
      valid = loaded && gy >= 0 && gy + 1 < c.ny && gx < c.nx;
      la = Tl::cell(ly, lx);
      lb = la + Tl::BW;
    }
    if constexpr (FX) {
      int m = 0;
      float fnm = 0.f, fnp = 0.f, ft = 0.f;
      if (valid) {
        if (east)
          face_fx(c, lamx_f, s.b[la], s.b[lb], s.h[la], s.h[lb], s.u[la], s.v[la], s.u[lb],
                  s.v[lb], s.cel[la], s.cel[lb], m, fnm, fnp, ft);
        else
          face_fx(c, lamy_f, s.b[la], s.b[lb], s.h[la], s.h[lb], s.v[la], s.u[la], s.v[lb],
                  s.u[lb], s.cel[la], s.cel[lb], m, fnm, fnp, ft);
      }
      if (east) {
        s.em[f] = m; s.enm[f] = fnm; s.enp[f] = fnp; s.et[f] = ft;
      } else {
        const int g = f - kEastFaces;
        s.nm[g] = m; s.nnm[g] = fnm; s.nnp[g] = fnp; s.nt[g] = ft;
      }
    } else {
      double fh = 0.0, fnm = 0.0, fnp = 0.0, ft = 0.0;
      if (valid) {
        if (east)
          face_fp64(c, s.b[la], s.b[lb], s.h[la], s.h[lb], s.qx[la], s.qy[la], s.qx[lb],
                    s.qy[lb], fh, fnm, fnp, ft);
        else
          face_fp64(c, s.b[la], s.b[lb], s.h[la], s.h[lb], s.qy[la], s.qx[la], s.qy[lb],
                    s.qx[lb], fh, fnm, fnp, ft);
      }
      if (east) {
        s.em[f] = fh; s.enm[f] = fnm; s.enp[f] = fnp; s.et[f] = ft;
      } else {
        const int g = f - kEastFaces;
        s.nm[g] = fh; s.nnm[g] = fnm; s.nnp[g] = fnp; s.nt[g] = ft;
      }
    }
  }
  __syncthreads();

  // ---- Cells --------------------------------------------------------------
  typename T::H* hdst = parity ? h0 : h1;
  R* qxdst = parity ? qx0 : qx1;
  R* qydst = parity ? qy0 : qy1;
  double acc[kFvDiag];
#pragma unroll
  for (int k = 0; k < kFvDiag; ++k) acc[k] = 0.0;
  double wave = 0.0;
  int neg = 0;
  for (int i = threadIdx.x; i < kTileX * kTileY; i += kThreads) {
    const int ly = i / kTileX, lx = i % kTileX;
    const int gy = gy0 + ly, gx = gx0 + lx;
    if (gy >= c.ny || gx >= c.nx || !loaded) continue;
    const int e = ly * (kTileX + 1) + lx + 1;  // east face of this cell
    const int w = e - 1;                       // west face
    const int n = (ly + 1) * kTileX + lx;      // north face
    const int so = n - kTileX;                 // south face
    const int cs = Tl::cell(ly, lx);
    const size_t gi = (size_t)gy * c.pitch + gx;
    R ax = R(0), ay = R(0);
    if (c.has_external) {
      ax = ext_x[gi];
      ay = ext_y[gi];
    }
    if constexpr (FX) {
      const int dh = ((0 - s.em[e] + s.em[w]) - s.nm[n]) + s.nm[so];
      const int hq = s.h[cs] + dh;
      const float zero = 0.f;
      const float dqx =
          (((zero - lamx_f * s.enm[e]) + lamx_f * s.enp[w]) - lamy_f * s.nt[n]) + lamy_f * s.nt[so];
      const float dqy =
          (((zero - lamx_f * s.et[e]) + lamx_f * s.et[w]) - lamy_f * s.nnm[n]) + lamy_f * s.nnp[so];
      const float qx_old = s.qx[cs], qy_old = s.qy[cs];
      const float hn = (float)hq * c.Qf;
      const bool wet = hn > c.dryf;
      const float qxn = wet ? qx_old + dqx : 0.f;
      const float qyn = wet ? qy_old + dqy : 0.f;
      float vbx = 0.f, vby = 0.f, qex = qxn, qey = qyn, vex = 0.f, vey = 0.f;
      if (wet) {
        const float inv = __frcp_rn(hn);
        vbx = qxn * inv;
        vby = qyn * inv;
        if (c.has_external) {
          const float dtf = (float)sub_dt;
          qex = qxn + (hn * ax) * dtf;
          qey = qyn + (hn * ay) * dtf;
          vex = qex * inv;
          vey = qey * inv;
        } else {
          vex = vbx;
          vey = vby;
        }
      }
      const float spd = sqrtf(vex * vex + vey * vey);
      const float dec = (float)(c.mu_g * sub_dt);
      const float fac = fmaxf(0.f, 1.f - dec / fmaxf(spd, 1.0e-15f));
      const float vax = vex * fac, vay = vey * fac;
      const float qxo = hn * vax, qyo = hn * vay;
      hdst[gi] = hq;
      qxdst[gi] = qxo;
      qydst[gi] = qyo;
      const double h64 = (double)hn;
      acc[0] += (double)qxn - (double)qx_old;
      acc[1] += (double)qyn - (double)qy_old;
      acc[2] += (double)qex - (double)qxn;
      acc[3] += (double)qey - (double)qyn;
      acc[4] += (double)qxo - (double)qex;
      acc[5] += (double)qyo - (double)qey;
      acc[6] += 0.5 * h64 *
                ((double)spd * (double)spd - ((double)vax * (double)vax + (double)vay * (double)vay));
      acc[7] += h64 * ((0.5 * ((double)vbx + (double)vex)) * (double)ax +
                       (0.5 * ((double)vby + (double)vey)) * (double)ay) * sub_dt;
      const float wv = spd * fac + sqrtf(c.KGf * hn);  // |new velocity| + celerity
      wave = fmax(wave, (double)wv);
    } else {
      const double dh = (((0.0 - lamx * s.em[e]) + lamx * s.em[w]) - lamy * s.nm[n]) + lamy * s.nm[so];
      const double dqx =
          (((0.0 - lamx * s.enm[e]) + lamx * s.enp[w]) - lamy * s.nt[n]) + lamy * s.nt[so];
      const double dqy =
          (((0.0 - lamx * s.et[e]) + lamx * s.et[w]) - lamy * s.nnm[n]) + lamy * s.nnp[so];
      double hn = s.h[cs] + dh;
      const double qx_old = s.qx[cs], qy_old = s.qy[cs];
      double qxn = qx_old + dqx, qyn = qy_old + dqy;
      if (hn < -2.0e-13) neg = 1;
      hn = fmax(hn, 0.0);
      const bool wet = hn > c.dry;
      if (!wet) {
        qxn = 0.0;
        qyn = 0.0;
      }
      double vbx = 0.0, vby = 0.0, vex = 0.0, vey = 0.0;
      const double qex = qxn + (hn * ax) * sub_dt;
      const double qey = qyn + (hn * ay) * sub_dt;
      if (wet) {
        vbx = qxn / hn;
        vby = qyn / hn;
        vex = qex / hn;
        vey = qey / hn;
      }
      const double spd = sqrt(vex * vex + vey * vey);
      const double dec = c.mu_g * sub_dt;
      const double fac = fmax(0.0, 1.0 - dec / fmax(spd, 1.0e-15));
      const double vax = vex * fac, vay = vey * fac;
      const double qxo = hn * vax, qyo = hn * vay;
      hdst[gi] = hn;
      qxdst[gi] = qxo;
      qydst[gi] = qyo;
      acc[0] += qxn - qx_old;
      acc[1] += qyn - qy_old;
      acc[2] += qex - qxn;
      acc[3] += qey - qyn;
      acc[4] += qxo - qex;
      acc[5] += qyo - qey;
      acc[6] += 0.5 * (hn * (spd * spd - (vax * vax + vay * vay)));
      acc[7] += hn * ((0.5 * (vbx + vex)) * ax + (0.5 * (vby + vey)) * ay) * sub_dt;
      double vx = 0.0, vy = 0.0;
      if (wet) {
        vx = qxo / hn;
        vy = qyo / hn;
      }
      wave = fmax(wave, sqrt(vx * vx + vy * vy) + sqrt(c.kg * hn));
    }
  }

  fv_finish(c, ctl, diag_acc, acc, wave, neg, &s.flag, sub_dt, parity, loop_handle,
            use_handle);
}

// --------------------------------------------------------------------------
// FX32 substep as a register-streaming stencil.
//
// A warp owns a strip of 32 columns (lanes 1..30 are output columns, lanes 0
// and 31 their west/east neighbours) and walks down a chunk of rows.  Per
// row every lane evaluates the east face of its column (the east neighbour's
// state arrives by shuffle) and the north face (the next row is already in
// registers); the west face is the previous lane's east face (one more
// shuffle) and the south face is the previous row's north face, carried in
// registers.  Each interior face is therefore evaluated once, in registers:
// nothing is staged in shared memory, the only shared memory use is the
// block reduction.  The row after next is loaded while the current row is
// computed.  The face and cell arithmetic is the same as the tile kernel's,
// so both produce identical fields.
// --------------------------------------------------------------------------
constexpr int kStripOut = 30;
constexpr int kMinChunkRows = 5;  // shortest row chunk of one strip warp (701^2 sweep: 4 / 5 / 6 / 8 rows -> 13.4 / 13.1 / 13.9 / 14.3 us per substep)

struct FxCell {
  int b, h;
  float qx, qy, u, v, cel;
};

// CG = false: read-only-cache loads (fields written by an earlier launch);
// CG = true: L2-coherent loads (fields written by other CTAs of the same
// persistent launch in the previous substep).
template <bool CG>
__device__ __forceinline__ void fx_load(const FvConst& c, const int32_t* __restrict__ b,
                                        const int32_t* __restrict__ h,
                                        const float* __restrict__ qx,
                                        const float* __restrict__ qy, int row, int gx, bool colok,
                                        FxCell& x) {
  if (colok && row >= 0 && row < c.ny) {
    const size_t gi = (size_t)row * c.pitch + gx;
    x.b = __ldg(b + gi);  // the support does not change during a substep loop
    if constexpr (CG) {
      x.h = __ldcg(h + gi);
      x.qx = __ldcg(qx + gi);
      x.qy = __ldcg(qy + gi);
    } else {
      x.h = __ldg(h + gi);
      x.qx = __ldg(qx + gi);
      x.qy = __ldg(qy + gi);
    }
  } else {
    x.b = 0;
    x.h = 0;
    x.qx = 0.f;
    x.qy = 0.f;
  }
}

// Per-cell velocity q/h (0 for an empty cell) and celerity sqrt(K g h).
template <bool FAST>
__device__ __forceinline__ void fx_prepare(const FvConst& c, FxCell& x) {
  if (x.h > 0) {
    const float hf = (float)x.h * c.Qf;
    const float inv = fx_rcp<FAST>(hf);
    x.u = x.qx * inv;
    x.v = x.qy * inv;
    x.cel = fx_sqrt<FAST>(c.KGf * hf);
  } else {  // empty cell (the same values: q * 0 and sqrt(0)); no reciprocal or root
    x.u = x.qx * 0.f;
    x.v = x.qy * 0.f;
    x.cel = 0.f;
  }
}

// One warp's strip: columns strip*30-1 .. strip*30+30, rows y0 .. y1-1
// of a grid whose row 0 starts at the given field pointers (row pitch
// c.pitch).  Accumulates the impulse/energy sums into acc and the largest
// next-substep wave speed into wave.  Every lane of the warp must call it.
template <bool FAST = false, bool CG = false>
__device__ __forceinline__ void fx_strip_run(const FvConst& c, const int32_t* __restrict__ bsrc,
                                             const int32_t* __restrict__ hsrc,
                                             const float* __restrict__ qxsrc,
                                             const float* __restrict__ qysrc,
                                             int32_t* __restrict__ hdst, float* __restrict__ qxdst,
                                             float* __restrict__ qydst,
                                             const float* __restrict__ ext_x,
                                             const float* __restrict__ ext_y, int strip, int y0,
                                             int y1, double sub_dt, double* acc, double& wave) {
  const int lane = threadIdx.x & 31;
  const int gx = strip * kStripOut - 1 + lane;
  const bool colok = gx >= 0 && gx < c.nx;
  const bool out_lane = lane >= 1 && lane <= kStripOut && colok;
  const bool east_ok = gx >= 0 && gx + 1 < c.nx && lane < 31;
  const float lamx_f = (float)(sub_dt / c.dx);
  const float lamy_f = (float)(sub_dt / c.dy);
  const float dtf = (float)sub_dt;
  const float dec = (float)(c.mu_g * sub_dt);
  if (y0 >= c.ny) return;  // warp-uniform
  float fa[kFvDiag] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  float fwave = 0.f;
  FxCell cur, nxt, nn;
  fx_load<CG>(c, bsrc, hsrc, qxsrc, qysrc, y0, gx, colok, cur);
  fx_load<CG>(c, bsrc, hsrc, qxsrc, qysrc, y0 + 1, gx, colok, nxt);
  // south face of the first row (the previous row's north face)
  int ms = 0;
  float nts = 0.f, nnps = 0.f;
  {
    FxCell prv;
    fx_load<CG>(c, bsrc, hsrc, qxsrc, qysrc, y0 - 1, gx, colok, prv);
    fx_prepare<FAST>(c, prv);
    fx_prepare<FAST>(c, cur);
    if (y0 > 0 && colok) {
      float fnm;
      face_fx<FAST>(c, lamy_f, prv.b, cur.b, prv.h, cur.h, prv.v, prv.u, cur.v, cur.u, prv.cel,
              cur.cel, ms, fnm, nnps, nts);
    }
  }
  fx_prepare<FAST>(c, nxt);
#pragma unroll 2
  for (int r = y0; r < y1; ++r) {
    fx_load<CG>(c, bsrc, hsrc, qxsrc, qysrc, r + 2, gx, colok, nn);
    // east face: this column and the next lane's
    const int eb = __shfl_down_sync(0xffffffffu, cur.b, 1);
    const int eh = __shfl_down_sync(0xffffffffu, cur.h, 1);
    const float eu = __shfl_down_sync(0xffffffffu, cur.u, 1);
    const float ev = __shfl_down_sync(0xffffffffu, cur.v, 1);
    const float ec = __shfl_down_sync(0xffffffffu, cur.cel, 1);
    int me = 0;
    float enm = 0.f, enp = 0.f, et = 0.f;
    if (east_ok)
      face_fx<FAST>(c, lamx_f, cur.b, eb, cur.h, eh, cur.u, cur.v, eu, ev, cur.cel, ec, me, enm, enp,
              et);
    // west face = the previous lane's east face
    const int mw = __shfl_up_sync(0xffffffffu, me, 1);
    const float enpw = __shfl_up_sync(0xffffffffu, enp, 1);
    const float etw = __shfl_up_sync(0xffffffffu, et, 1);
    // north face: this row and the next
    int mn = 0;
    float nnm = 0.f, nnp = 0.f, nt = 0.f;
    if (colok && r + 1 < c.ny)
      face_fx<FAST>(c, lamy_f, cur.b, nxt.b, cur.h, nxt.h, cur.v, cur.u, nxt.v, nxt.u, cur.cel,
              nxt.cel, mn, nnm, nnp, nt);
    if (out_lane) {
      const size_t gi = (size_t)r * c.pitch + gx;
      float ax = 0.f, ay = 0.f;
      if (c.has_external) {
        ax = ext_x[gi];
        ay = ext_y[gi];
      }
      const int dh = ((0 - me + mw) - mn) + ms;
      const int hq = cur.h + dh;
      const float zero = 0.f;
      const float dqx = (((zero - lamx_f * enm) + lamx_f * enpw) - lamy_f * nt) + lamy_f * nts;
      const float dqy = (((zero - lamx_f * et) + lamx_f * etw) - lamy_f * nnm) + lamy_f * nnps;
      const float hn = (float)hq * c.Qf;
      const bool wet = hn > c.dryf;
      const float qxn = wet ? cur.qx + dqx : 0.f;
      const float qyn = wet ? cur.qy + dqy : 0.f;
      float vbx = 0.f, vby = 0.f, qex = qxn, qey = qyn, vex = 0.f, vey = 0.f;
      if (wet) {
        const float inv = fx_rcp<FAST>(hn);
        vbx = qxn * inv;
        vby = qyn * inv;
        if (c.has_external) {
          qex = qxn + (hn * ax) * dtf;
          qey = qyn + (hn * ay) * dtf;
          vex = qex * inv;
          vey = qey * inv;
        } else {
          vex = vbx;
          vey = vby;
        }
      }
      const float spd = fx_sqrt<FAST>(vex * vex + vey * vey);
      const float fac = fx_friction<FAST>(dec, spd);
      const float vax = vex * fac, vay = vey * fac;
      const float qxo = hn * vax, qyo = hn * vay;
      hdst[gi] = hq;
      qxdst[gi] = qxo;
      qydst[gi] = qyo;
      // per-lane diagnostics in float over this strip (one cell per row of
      // the chunk), folded into the double sums once at the end
      fa[0] += qxn - cur.qx;
      fa[1] += qyn - cur.qy;
      fa[2] += qex - qxn;
      fa[3] += qey - qyn;
      fa[4] += qxo - qex;
      fa[5] += qyo - qey;
      // friction dissipation 0.5 h (|v|^2 - |v fac|^2) = 0.5 h |v|^2 (1 - fac)(1 + fac)
      fa[6] += ((0.5f * hn) * (spd * spd)) * ((1.f - fac) * (1.f + fac));
      if (c.has_external)
        fa[7] += (hn * ((0.5f * (vbx + vex)) * ax + (0.5f * (vby + vey)) * ay)) * dtf;
      const float wv = spd * fac + fx_sqrt<FAST>(c.KGf * hn);  // |new velocity| + celerity
      fwave = fmaxf(fwave, wv);
    }
    ms = mn;
    nts = nt;
    nnps = nnp;
    cur = nxt;
    nxt = nn;
    fx_prepare<FAST>(c, nxt);
  }
#pragma unroll
  for (int k = 0; k < kFvDiag; ++k) acc[k] += (double)fa[k];
  wave = fmax(wave, (double)fwave);
}

template <bool FAST>
__global__ void __launch_bounds__(kThreads, 4)
    fv_stream_kernel(const FvConst c, const int32_t* __restrict__ bsrc, int32_t* __restrict__ h0,
                     int32_t* __restrict__ h1, float* __restrict__ qx0, float* __restrict__ qx1,
                     float* __restrict__ qy0, float* __restrict__ qy1,
                     const float* __restrict__ ext_x, const float* __restrict__ ext_y,
                     FvControl* ctl, double* __restrict__ diag_acc,
                     cudaGraphConditionalHandle loop_handle, int use_handle) {
  __shared__ int flag;
  if (*(volatile int*)&ctl->done) return;  // uniform across the grid
  const double sub_dt = ctl->sub_dt;
  const int parity = ctl->parity;
  const int gw = blockIdx.x * (kThreads / 32) + (threadIdx.x >> 5);
  double acc[kFvDiag];
#pragma unroll
  for (int k = 0; k < kFvDiag; ++k) acc[k] = 0.0;
  double wave = 0.0;
  // row chunk j of the strip: rows [j*ny/J, (j+1)*ny/J), balanced to within one row
  const int j = gw / c.tiles_x, nchunk = c.row_chunks;
  const int y0 = j < nchunk ? (int)((long long)j * c.ny / nchunk) : c.ny;
  const int y1 = j < nchunk ? (int)((long long)(j + 1) * c.ny / nchunk) : c.ny;
  fx_strip_run<FAST>(c, bsrc, parity ? h1 : h0, parity ? qx1 : qx0, parity ? qy1 : qy0,
               parity ? h0 : h1, parity ? qx0 : qx1, parity ? qy0 : qy1, ext_x, ext_y,
               gw % c.tiles_x, y0, y1, sub_dt, acc, wave);
  fv_finish(c, ctl, diag_acc, acc, wave, 0, &flag, sub_dt, parity, loop_handle, use_handle);
}

// --------------------------------------------------------------------------
// Persistent FX32 substep loop: one cooperative launch (every CTA resident)
// runs all CFL substeps of a physics step.  Each warp keeps its strip chunk
// for the whole step; between substeps the CTAs meet at a grid barrier whose
// last arrival advances the loop control (fv_advance: count, remaining time,
// parity, status, next dt from the substep's wave-speed maximum, which every
// CTA sent by atomicMax) and releases the others by bumping a generation
// word.  The impulse/energy sums stay in each lane's registers across the
// substeps and are folded once per step, so a substep ends with one warp
// maximum and one atomic per CTA.  Field loads in the loop are L2-coherent
// (the previous substep's writes come from other CTAs of this launch).  The
// barrier wait is bounded: after kFvBarrierPolls polls the CTA records a wait
// failure (SB_ERR_WAIT_LIMIT) and the loop ends.
// --------------------------------------------------------------------------
constexpr unsigned kFvBarrierPolls = 1u << 22;

template <bool FAST>
__global__ void __launch_bounds__(kThreads, 4)
    fv_loop_kernel(const FvConst c, const int32_t* __restrict__ bsrc, int32_t* h0, int32_t* h1,
                   float* qx0, float* qx1, float* qy0, float* qy1,
                   const float* __restrict__ ext_x, const float* __restrict__ ext_y,
                   FvControl* ctl, double* __restrict__ diag_acc) {
  __shared__ double fold[fold_words(kFvDiag)];
  __shared__ double wred[kThreads / 32];
  __shared__ unsigned s_gen;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int gw = blockIdx.x * (kThreads / 32) + warp;
  const int j = gw / c.tiles_x, nchunk = c.row_chunks;
  const int y0 = j < nchunk ? (int)((long long)j * c.ny / nchunk) : c.ny;
  const int y1 = j < nchunk ? (int)((long long)(j + 1) * c.ny / nchunk) : c.ny;
  const int strip = gw % c.tiles_x;
  double acc[kFvDiag];
#pragma unroll
  for (int k = 0; k < kFvDiag; ++k) acc[k] = 0.0;
  // The loop control (remaining time, dt, parity, substep count) is the same
  // arithmetic in every CTA, so each CTA keeps its own copy in shared memory
  // (thread 0 advances it): a barrier needs one wave-speed maximum (slot
  // k % 3) and the release, and no CTA waits for one thread of another CTA to
  // plan the next substep.
  struct LoopCtl {
    double remaining, sub_dt, max_cfl, wave;
    int parity, substeps, cfl_limited, status, done;
  };
  __shared__ LoopCtl L;
  if (threadIdx.x == 0) {
    L.remaining = *(volatile double*)&ctl->remaining;
    L.sub_dt = *(volatile double*)&ctl->sub_dt;
    L.max_cfl = *(volatile double*)&ctl->max_cfl;
    L.wave = *(volatile double*)&ctl->wave;
    L.parity = *(volatile int*)&ctl->parity;
    L.substeps = *(volatile int*)&ctl->substeps;
    L.cfl_limited = *(volatile int*)&ctl->cfl_limited;
    L.status = *(volatile int*)&ctl->status;
    L.done = *(volatile int*)&ctl->done;
  }
  __syncthreads();
  for (int k = 0; !L.done; ++k) {
    const double sub_dt = L.sub_dt;
    const int parity = L.parity;
    if (threadIdx.x == 0) s_gen = *(volatile unsigned*)&ctl->gen;
    double wave = 0.0;
    fx_strip_run<FAST, true>(c, bsrc, parity ? h1 : h0, parity ? qx1 : qx0, parity ? qy1 : qy0,
                             parity ? h0 : h1, parity ? qx0 : qx1, parity ? qy0 : qy1, ext_x,
                             ext_y, strip, y0, y1, sub_dt, acc, wave);
    wave = warp_max(wave);
    if (lane == 0) wred[warp] = wave;
    // the CTA barrier orders every thread's field writes before thread 0's
    // device-scope fence and arrival (the grid-barrier pattern: one fence)
    __syncthreads();
    if (threadIdx.x == 0) {
      double m = 0.0;
#pragma unroll
      for (int w = 0; w < kThreads / 32; ++w) m = fmax(m, wred[w]);
      atomicMax(&ctl->wave3[k % 3], (unsigned long long)__double_as_longlong(m));
      __threadfence();
      const unsigned prev = atomicAdd(&ctl->arrive, 1u);
      bool failed = false;
      if (prev == gridDim.x - 1) {
        ctl->arrive = 0;
        ctl->wave3[(k + 1) % 3] = 0ull;  // read by every CTA two barriers ago
        __threadfence();
        atomicAdd(&ctl->gen, 1u);  // release
      } else {
        unsigned polls = 0;
        while (*(volatile unsigned*)&ctl->gen == s_gen) {
          if (++polls > kFvBarrierPolls) {
            failed = true;
            break;
          }
          if (polls > 64) __nanosleep(32);
        }
        __threadfence();
      }
      // fv_advance on this CTA's copy
      L.substeps += 1;
      L.remaining -= sub_dt;
      L.parity = parity ^ 1;
      if (failed) {
        L.status = 6;  // SB_ERR_WAIT_LIMIT
        L.done = 1;
        ctl->wait_fail = 1;
      } else {
        const double w = __longlong_as_double((long long)__ldcg(&ctl->wave3[k % 3]));
        L.wave = w;
        if (!(L.remaining > 1.0e-14)) {
          L.done = 1;
        } else if (L.substeps >= c.max_substeps) {
          L.status = 2;  // SB_ERR_SUBSTEP_CAP
          L.done = 1;
        } else {  // plan_substep
          const double rem = L.remaining;
          const double stable = w <= 1.0e-14 ? rem : c.cfl * c.min_spacing / w;
          const double sub = fmin(rem, stable);
          if (sub < rem - 1.0e-14) L.cfl_limited = 1;
          L.max_cfl = fmax(L.max_cfl, w * sub / c.min_spacing);
          L.sub_dt = sub;
        }
      }
    }
    __syncthreads();
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    // every CTA holds the same loop control; one writes it back
    ctl->remaining = L.remaining;
    ctl->sub_dt = L.sub_dt;
    ctl->max_cfl = L.max_cfl;
    ctl->wave = L.wave;
    ctl->parity = L.parity;
    ctl->substeps = L.substeps;
    ctl->cfl_limited = L.cfl_limited;
    ctl->status = L.status;
    ctl->done = 1;
  }
  // the step's impulse/energy sums of this CTA, once
  const double* bt = block_fold<double, kFvDiag, kFvDiag>(acc, fold);
  if (threadIdx.x < kFvDiag) {
    double* a = diag_acc + (size_t)threadIdx.x * c.nblocks + blockIdx.x;
    *a = *a + bt[threadIdx.x];
  }
}

}  // namespace sb
