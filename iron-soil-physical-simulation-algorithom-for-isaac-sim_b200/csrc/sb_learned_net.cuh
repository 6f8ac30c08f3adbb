// Inference of the whole proposal network (four 3x3 convolutions, 16 -> 32
// -> 32 -> 32 -> 16 channels, ReLU after the first three) in one kernel.
//
// The layer-by-layer path writes every activation tensor to global memory
// and reads it back with a halo in the next launch.  Here one CTA owns a
// column strip of the image and streams down a band of rows; each layer's
// output rows live in a four-row ring in shared memory, where the next
// layer's MMAs read them as K-major operands (the staging layout of the
// layer kernels), so activations never leave the SM.
//
// Geometry.  The tensor core works on 128-pixel rows.  A layer's output at
// pixel slot p needs its input at p-1 .. p+1, so the valid slots shrink by
// one on each side per layer after the first: 122 of the 128 slots of the
// last layer are valid, and strips advance by 122 pixels (slot p of strip s
// is pixel x = 122 s - 3 + p).  Rows: for the band [B, B+n) the layers
// compute rows B-3 .. B+n+2, B-2 .. B+n+1, B-1 .. B+n and B .. B+n-1; the
// features rows B-4 .. B+n+3 arrive by TMA.  Positions outside the image are
// stored as zeros, which is the zero padding of every layer.
//
// Schedule.  In round s layer L (0-based) computes its use u = s - 3L (row
// B-3+L+u), so a layer trails the one before it by two rows: the rows it
// reads were finished in an earlier round, and the four layers of a round
// are independent.  Warp roles:
//   warps 0-15 epilogue, one group of four warps per layer (TMEM lane =
//              pixel slot): ReLU, BF16, into the layer's ring (the last
//              layer: its four f32 outputs to global memory).  A row's
//              epilogue is a chain of dependent steps (TMEM load, convert,
//              stores, proxy fence, arrival) of about a microsecond, so the
//              four layers' epilogues run side by side;
//   warp 16    one thread issues the MMAs (tcgen05.mma, accumulators double
//              buffered per layer in TMEM);
//   warp 17    one thread issues the TMA loads of feature rows (6-row ring).
// Every hand-off is an mbarrier: feature row landed (TMA transaction bytes),
// feature slot free and accumulator ready (tcgen05.commit), epilogue done
// (128 arrivals: the accumulator buffer is free and the output row is in the
// ring).  Ring slots need no barrier of their own: layer L's use u rewrites
// the slot of its use u-4, whose last reader is layer L+1's use u-4, issued
// one round before layer L's use u; MMAs complete in issue order, so the
// completion that the epilogue waits for before writing use u implies it.
//
// The MMAs of a row are issued in the same order (dy, dx, K chunk) as the
// layer kernels', and the epilogue rounds the same way, so the output equals
// the layer-by-layer path bit for bit.  All waits are bounded; a wait that
// gives up sets the CTA's abort flag (the other roles leave their loops) and
// the caller's status word.
#pragma once

#include "sb_learned.cuh"

namespace sb {

constexpr int kNetEpiGroups = 4;                           // one epilogue warp group per layer
constexpr int kNetThreads = (4 * kNetEpiGroups + 2) * 32;  // + MMA warp + TMA warp
constexpr int kNetHalo = 3;                                // slots lost per side, layers 2-4
constexpr int kNetTileOut = kConvTileOut - 2 * kNetHalo;   // 122 valid output pixels per strip
constexpr int kNetFeatSlots = 6;
constexpr int kNetActSlots = 4;
constexpr uint32_t kNetFeatLbo = 2176;  // 130 pixels x 16 B rounded up to 128 B (TMA destination)

struct NetSmem {
  static constexpr int W1 = 0;                                 // 16 -> 32, 9 taps
  static constexpr int W2 = W1 + 9 * 32 * 16 * 2;              // 32 -> 32
  static constexpr int W3 = W2 + 9 * 32 * 32 * 2;              // 32 -> 32
  static constexpr int W4 = W3 + 9 * 32 * 32 * 2;              // 32 -> 16
  static constexpr int W_END = W4 + 9 * 16 * 32 * 2;
  static constexpr int FEAT_SLOT = 2 * (int)kNetFeatLbo;       // 16 channels
  static constexpr int FEAT = W_END;
  static constexpr int ACT_SLOT = 4 * (int)kRowLbo;            // 32 channels
  static constexpr int ACT_RING = kNetActSlots * ACT_SLOT;
  static constexpr int ACT = FEAT + kNetFeatSlots * FEAT_SLOT;
  static constexpr int BARS = ACT + 3 * ACT_RING;
  static constexpr int NBARS = 2 * kNetFeatSlots + 8 + 8 + 1;  // full, free, mma, epilogue, final
  static constexpr int BYTES = BARS + NBARS * 8 + 16;
  static constexpr uint32_t TMEM_COLS = 256;
  // accumulator of layer L, buffer j: 32 columns each for layers 0-2, 16 for layer 3
  __host__ __device__ static constexpr uint32_t acc_col(int L, int j) {
    return L < 3 ? (uint32_t)(L * 64 + j * 32) : (uint32_t)(192 + j * 16);
  }
};
static_assert(NetSmem::FEAT % 128 == 0 && NetSmem::FEAT_SLOT % 128 == 0,
              "TMA destinations are 128-byte aligned");
static_assert(NetSmem::BYTES <= 227 * 1024, "one CTA per SM");

struct NetArgs {
  const __nv_bfloat16* wpk[4];  // packed weights of the four layers (layer kernels' packing)
  float* flux;                // [batch][h][w][4]
  int batch, h, w;
  int rows_per_cta;
  int* status;                // set to 1 if a bounded wait gave up
};

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Bounded wait that also gives up once another role has set the abort flag.
__device__ __forceinline__ bool net_wait(uint64_t* bar, unsigned parity, volatile int* abort_flag) {
  const uint32_t a = smem_u32(bar);
  for (unsigned i = 0; i < kSpinLimit; ++i) {
    uint32_t done;
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if ((i & 255u) == 255u && *abort_flag) return false;
  }
  return false;
}

// 4-D tiled TMA load (x = the channel coordinate, a multiple of 8 BF16).
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int c0, int c1,
                                            int c2, int c3, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
      "[%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_u32(dst)),
      "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
      : "memory");
}

// One output row of a layer: nine taps (dy, dx) x CIN/16 K chunks of
// M = 128 pixels x N = COUT, in the layer kernels' order.  r0..r2: the
// staged input rows y-1, y, y+1; LBO: their channel-chunk stride.
template <int CIN, int COUT, uint32_t LBO>
__device__ __forceinline__ void net_issue(uint32_t tmem_d, uint32_t r0, uint32_t r1, uint32_t r2,
                                          uint32_t w_base) {
  constexpr int W_BLOCK = COUT * CIN * 2;
  constexpr uint32_t idesc = umma_idesc_bf16(128, COUT);
  const uint64_t bdesc0 = umma_desc(w_base, 128, (CIN / 8) * 128);
#pragma unroll
  for (int dy = 0; dy < 3; ++dy) {
    const uint64_t adesc0 = umma_desc(dy == 0 ? r0 : dy == 1 ? r1 : r2, LBO, 128);
#pragma unroll
    for (int dx = 0; dx < 3; ++dx) {
#pragma unroll
      for (int kk = 0; kk < CIN / 16; ++kk)
        umma_bf16(tmem_d, adesc0 + (uint64_t)((kk * 2 * LBO + dx * 16) >> 4),
                  bdesc0 + (uint64_t)(((dy * 3 + dx) * W_BLOCK + kk * 256) >> 4), idesc,
                  (dy | dx | kk) != 0);
    }
  }
}

__global__ void __launch_bounds__(kNetThreads, 1)
    net_forward_kernel(const __grid_constant__ CUtensorMap feat_map, const NetArgs a) {
  using S = NetSmem;
  extern __shared__ __align__(1024) unsigned char smem[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + S::BARS);
  uint64_t* feat_full = bars;
  uint64_t* feat_free = bars + kNetFeatSlots;
  uint64_t* mma_done = bars + 2 * kNetFeatSlots;  // [layer][buffer]
  uint64_t* epi_done = mma_done + 8;              // [layer][buffer]
  uint64_t* fin = epi_done + 8;
  uint32_t* tslot = reinterpret_cast<uint32_t*>(fin + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tslot + 1);

  const int tid = threadIdx.x, warp = tid >> 5;
  const int x0 = blockIdx.x * kNetTileOut - kNetHalo;  // pixel of slot 0
  const int B = blockIdx.y * a.rows_per_cta;
  const int n = min(a.rows_per_cta, a.h - B);
  const int img = blockIdx.z;

  {
    constexpr int kOff[4] = {S::W1, S::W2, S::W3, S::W4};
    constexpr int kEnd[4] = {S::W2, S::W3, S::W4, S::W_END};
#pragma unroll
    for (int L = 0; L < 4; ++L) {
      const uint4* src = reinterpret_cast<const uint4*>(a.wpk[L]);
      uint4* dst = reinterpret_cast<uint4*>(smem + kOff[L]);
      for (int i = tid; i < (kEnd[L] - kOff[L]) / 16; i += kNetThreads) dst[i] = src[i];
    }
  }
  // staged pixels 0 and 129 of the activation rings feed only invalid slots;
  // zero them so that they hold no stale bits
  for (int i = tid; i < 3 * kNetActSlots * 4 * 2; i += kNetThreads) {
    const int q = i >> 1;  // (ring, slot) * 4 + channel chunk
    *reinterpret_cast<uint4*>(smem + S::ACT + (q >> 2) * S::ACT_SLOT + (q & 3) * kRowLbo +
                              ((i & 1) ? 129 * 16 : 0)) = make_uint4(0u, 0u, 0u, 0u);
  }
  if (tid == 0) {
    for (int k = 0; k < kNetFeatSlots; ++k) {
      mbar_init(&feat_full[k], 1);
      mbar_init(&feat_free[k], 1);
    }
    for (int k = 0; k < 8; ++k) {
      mbar_init(&mma_done[k], 1);
      mbar_init(&epi_done[k], 128);
    }
    mbar_init(fin, 1);
    *abort_flag = 0;
  }
  if (warp == 0) tmem_alloc(tslot, S::TMEM_COLS);
  fence_async_smem();  // weights and zeros (generic stores) before the tensor core reads them
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  const uint32_t sbase = smem_u32(smem);
  const int rounds = n + 9;

  if (warp == 4 * kNetEpiGroups + 1) {
    // ---- feature rows B-4 .. B+n+3 by TMA (relative row f, slot f % 6)
    if ((tid & 31) == 0) {
      prefetch_tmap(&feat_map);
      bool ok = true;
      int f = 0;
      for (; f < n + 8; ++f) {
        const int slot = f % kNetFeatSlots;
        if (f >= kNetFeatSlots &&
            !net_wait(&feat_free[slot], (unsigned)((f / kNetFeatSlots - 1) & 1), abort_flag)) {
          ok = false;
          break;
        }
        unsigned char* dst = smem + S::FEAT + slot * S::FEAT_SLOT;
        mbar_expect_tx(&feat_full[slot], 2u * kRowPixels * 16u);
        tma_load_4d(dst, &feat_map, 0, x0 - 1, B - 4 + f, img, &feat_full[slot]);
        tma_load_4d(dst + kNetFeatLbo, &feat_map, 8, x0 - 1, B - 4 + f, img, &feat_full[slot]);
      }
      if (!ok) {
        *abort_flag = 1;
        if (a.status) atomicExch(a.status, 1);
      }
      // copies still in flight land before the CTA ends
      for (int g = f > kNetFeatSlots ? f - kNetFeatSlots : 0; g < f; ++g)
        mbar_wait(&feat_full[g % kNetFeatSlots], (unsigned)((g / kNetFeatSlots) & 1));
    }
  } else if (warp == 4 * kNetEpiGroups) {
    // ---- MMA issue
    if ((tid & 31) == 0) {
      bool ok = true;
      for (int s = 0; s < rounds && ok; ++s) {
        for (int L = 0; L < 4; ++L) {
          const int u = s - 3 * L;
          if (u < 0 || u > n + 5 - 2 * L) continue;
          if (L == 0) {
            for (int f = (u == 0 ? 0 : u + 2); f <= u + 2 && ok; ++f)
              ok = net_wait(&feat_full[f % kNetFeatSlots], (unsigned)((f / kNetFeatSlots) & 1),
                            abort_flag);
          } else {
            const int v = u + 2;  // the newest input row is use v of layer L-1
            ok = net_wait(&epi_done[(L - 1) * 2 + (v & 1)], (unsigned)((v >> 1) & 1), abort_flag);
          }
          if (ok && u >= 2)  // accumulator buffer: use u-2 drained
            ok = net_wait(&epi_done[L * 2 + (u & 1)], (unsigned)(((u - 2) >> 1) & 1), abort_flag);
          if (!ok) break;
          tc_fence_after();
          const uint32_t d = tmem + S::acc_col(L, u & 1);
          if (L == 0) {
            auto fs = [&](int f) {
              return sbase + S::FEAT + (uint32_t)((f % kNetFeatSlots) * S::FEAT_SLOT);
            };
            net_issue<16, 32, kNetFeatLbo>(d, fs(u), fs(u + 1), fs(u + 2), sbase + S::W1);
          } else {
            const uint32_t ring = sbase + S::ACT + (uint32_t)((L - 1) * S::ACT_RING);
            auto as = [&](int v) { return ring + (uint32_t)((v % kNetActSlots) * S::ACT_SLOT); };
            if (L == 1)
              net_issue<32, 32, kRowLbo>(d, as(u), as(u + 1), as(u + 2), sbase + S::W2);
            else if (L == 2)
              net_issue<32, 32, kRowLbo>(d, as(u), as(u + 1), as(u + 2), sbase + S::W3);
            else
              net_issue<32, 16, kRowLbo>(d, as(u), as(u + 1), as(u + 2), sbase + S::W4);
          }
          umma_commit(&mma_done[L * 2 + (u & 1)]);
          if (L == 0) umma_commit(&feat_free[u % kNetFeatSlots]);  // feature row u is done
        }
      }
      if (!ok) {
        *abort_flag = 1;
        if (a.status) atomicExch(a.status, 1);
      }
      umma_commit(fin);  // completes once every MMA issued above has
      mbar_wait(fin, 0);
    }
  } else {
    // ---- epilogue: group g = warp / 4 owns the layers L with L % groups == g;
    // pixel slot p = TMEM lane (warp w reads lanes 32 (w % 4) ..)
    const int g = warp >> 2;
    const int p = ((warp & 3) << 5) | (tid & 31);
    const int x = x0 + p;
    const uint32_t lane_addr = tmem + ((uint32_t)((warp & 3) * 32) << 16);
    bool ok = true;
    for (int s = 0; s < rounds && ok; ++s) {
      for (int L = g; L < 4; L += kNetEpiGroups) {
        const int u = s - 3 * L;
        if (u < 0 || u > n + 5 - 2 * L) continue;
        if (!net_wait(&mma_done[L * 2 + (u & 1)], (unsigned)((u >> 1) & 1), abort_flag)) {
          ok = false;
          break;
        }
        tc_fence_after();
        const int r = B - 3 + L + u;
        const uint32_t taddr = lane_addr + S::acc_col(L, u & 1);
        if (L < 3) {
          float d[32];
          tmem_ld32(taddr, d);
          tc_fence_before();
          const bool inside = x >= 0 && x < a.w && r >= 0 && r < a.h;
          unsigned char* dst = smem + S::ACT + L * S::ACT_RING + (u % kNetActSlots) * S::ACT_SLOT +
                               (p + 1) * 16;
#pragma unroll
          for (int c8 = 0; c8 < 4; ++c8) {
            __align__(16) __nv_bfloat162 ob[4];
#pragma unroll
            for (int j = 0; j < 4; ++j)
              ob[j] = inside ? __floats2bfloat162_rn(fmaxf(d[c8 * 8 + 2 * j], 0.f),
                                                     fmaxf(d[c8 * 8 + 2 * j + 1], 0.f))
                             : __floats2bfloat162_rn(0.f, 0.f);
            *reinterpret_cast<uint4*>(dst + c8 * kRowLbo) = *reinterpret_cast<const uint4*>(ob);
          }
          fence_async_smem();  // the next layer's MMAs read this row
        } else {
          float d[16];
          tmem_ld16(taddr, d);
          tc_fence_before();
          if (p >= kNetHalo && p < kNetHalo + kNetTileOut && x < a.w)
            *reinterpret_cast<float4*>(a.flux + (((size_t)img * a.h + r) * a.w + x) * 4) =
                make_float4(d[0], d[1], d[2], d[3]);
        }
        mbar_arrive(&epi_done[L * 2 + (u & 1)]);
      }
    }
    if (!ok) {
      *abort_flag = 1;
      if (a.status) atomicExch(a.status, 1);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_free(tmem, S::TMEM_COLS);
  }
}

}  // namespace sb
