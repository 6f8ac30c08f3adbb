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
// is pixel x = 122 s - 3 + p).  Rows: for the band [B, B+n) layer L (0-3)
// reads input rows B-4+L .. B+n+3-L (input i = row B-4+L+i) and produces the
// rows B-3+L .. B+n+2-L; the feature rows arrive by TMA.  Positions outside
// the image are stored as zeros, which is the zero padding of every layer.
//
// Rotating accumulators.  A tcgen05.mma instruction costs tens of cycles
// whatever its size (measured: ~50 ns per M128 x N32 x K16 MMA issued from
// one thread, most of it not tensor-pipe time), so small MMAs leave the
// tensor core idle.  Each input row is therefore consumed once, by
// 3 x CIN/16 MMAs of N = 3 x COUT: input i feeds the outputs i, i+1, i+2
// (numbered from the layer's first input) through the kernel rows dy = 2,
// 1, 0, into three accumulators side by side in TMEM.  Output j lives in
// slot j % 3, and the staged weights per dx are the five blocks
// W(2) W(1) W(0) W(2) W(1), so the operand for input i is the three
// consecutive blocks from (3 - i % 3) % 3.  Output j is complete after input
// j; its epilogue reads the slot and clears it (tcgen05.st of zeros) before
// input j+1 adds to it as output j+3.  Every output thus receives its inputs
// j-2, j-1, j in the (dy, dx, K chunk) order of the layer kernels, starting
// from zero, and the epilogue rounds the same way, so the fluxes equal the
// layer-by-layer path's.  Outputs 0 and 1 only collect partial sums and are
// dropped.
//
// Roles.
//   warps 0-15  epilogue, one group of four warps per layer (TMEM lane =
//               pixel slot): ReLU, BF16, into the layer's ring (the last
//               layer: its four f32 outputs to global memory);
//   warps 16-19 one thread per layer issues that layer's MMAs, input after
//               input: input i of layer L is output i+2 of layer L-1, and
//               the accumulator slot it starts held output i-1, so it waits
//               for those two epilogues.  Issue from one thread is serial
//               (about 60 ns per MMA and 70 ns per barrier wait, measured),
//               so the four layers issue side by side;
//   warp 20     one thread issues the TMA loads of feature rows (6-row ring).
// Hand-offs are mbarriers: feature row landed (TMA transaction bytes); the
// MMAs of an input done and feature slot free (tcgen05.commit); an output's
// accumulator read and cleared, then its row in the ring (128 arrivals each:
// the issuer of the same layer needs only the first).  A phase-parity wait only tells completion
// #k from #k-1, so each waiter observes a barrier's completions in order, and
// the barriers of a kind rotate over four per layer: no producer gets two
// completions ahead of a waiter (layer L-1 can finish at most three outputs
// beyond the one layer L waits for).  Commits track only their own thread's
// MMAs, so a ring slot is guarded explicitly: the epilogue that writes ring
// entry j-2 (replacing entry j-6) first waits for layer L+1's input j-6.
// The protocol (ordering, slot reuse, parity aliasing) was checked by a
// simulation over band heights 1-40 and random interleavings.  All waits are
// bounded; a wait that gives up sets the CTA's abort flag (the other roles
// leave their loops) and the caller's status word.
#pragma once

#include "sb_learned.cuh"

namespace sb {

constexpr int kNetEpiGroups = 4;                           // one epilogue warp group per layer
constexpr int kNetThreads = (4 * kNetEpiGroups + 4 + 1) * 32;  // + 4 MMA warps + TMA warp
constexpr int kNetBars = 4;  // mbarriers per layer and kind, used in turn (see the protocol note)
constexpr int kNetHalo = 3;                                // slots lost per side, layers 2-4
constexpr int kNetTileOut = kConvTileOut - 2 * kNetHalo;   // 122 valid output pixels per strip
constexpr int kNetFeatSlots = 6;
constexpr int kNetActSlots = 4;
constexpr uint32_t kNetFeatLbo = 2176;  // 130 pixels x 16 B rounded up to 128 B (TMA destination)

__host__ __device__ constexpr int net_cin(int L) { return L == 0 ? 16 : 32; }
__host__ __device__ constexpr int net_cout(int L) { return L == 3 ? 16 : 32; }

struct NetSmem {
  // weights per layer: 3 dx x 5 staged blocks of COUT x CIN
  static constexpr int W1 = 0;
  static constexpr int W2 = W1 + 15 * 32 * 16 * 2;
  static constexpr int W3 = W2 + 15 * 32 * 32 * 2;
  static constexpr int W4 = W3 + 15 * 32 * 32 * 2;
  static constexpr int W_END = W4 + 15 * 16 * 32 * 2;
  static constexpr int FEAT_SLOT = 2 * (int)kNetFeatLbo;       // 16 channels
  static constexpr int FEAT = W_END;
  static constexpr int ACT_SLOT = 4 * (int)kRowLbo;            // 32 channels
  static constexpr int ACT_RING = kNetActSlots * ACT_SLOT;
  static constexpr int ACT = FEAT + kNetFeatSlots * FEAT_SLOT;
  static constexpr int BARS = ACT + 3 * ACT_RING;
  static constexpr int NBARS = 2 * kNetFeatSlots + 3 * 4 * kNetBars + 4;  // + final per layer
  static constexpr int BYTES = BARS + NBARS * 8 + 16;
  static constexpr uint32_t TMEM_COLS = 512;
  // first accumulator column of layer L (three slots of COUT columns)
  __host__ __device__ static constexpr uint32_t acc_col(int L) { return (uint32_t)(L * 96); }
  __host__ __device__ static constexpr int w_off(int L) {
    return L == 0 ? W1 : L == 1 ? W2 : L == 2 ? W3 : W4;
  }
};
static_assert(NetSmem::FEAT % 128 == 0 && NetSmem::FEAT_SLOT % 128 == 0,
              "TMA destinations are 128-byte aligned");
static_assert(NetSmem::BYTES <= 227 * 1024, "one CTA per SM");
static_assert(NetSmem::acc_col(3) + 3 * 16 <= NetSmem::TMEM_COLS, "accumulators fit in TMEM");

struct NetArgs {
  const __nv_bfloat16* wpk[4];  // packed weights of the four layers (layer kernels' packing)
  float* flux;                  // [batch][h][w][4]
  int batch, h, w;
  int rows_per_cta;
  int* status;                  // set to 1 if a bounded wait gave up
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

// The MMAs of one input row of a layer: per (dx, K chunk) one M = 128
// pixels x N = 3 COUT MMA into the layer's three accumulator slots.  row:
// the staged input row, LBO its channel-chunk stride; first: the staged
// weight block (of five per dx) that feeds slot 0.
template <int CIN, int COUT, uint32_t LBO>
__device__ __forceinline__ void net_issue_input(uint32_t tmem_d, uint32_t row, uint32_t w_base,
                                                int first) {
  constexpr int W_BLOCK = COUT * CIN * 2;
  constexpr uint32_t idesc = umma_idesc_bf16(128, 3 * COUT);
  const uint64_t adesc0 = umma_desc(row, LBO, 128);
  const uint64_t bdesc0 = umma_desc(w_base, 128, (CIN / 8) * 128);
#pragma unroll
  for (int dx = 0; dx < 3; ++dx)
#pragma unroll
    for (int kk = 0; kk < CIN / 16; ++kk)
      umma_bf16(tmem_d, adesc0 + (uint64_t)((kk * 2 * LBO + dx * 16) >> 4),
                bdesc0 + (uint64_t)(((dx * 5 + first) * W_BLOCK + kk * 256) >> 4), idesc, 1);
}

__global__ void __launch_bounds__(kNetThreads, 1)
    net_forward_kernel(const __grid_constant__ CUtensorMap feat_map, const NetArgs a) {
  using S = NetSmem;
  extern __shared__ __align__(1024) unsigned char smem[];
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + S::BARS);
  uint64_t* feat_full = bars;
  uint64_t* feat_free = bars + kNetFeatSlots;
  uint64_t* mma_done = bars + 2 * kNetFeatSlots;  // [layer][input % kNetBars]
  uint64_t* epi_done = mma_done + 4 * kNetBars;   // [layer][output % kNetBars]
  uint64_t* acc_free = epi_done + 4 * kNetBars;   // [layer][output % kNetBars]
  uint64_t* fin = acc_free + 4 * kNetBars;        // [layer]
  uint32_t* tslot = reinterpret_cast<uint32_t*>(fin + 4);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tslot + 1);

  const int tid = threadIdx.x, warp = tid >> 5;
  const int x0 = blockIdx.x * kNetTileOut - kNetHalo;  // pixel of slot 0
  const int B = blockIdx.y * a.rows_per_cta;
  const int n = min(a.rows_per_cta, a.h - B);
  const int img = blockIdx.z;

  // weights: per layer and dx the blocks of dy = 2, 1, 0, 2, 1 (the packed
  // input holds block dy * 3 + dx)
#pragma unroll
  for (int L = 0; L < 4; ++L) {
    constexpr int kChunks[4] = {32 * 16 * 2 / 16, 32 * 32 * 2 / 16, 32 * 32 * 2 / 16,
                                16 * 32 * 2 / 16};
    const int chunks = kChunks[L];
    const uint4* src = reinterpret_cast<const uint4*>(a.wpk[L]);
    uint4* dst = reinterpret_cast<uint4*>(smem + S::w_off(L));
    for (int i = tid; i < 15 * chunks; i += kNetThreads) {
      const int blk = i / chunks, c = i - blk * chunks;
      const int dx = blk / 5, jj = blk - dx * 5;
      const int dy = (jj == 0 || jj == 3) ? 2 : (jj == 1 || jj == 4) ? 1 : 0;
      dst[i] = src[(dy * 3 + dx) * chunks + c];
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
    for (int k = 0; k < 4 * kNetBars; ++k) {
      mbar_init(&mma_done[k], 1);
      mbar_init(&epi_done[k], 128);
      mbar_init(&acc_free[k], 128);
    }
    for (int k = 0; k < 4; ++k) mbar_init(&fin[k], 1);
    *abort_flag = 0;
  }
  if (warp == 0) tmem_alloc(tslot, S::TMEM_COLS);
  fence_async_smem();  // weights and zeros (generic stores) before the tensor core reads them
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  const uint32_t sbase = smem_u32(smem);
  // epilogue warps: every layer's three accumulator slots start at zero
  if (warp < 4 * kNetEpiGroups) {
    const int L = warp >> 2;
    const uint32_t lanes = tmem + ((uint32_t)((warp & 3) * 32) << 16) + S::acc_col(L);
    if (L < 3)
      for (int sl = 0; sl < 3; ++sl) tmem_zero<32>(lanes + (uint32_t)(sl * 32));
    else
      for (int sl = 0; sl < 3; ++sl) tmem_zero<16>(lanes + (uint32_t)(sl * 16));
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();

  if (warp == 4 * kNetEpiGroups + 4) {
    // ---- feature rows B-4 .. B+n+3 by TMA (input i of layer 0, slot i % 6)
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
  } else if (warp >= 4 * kNetEpiGroups) {
    // ---- MMA issue: warp 16 + L issues layer L's inputs in order
    const int L = warp - 4 * kNetEpiGroups;
    if ((tid & 31) == 0) {
      bool ok = true;
      const int inputs = n + 8 - 2 * L;
      for (int i = 0; i < inputs && ok; ++i) {
        if (L == 0) {  // feature row i landed
          ok = net_wait(&feat_full[i % kNetFeatSlots], (unsigned)((i / kNetFeatSlots) & 1),
                        abort_flag);
        } else {  // output i + 2 of layer L-1 in the ring (outputs 0-2 first, in order)
          for (int v = i == 0 ? 0 : i + 2; v <= i + 2 && ok; ++v)
            ok = net_wait(&epi_done[(L - 1) * kNetBars + (v % kNetBars)],
                          (unsigned)((v / kNetBars) & 1), abort_flag);
        }
        if (ok && i >= 1)  // output i-1 read and cleared: the slot output i+2 starts
          ok = net_wait(&acc_free[L * kNetBars + ((i - 1) % kNetBars)],
                        (unsigned)(((i - 1) / kNetBars) & 1), abort_flag);
        if (!ok) break;
        tc_fence_after();
        const uint32_t d = tmem + S::acc_col(L);
        const int first = (3 - i % 3) % 3;
        if (L == 0) {
          net_issue_input<16, 32, kNetFeatLbo>(
              d, sbase + S::FEAT + (uint32_t)((i % kNetFeatSlots) * S::FEAT_SLOT), sbase + S::W1,
              first);
        } else {
          // input i of layer L = output i + 2 of layer L-1 = ring entry i
          const uint32_t row = sbase + S::ACT + (uint32_t)((L - 1) * S::ACT_RING) +
                               (uint32_t)((i % kNetActSlots) * S::ACT_SLOT);
          if (L == 3)
            net_issue_input<32, 16, kRowLbo>(d, row, sbase + S::W4, first);
          else
            net_issue_input<32, 32, kRowLbo>(d, row, sbase + (L == 1 ? S::W2 : S::W3), first);
        }
        umma_commit(&mma_done[L * kNetBars + (i % kNetBars)]);
        if (L == 0) umma_commit(&feat_free[i % kNetFeatSlots]);  // feature row consumed
      }
      if (!ok) {
        *abort_flag = 1;
        if (a.status) atomicExch(a.status, 1);
      }
      umma_commit(&fin[L]);  // completes once every MMA this thread issued has
      mbar_wait(&fin[L], 0);
    }
  } else {
    // ---- epilogue: warp group L = warp / 4 drains layer L; pixel slot p =
    // TMEM lane (warp w reads lanes 32 (w % 4) ..)
    const int L = warp >> 2;
    const int p = ((warp & 3) << 5) | (tid & 31);
    const int x = x0 + p;
    const uint32_t lanes = tmem + ((uint32_t)((warp & 3) * 32) << 16) + S::acc_col(L);
    const int outputs = n + 8 - 2 * L;
    bool ok = true;
    for (int j = 0; j < outputs; ++j) {
      if (!net_wait(&mma_done[L * kNetBars + (j % kNetBars)], (unsigned)((j / kNetBars) & 1),
                    abort_flag)) {
        ok = false;
        break;
      }
      tc_fence_after();
      const int r = B - 5 + L + j;  // output j of layer L
      if (L < 3) {
        const uint32_t taddr = lanes + (uint32_t)((j % 3) * 32);
        float d[32];
        tmem_ld32(taddr, d);
        tmem_zero<32>(taddr);
        tc_fence_before();
        mbar_arrive(&acc_free[L * kNetBars + (j % kNetBars)]);
        // ring entry j-2 replaces entry j-6: layer L+1's input j-6 must be done
        if (j >= 6 && !net_wait(&mma_done[(L + 1) * kNetBars + ((j - 6) % kNetBars)],
                                (unsigned)(((j - 6) / kNetBars) & 1), abort_flag)) {
          ok = false;
          break;
        }
        if (j >= 2) {
          const bool inside = x >= 0 && x < a.w && r >= 0 && r < a.h;
          unsigned char* dst = smem + S::ACT + L * S::ACT_RING +
                               ((j - 2) % kNetActSlots) * S::ACT_SLOT + (p + 1) * 16;
#pragma unroll
          for (int c8 = 0; c8 < 4; ++c8) {
            __align__(16) __nv_bfloat162 ob[4];
#pragma unroll
            for (int k = 0; k < 4; ++k)
              ob[k] = inside ? __floats2bfloat162_rn(fmaxf(d[c8 * 8 + 2 * k], 0.f),
                                                     fmaxf(d[c8 * 8 + 2 * k + 1], 0.f))
                             : __floats2bfloat162_rn(0.f, 0.f);
            *reinterpret_cast<uint4*>(dst + c8 * kRowLbo) = *reinterpret_cast<const uint4*>(ob);
          }
          fence_async_smem();  // the next layer's MMAs read this row
        }
      } else {
        const uint32_t taddr = lanes + (uint32_t)((j % 3) * 16);
        float d[16];
        tmem_ld16(taddr, d);
        tmem_zero<16>(taddr);
        tc_fence_before();
        mbar_arrive(&acc_free[L * kNetBars + (j % kNetBars)]);
        if (j >= 2 && p >= kNetHalo && p < kNetHalo + kNetTileOut && x < a.w)
          *reinterpret_cast<float4*>(a.flux + (((size_t)img * a.h + r) * a.w + x) * 4) =
              make_float4(d[0], d[1], d[2], d[3]);
      }
      if (L < 3) mbar_arrive(&epi_done[L * kNetBars + (j % kNetBars)]);
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
