// Learned repose proposal: a 4-layer 3x3 convolution net (4 -> 32 -> 32 ->
// 32 -> 4 channels, ReLU between, no bias, BF16 operands, FP32 accumulate)
// proposes per-edge outflows of a height field; they are applied in flux
// form (every transfer leaves one cell and enters its neighbour, in whole
// height quanta in the fixed-point state), and plain relaxation sweeps then
// finish to the repose tolerance.  The reference has no counterpart: its
// repose relaxation is the plain sweep (slope_model.py:273-343) alone.
//
// Convolutions are implicit GEMMs on the 5th-generation tensor cores
// (tcgen05.mma, kind::f16, operands in shared memory, accumulator in TMEM):
//
//   forward / data gradient: per output row of a 128-pixel tile, the nine
//     taps (dy, dx) are nine K-major operands (M = 128 pixels, K = input
//     channels) read straight out of the staged input rows -- a column
//     offset is a 16-byte start offset in the pixel-major staging layout --
//     against the tap's weights (N = output channels), accumulated in one
//     TMEM tile that is the output row.  The data gradient is the same kernel
//     run with the flipped, transposed weights and the ReLU mask of the
//     layer's input.
//   weight gradient: per input row, A = the row shifted by dx (M = (dx, ci),
//     K = 128 pixels) times B = output-gradient rows (N = co), accumulated in
//     TMEM over the CTA's band for the three row offsets; per-CTA partials
//     are summed in a fixed order by a second kernel.
//
// Operands use the canonical no-swizzle K-major layout: 8 x 16-byte core
// matrices, element (r, k) at ((r/8)*(K/8) + k/8)*128 + (r%8)*16 + (k%8)*2.
#pragma once

#include <cuda_bf16.h>

#include "sb_common.cuh"

namespace sb {

constexpr int kConvThreads = 128;   // 4 warps: TMEM lanes 0..127 = tile pixels
// Forward kernel: the four pixel warps plus one warp whose lane 0 issues the
// MMAs, so that a row's MMA issue overlaps the pixel warps' epilogue.
constexpr int kConvFwdThreads = 160;
constexpr int kConvTileOut = 128;   // output pixels per CTA row tile

// ---------------------------------------------------------------- tcgen05
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version of sm_100; no swizzle, base offset 0
  return d;
}

// kind::f16 instruction descriptor: D f32, A/B bf16, both K-major.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc,
                                          int accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Warp 0 allocates ncols TMEM columns; the base address lands in *slot.
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_u32(slot)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t base, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(ncols)
               : "memory");
}

// 16 consecutive f32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,"
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// 32 consecutive f32 columns of this thread's TMEM lane (one load, one wait).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,"
      "%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
        "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
        "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ uint32_t core_off(int r, int k, int kdim) {
  return (uint32_t)(((r >> 3) * (kdim >> 3) + (k >> 3)) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

struct ConvArgs {
  const __nv_bfloat16* in;      // [batch][h][w][cin]
  void* out;                    // bf16 [batch][h][w][cout], or f32 [batch][h][w][out_f32]
  const __nv_bfloat16* wpk;     // 3 row offsets x canonical B (n = dx*cout + co, k = ci)
  const __nv_bfloat16* mask;    // optional [batch][h][w][cout]: out *= (mask > 0)
  int batch, h, w;
  int rows_per_cta;
  int relu;
  int out_f32;                  // 0: bf16, all channels; k (multiple of 4): f32, first k channels
  int* status;                  // set to 1 if a bounded wait gave up
};

// Input rows are staged pixel-major: 130 pixels (x0-1 .. x0+128) of 16 bytes
// (8 channels) per K chunk, chunks kRowLbo bytes apart.  In the canonical
// K-major layout that is SBO = 128 B (8 consecutive pixels per core matrix,
// core matrices contiguous) and LBO = kRowLbo, so the operand for column
// offset dx is the same rows starting dx * 16 bytes later: no copies.
constexpr int kRowPixels = 130;
constexpr uint32_t kRowLbo = kRowPixels * 16;

template <int CIN, int COUT>
struct ConvSmem {
  static constexpr int W_BLOCK = COUT * CIN * 2;         // one tap's weights (canonical B)
  static constexpr int W_BYTES = 9 * W_BLOCK;
  static constexpr int ROW_BYTES = (CIN / 8) * kRowLbo;  // one staged input row
  static constexpr int SLOTS = 4;                        // rows y..y+2 in use + one in flight
  static constexpr int BYTES = W_BYTES + SLOTS * ROW_BYTES + 64;
  static constexpr uint32_t TMEM_COLS = 32;              // N = COUT <= 32 f32 columns
};

// Starts the asynchronous copy of input row r (pixels x0-1 .. x0+128) into
// a ring slot; 16-byte cp.async chunks, zero-filled outside the image.
template <int CIN, int NT = kConvThreads>
__device__ __forceinline__ void conv_row_async(const __nv_bfloat16* __restrict__ in, int b, int h,
                                               int w, int r, int x0, unsigned char* slot) {
  for (int j = threadIdx.x; j < kRowPixels; j += NT) {
    const int x = x0 - 1 + j;
    const bool ok = r >= 0 && r < h && x >= 0 && x < w;
    const __nv_bfloat16* src = in + (((size_t)b * h + (ok ? r : 0)) * w + (ok ? x : 0)) * CIN;
    const unsigned bytes = ok ? 16u : 0u;
#pragma unroll
    for (int kb = 0; kb < CIN / 8; ++kb)
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(
                       smem_u32(slot + kb * kRowLbo + j * 16)),
                   "l"(src + kb * 8), "r"(bytes)
                   : "memory");
  }
  asm volatile("cp.async.commit_group;" ::: "memory");
}

__device__ __forceinline__ void conv_row_wait() {
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  fence_async_smem();  // the rows are read by the tensor core (async proxy)
}

// Waits until at most `pending` (0..2) of this thread's most recent row copies
// are still in flight.
__device__ __forceinline__ void conv_row_wait_pending(int pending) {
  if (pending >= 2)
    asm volatile("cp.async.wait_group 2;" ::: "memory");
  else if (pending == 1)
    asm volatile("cp.async.wait_group 1;" ::: "memory");
  else
    asm volatile("cp.async.wait_group 0;" ::: "memory");
  fence_async_smem();
}

// D[pixel, co] for output row y: nine taps (dy, dx), each M = 128 pixels x
// K = CIN against the tap's weights (N = COUT), accumulated in TMEM.
template <int CIN, int COUT>
__device__ __forceinline__ void conv_issue_row(uint32_t tmem, uint32_t ring_base,
                                               uint32_t w_base, int y, uint32_t idesc) {
  using S = ConvSmem<CIN, COUT>;
  // descriptors are built once per row; a tap's operand is the same descriptor
  // with a 16-byte-multiple start offset added to its address field (bits
  // 0-13 hold addr >> 4; shared-memory offsets stay below 2^18, so no carry)
  const uint64_t bdesc0 = umma_desc(w_base, 128, (CIN / 8) * 128);
#pragma unroll
  for (int dy = 0; dy < 3; ++dy) {
    const uint32_t slot = ring_base + ((y - 1 + dy + S::SLOTS) % S::SLOTS) * S::ROW_BYTES;
    const uint64_t adesc0 = umma_desc(slot, kRowLbo, 128);
#pragma unroll
    for (int dx = 0; dx < 3; ++dx) {
#pragma unroll
      for (int kk = 0; kk < CIN / 16; ++kk)
        umma_bf16(tmem, adesc0 + (uint64_t)((kk * 2 * kRowLbo + dx * 16) >> 4),
                  bdesc0 + (uint64_t)(((dy * 3 + dx) * S::W_BLOCK + kk * 256) >> 4), idesc,
                  (dy | dx | kk) != 0);
    }
  }
}

// Per CTA: one 128-pixel tile of rows [y0, y1).  Row y+1's MMAs are issued as
// soon as row y's accumulator has been read, so they run while row y's
// epilogue converts and stores; input rows are fetched by cp.async into a
// ring of SLOTS rows, SLOTS - 3 rows ahead of the rows the next MMA batch
// reads.  (Six slots measured slower than four: the extra 16 KB per CTA of
// the 32-channel layers cost a CTA per SM, and the per-row time is set by the
// tensor core's shared-memory operand reads -- 40 wavefronts per
// M128 x N32 x K16 MMA -- not by the copies.)
template <int CIN, int COUT>
__global__ void __launch_bounds__(kConvFwdThreads) conv3x3_tc_kernel(const ConvArgs a) {
  using S = ConvSmem<CIN, COUT>;
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char* wsm = smem;
  unsigned char* ring = smem + S::W_BYTES;
  uint64_t* bar = reinterpret_cast<uint64_t*>(ring + S::SLOTS * S::ROW_BYTES);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 1);

  const int tid = threadIdx.x, warp = tid >> 5;
  const int x0 = blockIdx.x * kConvTileOut;
  const int y0 = blockIdx.y * a.rows_per_cta;
  const int y1 = min(y0 + a.rows_per_cta, a.h);
  const int b = blockIdx.z;
  auto slot = [&](int r) { return ring + ((r + S::SLOTS) % S::SLOTS) * S::ROW_BYTES; };

  // weights -> shared memory (already in canonical layout)
  {
    const uint4* src = reinterpret_cast<const uint4*>(a.wpk);
    uint4* dst = reinterpret_cast<uint4*>(wsm);
    for (int i = tid; i < S::W_BYTES / 16; i += kConvFwdThreads) dst[i] = src[i];
  }
  if (tid == 0) mbar_init(bar, 1);
  if (warp == 0) tmem_alloc(tslot, S::TMEM_COLS);
  conv_row_async<CIN, kConvFwdThreads>(a.in, b, a.h, a.w, y0 - 1, x0, slot(y0 - 1));
  conv_row_async<CIN, kConvFwdThreads>(a.in, b, a.h, a.w, y0, x0, slot(y0));
  conv_row_async<CIN, kConvFwdThreads>(a.in, b, a.h, a.w, y0 + 1, x0, slot(y0 + 1));
  conv_row_wait();
  fence_async_smem();  // the weights (generic stores) too
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  const uint32_t idesc = umma_idesc_bf16(128, COUT);
  const uint32_t w_base = smem_u32(wsm), ring_base = smem_u32(ring);
  const uint32_t lane_addr = tmem + ((uint32_t)((warp & 3) * 32) << 16);
  const bool issuer = tid == 4 * 32;  // lane 0 of warp 4
  const bool pixel = warp < 4;         // the epilogue warps (TMEM lanes 0..127)
  unsigned phase = 0;
  bool ok = true;
  int issued = y0 + 1;  // last input row whose copy has been started
  if (y0 < y1) {
    if (issuer) {
      conv_issue_row<CIN, COUT>(tmem, ring_base, w_base, y0, idesc);
      umma_commit(bar);
    }
    // rows up to y1 are read (the last MMA batch, row y1-1, reads y1)
    for (int r = y0 + 2; r <= y0 + S::SLOTS - 2 && r <= y1; ++r) {
      conv_row_async<CIN, kConvFwdThreads>(a.in, b, a.h, a.w, r, x0, slot(r));
      issued = r;
    }
  }

  for (int y = y0; y < y1; ++y) {
    float d[COUT];  // this thread's pixel of the output row
    if (pixel) {
      ok = mbar_wait(bar, phase) && ok;
      tc_fence_after();
      if constexpr (COUT == 32)
        tmem_ld32(lane_addr, d);
      else
        tmem_ld16(lane_addr, d);
    }
    phase ^= 1;
    tc_fence_before();
    if (y + 1 < y1) conv_row_wait_pending(issued - (y + 2));  // row y+2 has landed
    __syncthreads();                                         // everyone has read the accumulator
    if (y + 1 < y1) {
      if (issuer) {
        tc_fence_after();
        conv_issue_row<CIN, COUT>(tmem, ring_base, w_base, y + 1, idesc);
        umma_commit(bar);
      }
      // the slot of row y-1 (= row y-1+SLOTS) is free: row y's MMAs have completed
      if (issued + 1 <= y1 && issued + 1 <= y + S::SLOTS - 1) {
        conv_row_async<CIN, kConvFwdThreads>(a.in, b, a.h, a.w, issued + 1, x0, slot(issued + 1));
        ++issued;
      }
    }
    const int xo = x0 + tid;
    if (pixel && xo < a.w) {
      const size_t pix = ((size_t)b * a.h + y) * a.w + xo;
#pragma unroll
      for (int c8 = 0; c8 < COUT; c8 += 8) {
        float o[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) o[j] = a.relu ? fmaxf(d[c8 + j], 0.f) : d[c8 + j];
        if (a.mask) {
          const uint4 mv = *reinterpret_cast<const uint4*>(a.mask + pix * COUT + c8);
          const __nv_bfloat16* mk = reinterpret_cast<const __nv_bfloat16*>(&mv);
#pragma unroll
          for (int j = 0; j < 8; ++j)
            if (!(__bfloat162float(mk[j]) > 0.f)) o[j] = 0.f;
        }
        if (a.out_f32) {
          float* op = reinterpret_cast<float*>(a.out) + pix * a.out_f32 + c8;
          if (c8 < a.out_f32) *reinterpret_cast<float4*>(op) = make_float4(o[0], o[1], o[2], o[3]);
          if (c8 + 4 < a.out_f32)
            *reinterpret_cast<float4*>(op + 4) = make_float4(o[4], o[5], o[6], o[7]);
        } else {
          __align__(16) __nv_bfloat162 ob[4];
#pragma unroll
          for (int j = 0; j < 4; ++j) ob[j] = __floats2bfloat162_rn(o[2 * j], o[2 * j + 1]);
          *reinterpret_cast<uint4*>(reinterpret_cast<__nv_bfloat16*>(a.out) + pix * COUT + c8) =
              *reinterpret_cast<const uint4*>(ob);
        }
      }
    }
  }
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  if (!ok && tid == 0 && a.status) atomicExch(a.status, 1);
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_free(tmem, S::TMEM_COLS);
}

// ------------------------------------------- forward, rotating accumulators
// Each staged input row is read by the tensor core once instead of three
// times.  Input row r feeds output rows r+1, r and r-1 through the kernel
// rows dy = 0, 1, 2; three TMEM accumulators of COUT columns (slot s holds
// output rows y with y % 3 == s) sit side by side, and for every column
// offset dx one MMA of N = 3 * COUT writes all three: its B operand is the
// three dy weight blocks in the order the slots want for this r.  The weights
// are staged per dx as five blocks W(2) W(1) W(0) W(2) W(1), so the operand
// for row r is the three consecutive blocks starting at block (1 - r) mod 3.
// Every MMA accumulates; a slot is cleared (tcgen05.st of zeros) right after
// its output row has been read, before the next row's MMAs add to it.  Per
// output row this issues 3 * CIN/16 MMAs (N = 3 * COUT) instead of
// 9 * CIN/16 (N = COUT): 2.1x less operand traffic from shared memory, which
// bounds the M128 x N32 form.  A CTA reads input rows y0-1 .. y1, so it runs
// two extra rows per row band.
template <int CIN, int COUT>
struct ConvRotSmem {
  static constexpr int W_BLOCK = COUT * CIN * 2;         // one (dy, dx) weight block
  static constexpr int W_BYTES = 15 * W_BLOCK;           // 3 dx x 5 staged blocks
  static constexpr int ROW_BYTES = (CIN / 8) * kRowLbo;  // one staged input row
  static constexpr int SLOTS = 4;                        // row in the MMA + three in flight
  static constexpr int BYTES = W_BYTES + SLOTS * ROW_BYTES + 64;
  static constexpr uint32_t TMEM_COLS = 3 * COUT <= 64 ? 64 : 128;
};

// Zeros COLS consecutive f32 columns of this thread's TMEM lane.
template <int COLS>
__device__ __forceinline__ void tmem_zero(uint32_t taddr) {
  static_assert(COLS == 16 || COLS == 32, "16 or 32 columns");
  const uint32_t z = 0u;
  if constexpr (COLS == 32) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,"
        "%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1};" ::"r"(taddr),
        "r"(z)
        : "memory");
  } else {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,%1,"
        "%1,%1};" ::"r"(taddr),
        "r"(z)
        : "memory");
  }
  asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}

// MMAs of input row r (staged in its ring slot) into the three accumulators.
template <int CIN, int COUT>
__device__ __forceinline__ void conv_rot_issue(uint32_t tmem, uint32_t slot_addr, uint32_t w_base,
                                               int r, uint32_t idesc) {
  using S = ConvRotSmem<CIN, COUT>;
  const int first = ((1 - r) % 3 + 3) % 3;  // staged block that feeds accumulator slot 0
  const uint64_t adesc0 = umma_desc(slot_addr, kRowLbo, 128);
  const uint64_t bdesc0 = umma_desc(w_base, 128, (CIN / 8) * 128);
#pragma unroll
  for (int dx = 0; dx < 3; ++dx) {
#pragma unroll
    for (int kk = 0; kk < CIN / 16; ++kk)
      umma_bf16(tmem, adesc0 + (uint64_t)((kk * 2 * kRowLbo + dx * 16) >> 4),
                bdesc0 + (uint64_t)(((dx * 5 + first) * S::W_BLOCK + kk * 256) >> 4), idesc, 1);
  }
}

template <int CIN, int COUT>
__global__ void __launch_bounds__(kConvThreads) conv3x3_rot_kernel(const ConvArgs a) {
  using S = ConvRotSmem<CIN, COUT>;
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char* wsm = smem;
  unsigned char* ring = smem + S::W_BYTES;
  uint64_t* bar = reinterpret_cast<uint64_t*>(ring + S::SLOTS * S::ROW_BYTES);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 1);

  const int tid = threadIdx.x, warp = tid >> 5;
  const int x0 = blockIdx.x * kConvTileOut;
  const int y0 = blockIdx.y * a.rows_per_cta;
  const int y1 = min(y0 + a.rows_per_cta, a.h);
  const int b = blockIdx.z;
  auto slot = [&](int r) { return ring + ((r + S::SLOTS) % S::SLOTS) * S::ROW_BYTES; };

  // weights -> shared memory: per dx the blocks of dy = 2, 1, 0, 2, 1 (the
  // packed input holds block (dy * 3 + dx) for each (dy, dx))
  {
    constexpr int kDyOf[5] = {2, 1, 0, 2, 1};
    constexpr int kChunks = S::W_BLOCK / 16;
    const uint4* src = reinterpret_cast<const uint4*>(a.wpk);
    uint4* dst = reinterpret_cast<uint4*>(wsm);
    for (int i = tid; i < 15 * kChunks; i += kConvThreads) {
      const int blk = i / kChunks, off = i % kChunks;
      const int dx = blk / 5, j = blk % 5;
      dst[i] = src[(kDyOf[j] * 3 + dx) * kChunks + off];
    }
  }
  if (tid == 0) mbar_init(bar, 1);
  if (warp == 0) tmem_alloc(tslot, S::TMEM_COLS);
  const int r_first = y0 - 1, r_last = y1;  // input rows this CTA reads
  int issued = r_first - 1;                 // last input row whose copy has been started
  for (int r = r_first; r <= r_first + S::SLOTS - 1 && r <= r_last; ++r) {
    conv_row_async<CIN>(a.in, b, a.h, a.w, r, x0, slot(r));
    issued = r;
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  const uint32_t idesc = umma_idesc_bf16(128, 3 * COUT);
  const uint32_t w_base = smem_u32(wsm);
  const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
  // all three accumulators start at zero
#pragma unroll
  for (int sl = 0; sl < 3; ++sl) tmem_zero<COUT>(lane_addr + (uint32_t)(sl * COUT));
  conv_row_wait_pending(issued - r_first);  // row r_first has landed
  fence_async_smem();                       // the weights (generic stores) too
  tc_fence_before();
  __syncthreads();
  unsigned phase = 0;
  bool ok = true;
  if (y0 < y1 && tid == 0) {
    tc_fence_after();
    conv_rot_issue<CIN, COUT>(tmem, smem_u32(slot(r_first)), w_base, r_first, idesc);
    umma_commit(bar);
  }
  for (int r = r_first; r <= r_last && y0 < y1; ++r) {
    ok = mbar_wait(bar, phase) && ok;
    phase ^= 1;
    tc_fence_after();
    // output row r - 1 is complete: read its accumulator, then clear the slot
    // for the output row r + 2 that the next MMAs start
    const int yo = r - 1;
    const uint32_t acc = lane_addr + (uint32_t)((((yo % 3) + 3) % 3) * COUT);
    float d[COUT];
    if constexpr (COUT == 32)
      tmem_ld32(acc, d);
    else
      tmem_ld16(acc, d);
    tmem_zero<COUT>(acc);
    tc_fence_before();
    if (r + 1 <= r_last) conv_row_wait_pending(issued - (r + 1));  // row r + 1 has landed
    __syncthreads();  // accumulator read and cleared by every thread, row r + 1 staged
    if (r + 1 <= r_last) {
      if (tid == 0) {
        tc_fence_after();
        conv_rot_issue<CIN, COUT>(tmem, smem_u32(slot(r + 1)), w_base, r + 1, idesc);
        umma_commit(bar);
      }
      // row r's MMAs have completed: its slot takes row r + SLOTS
      if (issued + 1 <= r_last && issued + 1 <= r + S::SLOTS) {
        conv_row_async<CIN>(a.in, b, a.h, a.w, issued + 1, x0, slot(issued + 1));
        ++issued;
      }
    }
    const int xo = x0 + tid;
    if (yo >= y0 && yo < y1 && xo < a.w) {
      const size_t pix = ((size_t)b * a.h + yo) * a.w + xo;
#pragma unroll
      for (int c8 = 0; c8 < COUT; c8 += 8) {
        float o[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) o[j] = a.relu ? fmaxf(d[c8 + j], 0.f) : d[c8 + j];
        if (a.mask) {
          const uint4 mv = *reinterpret_cast<const uint4*>(a.mask + pix * COUT + c8);
          const __nv_bfloat16* mk = reinterpret_cast<const __nv_bfloat16*>(&mv);
#pragma unroll
          for (int j = 0; j < 8; ++j)
            if (!(__bfloat162float(mk[j]) > 0.f)) o[j] = 0.f;
        }
        if (a.out_f32) {
          float* op = reinterpret_cast<float*>(a.out) + pix * a.out_f32 + c8;
          if (c8 < a.out_f32) *reinterpret_cast<float4*>(op) = make_float4(o[0], o[1], o[2], o[3]);
          if (c8 + 4 < a.out_f32)
            *reinterpret_cast<float4*>(op + 4) = make_float4(o[4], o[5], o[6], o[7]);
        } else {
          __align__(16) __nv_bfloat162 ob[4];
#pragma unroll
          for (int j = 0; j < 4; ++j) ob[j] = __floats2bfloat162_rn(o[2 * j], o[2 * j + 1]);
          *reinterpret_cast<uint4*>(reinterpret_cast<__nv_bfloat16*>(a.out) + pix * COUT + c8) =
              *reinterpret_cast<const uint4*>(ob);
        }
      }
    }
  }
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  if (!ok && tid == 0 && a.status) atomicExch(a.status, 1);
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_free(tmem, S::TMEM_COLS);
}

// ----------------------------------------------------------- weight grad
struct WgradArgs {
  const __nv_bfloat16* in;    // layer input [batch][h][w][cin]
  const __nv_bfloat16* grad;  // gradient at the layer output [batch][h][w][cout]
  float* partial;             // per CTA: [3 dy][128 (dx, ci)][cout]
  int batch, h, w;
  int rows_per_cta;
  int* status;
};

template <int CIN, int COUT>
struct WgradSmem {
  static constexpr int T_BYTES = 128 * 128 * 2;       // A: (dx, ci) rows x 128 pixels
  static constexpr int G_BYTES = COUT * 128 * 2;      // B: co rows x 128 pixels
  static constexpr int BYTES = T_BYTES + 3 * G_BYTES + 64;
  static constexpr uint32_t TMEM_COLS = 3 * COUT <= 64 ? 64 : 128;
};

template <int CIN, int COUT>
__global__ void __launch_bounds__(kConvThreads) conv3x3_wgrad_tc_kernel(const WgradArgs a) {
  using S = WgradSmem<CIN, COUT>;
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char* tbuf = smem;
  unsigned char* gring = smem + S::T_BYTES;
  uint64_t* bar = reinterpret_cast<uint64_t*>(gring + 3 * S::G_BYTES);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bar + 1);
  const int tid = threadIdx.x, warp = tid >> 5;
  const int x0 = blockIdx.x * 128;
  const int y0 = blockIdx.y * a.rows_per_cta;
  const int y1 = min(y0 + a.rows_per_cta, a.h);
  const int b = blockIdx.z;
  const size_t cta = ((size_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;

  // zero A (the (dx, ci) rows beyond 3*CIN stay zero)
  for (int i = tid; i < S::T_BYTES / 16; i += kConvThreads)
    reinterpret_cast<uint4*>(tbuf)[i] = make_uint4(0, 0, 0, 0);
  if (tid == 0) mbar_init(bar, 1);
  if (warp == 0) tmem_alloc(tslot, S::TMEM_COLS);

  // gradient row r -> ring slot (B operand: element (co, pixel k))
  auto load_grad = [&](int r) {
    unsigned char* dst = gring + ((r + 3) % 3) * S::G_BYTES;
    const int k = tid, x = x0 + k;
    const bool okp = r >= 0 && r < a.h && x < a.w;
    const __nv_bfloat16* src = a.grad + (((size_t)b * a.h + (okp ? r : 0)) * a.w + (okp ? x : 0)) * COUT;
#pragma unroll
    for (int co = 0; co < COUT; ++co) {
      const __nv_bfloat16 v = okp ? src[co] : __float2bfloat16_rn(0.f);
      *reinterpret_cast<__nv_bfloat16*>(dst + core_off(co, k, 128)) = v;
    }
  };
  load_grad(y0 - 1);
  load_grad(y0);
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  const uint32_t idesc = umma_idesc_bf16(128, COUT);
  const uint32_t t_base = smem_u32(tbuf), g_base = smem_u32(gring);
  const uint32_t lbo = 128;
  unsigned phase = 0;
  bool ok = true;
  int started[3] = {0, 0, 0};

  // input rows r contribute to output rows y = r - dy + 1 in [y0, y1)
  for (int r = y0 - 1; r <= y1; ++r) {
    if (r + 1 <= y1) load_grad(r + 1);
    // A: element ((dx, ci), k) = input[r][x0 + k + dx - 1][ci]
    if (r >= 0 && r < a.h) {
      for (int j = tid; j < 130; j += kConvThreads) {
        const int x = x0 + j - 1;
        const bool okp = x >= 0 && x < a.w;
        const __nv_bfloat16* src = a.in + (((size_t)b * a.h + r) * a.w + (okp ? x : 0)) * CIN;
        for (int ci = 0; ci < CIN; ++ci) {
          const __nv_bfloat16 v = okp ? src[ci] : __float2bfloat16_rn(0.f);
#pragma unroll
          for (int dx = 0; dx < 3; ++dx) {
            const int k = j - dx;
            if (k >= 0 && k < 128)
              *reinterpret_cast<__nv_bfloat16*>(tbuf + core_off(dx * CIN + ci, k, 128)) = v;
          }
        }
      }
    } else {
      for (int i = tid; i < (3 * CIN) * 128 / 8; i += kConvThreads) {
        const int row = i / 16, kb = i % 16;
        *reinterpret_cast<uint4*>(tbuf + core_off(row, kb * 8, 128)) = make_uint4(0, 0, 0, 0);
      }
    }
    fence_async_smem();
    __syncthreads();
    bool issued = false;
    if (tid == 0) {
      tc_fence_after();
      for (int dy = 0; dy < 3; ++dy) {
        const int y = r - dy + 1;
        if (y < y0 || y >= y1) continue;
        const uint32_t g_row = g_base + ((y + 3) % 3) * S::G_BYTES;
#pragma unroll
        for (int kk = 0; kk < 8; ++kk)
          umma_bf16(tmem + dy * COUT, umma_desc(t_base + kk * 256, lbo, 16 * 128),
                    umma_desc(g_row + kk * 256, lbo, 16 * 128), idesc, started[dy] | (kk > 0));
        started[dy] = 1;
        issued = true;
      }
      if (issued) umma_commit(bar);
    }
    issued = __syncthreads_or(issued ? 1 : 0);
    if (issued) {
      ok = mbar_wait(bar, phase) && ok;
      phase ^= 1;
    }
    tc_fence_after();
    __syncthreads();
  }
  // epilogue: lane m = (dx, ci), columns (dy, co)
  tc_fence_after();
  const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
  float* out = a.partial + cta * (size_t)(3 * 128 * COUT);
  for (int dy = 0; dy < 3; ++dy) {
#pragma unroll
    for (int c = 0; c < COUT; c += 16) {
      float v[16];
      tmem_ld16(lane_addr + dy * COUT + c, v);
#pragma unroll
      for (int j = 0; j < 16; ++j) out[((size_t)dy * 128 + tid) * COUT + c + j] = y0 < y1 ? v[j] : 0.f;
    }
  }
  if (!ok && tid == 0 && a.status) atomicExch(a.status, 1);
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_free(tmem, S::TMEM_COLS);
}

// dW[dy][dx][ci][co] = sum over CTAs (fixed order) of partial[cta][dy][dx*cin+ci][co].
__global__ void wgrad_reduce_kernel(const float* __restrict__ partial, int nctas, int cin, int cout,
                                    float* __restrict__ dw) {
  const int n = 9 * cin * cout;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int co = i % cout;
    const int ci = (i / cout) % cin;
    const int dx = (i / (cout * cin)) % 3;
    const int dy = i / (3 * cout * cin);
    const size_t off = ((size_t)dy * 128 + dx * cin + ci) * cout + co;
    double s = 0.0;
    for (int c = 0; c < nctas; ++c) s += (double)partial[(size_t)c * 3 * 128 * cout + off];
    dw[i] = (float)s;
  }
}

// --------------------------------------------------- features and fluxes
// Edges of cell (r, c): 0 east (r, c+1), 1 north (r+1, c), 2 north-east
// (r+1, c+1), 3 north-west (r+1, c-1); lengths dx, dy, and the diagonal.
__device__ __forceinline__ void edge_of(int k, int& dr, int& dc) {
  dr = k == 0 ? 0 : 1;
  dc = k == 0 ? 1 : (k == 1 ? 0 : (k == 2 ? 1 : -1));
}

struct LearnedGeom {
  int batch, h, w, pitch;       // height fields [batch][h][pitch]
  double dx, dy, tan_crit;
  double Q;                     // FX quantum (0 for FP64 heights)
  double datum;
};

// The per-pixel kernels below take one image row per block iteration
// (blockIdx.x strides over batch * h rows, threads over the row's columns), so
// no pixel index is divided into (batch, row, column).

// Features: per edge k, (H[c] - H[n_k]) / (L_k tan_crit) as BF16 channels
// 0..3 of a 16-channel pixel (12 zero channels); 0 for edges leaving the grid.
template <typename HT>
__global__ void learned_features_kernel(const LearnedGeom g, const HT* __restrict__ hgt,
                                        __nv_bfloat16* __restrict__ feat) {
  const double diag = sqrt(g.dx * g.dx + g.dy * g.dy);
  const double scale = g.Q > 0.0 ? g.Q : 1.0;
  const double inv_l[4] = {scale / (g.dx * g.tan_crit), scale / (g.dy * g.tan_crit),
                           scale / (diag * g.tan_crit), scale / (diag * g.tan_crit)};
  for (int row = blockIdx.x; row < g.batch * g.h; row += gridDim.x) {
    const int bb = row / g.h, r = row - bb * g.h;
    const HT* H = hgt + (size_t)bb * g.h * g.pitch;
    for (int c = threadIdx.x; c < g.w; c += blockDim.x) {
      const double hc = (double)H[(size_t)r * g.pitch + c];
      __align__(16) __nv_bfloat16 f[16];
#pragma unroll
      for (int k = 0; k < 16; ++k) f[k] = __float2bfloat16_rn(0.f);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        int dr, dc;
        edge_of(k, dr, dc);
        const int rn = r + dr, cn = c + dc;
        if (rn < g.h && cn >= 0 && cn < g.w)
          f[k] = __float2bfloat16_rn((float)((hc - (double)H[(size_t)rn * g.pitch + cn]) * inv_l[k]));
      }
      uint4* dst = reinterpret_cast<uint4*>(feat + ((size_t)row * g.w + c) * 16);
      dst[0] = reinterpret_cast<const uint4*>(f)[0];
      dst[1] = reinterpret_cast<const uint4*>(f)[1];
    }
  }
}

// Proposed transfer on edge k of cell c, in metres: flux * tan_crit * dx,
// limited to half the height difference across that edge (the proposal never
// reverses a difference on its own).  Edges leaving the grid carry nothing.
__device__ __forceinline__ double learned_transfer(const LearnedGeom& g, double flux, double hc,
                                                   double hn) {
  const double t = flux * g.tan_crit * g.dx;
  const double lim = 0.5 * fabs(hc - hn);
  return fmin(fmax(t, -lim), lim);
}

// Fixed point: transfers rounded to whole quanta per edge (int32 [pixel][4]),
// then gathered -- every quantum leaves one cell and enters one neighbour.
// Q is a power of two, so t / Q == t * (1 / Q) exactly.
__global__ void learned_quantize_kernel(const LearnedGeom g, const int32_t* __restrict__ hq,
                                        const float* __restrict__ flux /*[pixel][4]*/,
                                        int32_t* __restrict__ tq /*[pixel][4]*/) {
  const double inv_q = 1.0 / g.Q;
  for (int row = blockIdx.x; row < g.batch * g.h; row += gridDim.x) {
    const int bb = row / g.h, r = row - bb * g.h;
    const int32_t* H = hq + (size_t)bb * g.h * g.pitch;
    for (int c = threadIdx.x; c < g.w; c += blockDim.x) {
      const size_t i = (size_t)row * g.w + c;
      const double hc = (double)H[(size_t)r * g.pitch + c] * g.Q;
      const float4 fl = *reinterpret_cast<const float4*>(flux + i * 4);
      const float fk[4] = {fl.x, fl.y, fl.z, fl.w};
      int q[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        int dr, dc;
        edge_of(k, dr, dc);
        const int rn = r + dr, cn = c + dc;
        q[k] = 0;
        if (rn < g.h && cn >= 0 && cn < g.w) {
          const double hn = (double)H[(size_t)rn * g.pitch + cn] * g.Q;
          const double t = learned_transfer(g, (double)fk[k], hc, hn);
          q[k] = (int)trunc(t * inv_q);  // toward zero: stays within the half-difference limit
        }
      }
      *reinterpret_cast<int4*>(tq + i * 4) = make_int4(q[0], q[1], q[2], q[3]);
    }
  }
}

__global__ void learned_apply_fx_kernel(const LearnedGeom g, int32_t* __restrict__ hq,
                                        const int32_t* __restrict__ tq) {
  for (int row = blockIdx.x; row < g.batch * g.h; row += gridDim.x) {
    const int bb = row / g.h, r = row - bb * g.h;
    int32_t* H = hq + (size_t)bb * g.h * g.pitch;
    for (int c = threadIdx.x; c < g.w; c += blockDim.x) {
      const size_t i = (size_t)row * g.w + c;
      const int4 own = *reinterpret_cast<const int4*>(tq + i * 4);
      long long d = -(long long)own.x - own.y - own.z - own.w;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        int dr, dc;
        edge_of(k, dr, dc);
        const int rs = r - dr, cs = c - dc;  // the cell whose edge k ends here
        if (rs >= 0 && cs >= 0 && cs < g.w)
          d += tq[(((size_t)bb * g.h + rs) * g.w + cs) * 4 + k];
      }
      H[(size_t)r * g.pitch + c] = (int32_t)((long long)H[(size_t)r * g.pitch + c] + d);
    }
  }
}

// Training loss: predicted height change dH = -div(t) (unlimited transfers,
// f32) against the plain relaxation's change; writes the residual per pixel
// and the loss partial per block (blockDim a multiple of 32, at most 1024).
__global__ void learned_loss_kernel(const LearnedGeom g, const float* __restrict__ flux,
                                    const float* __restrict__ target_dh /*[pixel] metres*/,
                                    float* __restrict__ resid /*[pixel]*/,
                                    double* __restrict__ loss_part, float inv_scale2_n) {
  const long long n = (long long)g.batch * g.h * g.w;
  const float s = (float)(g.tan_crit * g.dx);
  double acc = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(i % g.w);
    const int r = (int)((i / g.w) % g.h);
    const int bb = (int)(i / ((long long)g.w * g.h));
    float dh = 0.f;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      int dr, dc;
      edge_of(k, dr, dc);
      if (r + dr < g.h && c + dc >= 0 && c + dc < g.w) dh -= flux[i * 4 + k] * s;
      const int rs = r - dr, cs = c - dc;
      if (rs >= 0 && cs >= 0 && cs < g.w)
        dh += flux[(((long long)bb * g.h + rs) * g.w + cs) * 4 + k] * s;
    }
    const float e = dh - target_dh[i];
    resid[i] = e;
    acc += (double)e * (double)e;
  }
  acc = warp_sum(acc);
  __shared__ double red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w2 = 0; w2 < (int)(blockDim.x >> 5); ++w2) t += red[w2];
    loss_part[blockIdx.x] = t * (double)inv_scale2_n;
  }
}

// dL/dflux[c][k] = 2 s (e[n_k] - e[c]) / (scale^2 N) for edges inside the grid.
__global__ void learned_dflux_kernel(const LearnedGeom g, const float* __restrict__ resid,
                                     __nv_bfloat16* __restrict__ dflux, float inv_scale2_n) {
  const long long n = (long long)g.batch * g.h * g.w;
  const float s = (float)(g.tan_crit * g.dx);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(i % g.w);
    const int r = (int)((i / g.w) % g.h);
    const int bb = (int)(i / ((long long)g.w * g.h));
    __align__(16) __nv_bfloat16 f[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) f[k] = __float2bfloat16_rn(0.f);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      int dr, dc;
      edge_of(k, dr, dc);
      const int rn = r + dr, cn = c + dc;
      if (rn < g.h && cn >= 0 && cn < g.w) {
        const float en = resid[((long long)bb * g.h + rn) * g.w + cn];
        f[k] = __float2bfloat16_rn(2.f * s * (en - resid[i]) * inv_scale2_n);
      }
    }
    uint4* dst = reinterpret_cast<uint4*>(dflux + i * 16);
    dst[0] = reinterpret_cast<const uint4*>(f)[0];
    dst[1] = reinterpret_cast<const uint4*>(f)[1];
  }
}

}  // namespace sb
