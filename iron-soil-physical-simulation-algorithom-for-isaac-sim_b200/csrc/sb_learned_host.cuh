// Host side of the learned repose proposal (C ABI sb_learned_*), included by
// soilb200.cu.  The convolution entry points take device pointers and a
// stream (the training harness owns the activation buffers); the proposal
// entry points work on a context's resident b_eff.
#pragma once

namespace {

using namespace sb;

// Forward / data-gradient convolution.  Default: the nine-tap kernel
// (N = COUT), measured faster at the proposal's sizes; SOILB200_CONV_ROT=1
// selects the rotating-accumulator kernel (each input row read once,
// N = 3 * COUT), which computes the same sums in another order.
template <int CIN, int COUT>
cudaError_t launch_conv(const ConvArgs& a, int rows, cudaStream_t st) {
  static bool attr_set[16] = {false};
  const char* rot_env = std::getenv("SOILB200_CONV_ROT");
  const bool rot = rot_env && rot_env[0] == '1';
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 16 && !attr_set[dev]) {
    cudaError_t e = cudaFuncSetAttribute(conv3x3_tc_kernel<CIN, COUT>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         ConvSmem<CIN, COUT>::BYTES);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(conv3x3_rot_kernel<CIN, COUT>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                               ConvRotSmem<CIN, COUT>::BYTES);
    if (e != cudaSuccess) return e;
    attr_set[dev] = true;
  }
  dim3 grid((a.w + kConvTileOut - 1) / kConvTileOut, (a.h + rows - 1) / rows, a.batch);
  if (rot)
    conv3x3_rot_kernel<CIN, COUT><<<grid, kConvThreads, ConvRotSmem<CIN, COUT>::BYTES, st>>>(a);
  else
    conv3x3_tc_kernel<CIN, COUT><<<grid, kConvFwdThreads, ConvSmem<CIN, COUT>::BYTES, st>>>(a);
  return cudaGetLastError();
}

template <int CIN, int COUT>
cudaError_t launch_wgrad(const WgradArgs& a, cudaStream_t st) {
  using S = WgradSmem<CIN, COUT>;
  static bool attr_set[16] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 16 && !attr_set[dev]) {
    cudaError_t e = cudaFuncSetAttribute(conv3x3_wgrad_tc_kernel<CIN, COUT>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, S::BYTES);
    if (e != cudaSuccess) return e;
    attr_set[dev] = true;
  }
  dim3 grid((a.w + 127) / 128, (a.h + a.rows_per_cta - 1) / a.rows_per_cta, a.batch);
  conv3x3_wgrad_tc_kernel<CIN, COUT><<<grid, kConvThreads, S::BYTES, st>>>(a);
  return cudaGetLastError();
}

bool conv_shape_ok(int cin, int cout) {
  return (cin == 16 || cin == 32) && (cout == 16 || cout == 32);
}

thread_local char g_learned_err[256] = {0};

int lfail(int code, const char* msg) {
  std::snprintf(g_learned_err, sizeof(g_learned_err), "%s", msg);
  return code;
}

// Blocks for the row-per-block pixel kernels: one per image row, at most
// 8 CTAs on each of the 148 SMs (the rest loop).
int learned_row_grid(int batch, int h) {
  const long long rows = (long long)batch * h;
  return (int)(rows < 148LL * 8 ? rows : 148LL * 8);
}

int lcuda(cudaError_t e) {
  if (e == cudaSuccess) return SB_OK;
  std::snprintf(g_learned_err, sizeof(g_learned_err), "CUDA error %s", cudaGetErrorString(e));
  return SB_ERR_CUDA;
}

}  // namespace

extern "C" {

const char* sb_learned_last_error(void) { return g_learned_err; }

int sb_learned_conv(const void* in, void* out, const void* wpk, const void* mask, int batch, int h,
                    int w, int cin, int cout, int relu, int out_f32, int rows_per_cta,
                    int* d_status, void* stream) {
  if (!in || !out || !wpk || batch <= 0 || h <= 0 || w <= 0 || !conv_shape_ok(cin, cout) ||
      rows_per_cta <= 0)
    return lfail(SB_ERR_BAD_ARG, "[soilb200] conv: bad arguments (cin, cout in {16, 32})");
  if (out_f32 < 0 || out_f32 > cout || (out_f32 & 3))
    return lfail(SB_ERR_BAD_ARG, "[soilb200] conv: out_f32 must be 0 or a multiple of 4 <= cout");
  if (((uintptr_t)in | (uintptr_t)out | (uintptr_t)wpk | (uintptr_t)mask) & 15)
    return lfail(SB_ERR_BAD_ARG, "[soilb200] conv: buffers must be 16-byte aligned");
  ConvArgs a{(const __nv_bfloat16*)in, out, (const __nv_bfloat16*)wpk,
             (const __nv_bfloat16*)mask, batch, h, w, rows_per_cta, relu, out_f32, d_status};
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e;
  if (cin == 16 && cout == 32) e = launch_conv<16, 32>(a, rows_per_cta, st);
  else if (cin == 32 && cout == 32) e = launch_conv<32, 32>(a, rows_per_cta, st);
  else if (cin == 32 && cout == 16) e = launch_conv<32, 16>(a, rows_per_cta, st);
  else e = launch_conv<16, 16>(a, rows_per_cta, st);
  return lcuda(e);
}

// partial must hold ceil(w/128) * ceil(h/rows) * batch * 3 * 128 * cout floats.
int sb_learned_wgrad(const void* in, const void* grad, float* partial, size_t partial_floats,
                     float* dw, int batch, int h, int w, int cin, int cout, int rows_per_cta,
                     int* d_status, void* stream) {
  if (!in || !grad || !partial || !dw || batch <= 0 || h <= 0 || w <= 0 ||
      !conv_shape_ok(cin, cout) || rows_per_cta <= 0)
    return lfail(SB_ERR_BAD_ARG, "[soilb200] wgrad: bad arguments (cin, cout in {16, 32})");
  const size_t nctas = (size_t)((w + 127) / 128) * ((h + rows_per_cta - 1) / rows_per_cta) * batch;
  if (partial_floats < nctas * 3 * 128 * (size_t)cout)
    return lfail(SB_ERR_CAPACITY, "[soilb200] wgrad: partial buffer too small");
  WgradArgs a{(const __nv_bfloat16*)in, (const __nv_bfloat16*)grad, partial, batch, h, w,
              rows_per_cta, d_status};
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e;
  if (cin == 16 && cout == 32) e = launch_wgrad<16, 32>(a, st);
  else if (cin == 32 && cout == 32) e = launch_wgrad<32, 32>(a, st);
  else if (cin == 32 && cout == 16) e = launch_wgrad<32, 16>(a, st);
  else e = launch_wgrad<16, 16>(a, st);
  if (e != cudaSuccess) return lcuda(e);
  wgrad_reduce_kernel<<<(9 * cin * cout + 255) / 256, 256, 0, st>>>(partial, (int)nctas, cin, cout, dw);
  return lcuda(cudaGetLastError());
}

// Features of device heights (float64 [batch][h][w]) for training.
int sb_learned_features_f64(const double* heights, void* feat, int batch, int h, int w, double dx,
                            double dy, double tan_crit, void* stream) {
  if (!heights || !feat || batch <= 0 || h <= 0 || w <= 0 || !(tan_crit > 0.0))
    return lfail(SB_ERR_BAD_ARG, "[soilb200] features: bad arguments");
  LearnedGeom g{batch, h, w, w, dx, dy, tan_crit, 0.0, 0.0};
  learned_features_kernel<double><<<learned_row_grid(batch, h), kThreads, 0,
                                    (cudaStream_t)stream>>>(g, heights, (__nv_bfloat16*)feat);
  return lcuda(cudaGetLastError());
}

// Training loss of predicted fluxes (f32 [pixel][4]) against target height
// changes (f32 [pixel]); resid (f32 [pixel]) and dflux (bf16 [pixel][16]) are
// outputs; loss_part holds one double per block (grid_for blocks).
int sb_learned_loss(const float* flux, const float* target_dh, float* resid, void* dflux,
                    double* loss_part, int batch, int h, int w, double dx, double dy,
                    double tan_crit, float inv_scale2_n, void* stream) {
  if (!flux || !target_dh || !resid || !dflux || !loss_part || batch <= 0)
    return lfail(SB_ERR_BAD_ARG, "[soilb200] loss: bad arguments");
  LearnedGeom g{batch, h, w, w, dx, dy, tan_crit, 0.0, 0.0};
  const int blocks = grid_for((long long)batch * h * w);
  cudaStream_t st = (cudaStream_t)stream;
  learned_loss_kernel<<<blocks, kThreads, 0, st>>>(g, flux, target_dh, resid, loss_part,
                                                   inv_scale2_n);
  learned_dflux_kernel<<<blocks, kThreads, 0, st>>>(g, resid, (__nv_bfloat16*)dflux, inv_scale2_n);
  return lcuda(cudaGetLastError());
}

// The whole network's forward pass in one kernel (inference only): features
// bf16 [batch][h][w][16] in, the last layer's first four channels as f32
// [batch][h][w][4] out; w1..w4 are the layers' packed weights.
int sb_learned_forward(const void* feat, float* flux, const void* w1, const void* w2,
                       const void* w3, const void* w4, int batch, int h, int w, int rows_per_cta,
                       int* d_status, void* stream) {
  if (!feat || !flux || !w1 || !w2 || !w3 || !w4 || batch <= 0 || h <= 0 || w <= 0 ||
      rows_per_cta < 0 || batch > 65535)
    return lfail(SB_ERR_BAD_ARG, "[soilb200] forward: bad arguments");
  if (((uintptr_t)feat | (uintptr_t)flux | (uintptr_t)w1 | (uintptr_t)w2 | (uintptr_t)w3 |
       (uintptr_t)w4) & 15)
    return lfail(SB_ERR_BAD_ARG, "[soilb200] forward: buffers must be 16-byte aligned");
  EncodeTiledFn enc = encode_fn();
  if (!enc) return lfail(SB_ERR_CUDA, "[soilb200] forward: cuTensorMapEncodeTiled unavailable");
  // features as a 4-D tensor (channel, x, y, image); one box = one channel
  // chunk of a staged row: 8 channels x 130 pixels, zeros outside the image
  CUtensorMap map;
  const cuuint64_t dims[4] = {16, (cuuint64_t)w, (cuuint64_t)h, (cuuint64_t)batch};
  const cuuint64_t strides[3] = {32, (cuuint64_t)w * 32, (cuuint64_t)w * (cuuint64_t)h * 32};
  const cuuint32_t box[4] = {8, (cuuint32_t)kRowPixels, 1, 1};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  if (enc(&map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void*>(feat), dims, strides, box,
          estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
          CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return lfail(SB_ERR_CUDA, "[soilb200] forward: feature tensor map rejected");
  const int strips = (w + kNetTileOut - 1) / kNetTileOut;
  int rows = rows_per_cta;
  if (rows == 0) {  // one CTA per SM: about one wave over the 148 SMs
    const long long per_band = (long long)strips * batch;
    const int bands = per_band >= 148 ? 1 : (int)(148 / per_band);
    rows = (h + bands - 1) / bands;
  }
  static bool attr_set[16] = {false};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 16 && !attr_set[dev]) {
    cudaError_t e = cudaFuncSetAttribute(net_forward_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         NetSmem::BYTES);
    if (e != cudaSuccess) return lcuda(e);
    attr_set[dev] = true;
  }
  NetArgs a{{(const __nv_bfloat16*)w1, (const __nv_bfloat16*)w2, (const __nv_bfloat16*)w3,
             (const __nv_bfloat16*)w4},
            flux, batch, h, w, rows, d_status};
  dim3 grid(strips, (h + rows - 1) / rows, batch);
  net_forward_kernel<<<grid, kNetThreads, NetSmem::BYTES, (cudaStream_t)stream>>>(map, a);
  return lcuda(cudaGetLastError());
}

int sb_learned_loss_blocks(int batch, int h, int w) {
  return grid_for((long long)batch * h * w);
}

// Proposal on a context's resident b_eff (SB_FX32): features into feat
// (bf16 [ny][nx][16]); after the caller's network has produced flux (f32
// [ny][nx][4]), sb_learned_apply moves the proposed transfers in whole
// quanta (tq: int32 [ny][nx][4] scratch), exactly conserving sum(b_eff).
int sb_learned_features(sb_ctx* ctx, void* feat, double tan_crit) {
  if (!ctx || !feat || !(tan_crit > 0.0)) return SB_ERR_BAD_ARG;
  if (!fx(ctx)) return fail(ctx, SB_ERR_BAD_ARG, "[soilb200] the learned proposal runs on SB_FX32 grids");
  LearnedGeom g{1, ctx->d.ny, ctx->d.nx, ctx->pitch, ctx->d.dx_m, ctx->d.dy_m, tan_crit,
                ctx->quantum, ctx->d.datum_m};
  learned_features_kernel<int32_t><<<learned_row_grid(1, ctx->d.ny), kThreads, 0, ctx->stream>>>(
      g, (const int32_t*)ctx->b, (__nv_bfloat16*)feat);
  ctx->launches++;
  SB_CUDA(ctx, cudaGetLastError());
  return SB_OK;
}

int sb_learned_apply(sb_ctx* ctx, const float* flux, int32_t* tq, double tan_crit) {
  if (!ctx || !flux || !tq || !(tan_crit > 0.0)) return SB_ERR_BAD_ARG;
  if (((uintptr_t)flux | (uintptr_t)tq) & 15)
    return fail(ctx, SB_ERR_BAD_ARG, "[soilb200] learned apply: flux and tq must be 16-byte aligned");
  if (!fx(ctx)) return fail(ctx, SB_ERR_BAD_ARG, "[soilb200] the learned proposal runs on SB_FX32 grids");
  LearnedGeom g{1, ctx->d.ny, ctx->d.nx, ctx->pitch, ctx->d.dx_m, ctx->d.dy_m, tan_crit,
                ctx->quantum, ctx->d.datum_m};
  const int blocks = learned_row_grid(1, ctx->d.ny);
  learned_quantize_kernel<<<blocks, kThreads, 0, ctx->stream>>>(g, (const int32_t*)ctx->b, flux, tq);
  learned_apply_fx_kernel<<<blocks, kThreads, 0, ctx->stream>>>(g, (int32_t*)ctx->b, tq);
  ctx->launches += 2;
  SB_CUDA(ctx, cudaGetLastError());
  return SB_OK;
}

}  // extern "C"
