// soilb200 C ABI: context/state ownership, field transfer and step orchestration.
//
// One sb_ctx owns one terrain grid on one GPU (the role of the reference's
// DeviceBulkState, runtime/bulk_state_authority.py:493-619): pitched SoA
// fields, TMA descriptors over them, device-resident loop control blocks and
// CUDA graphs.  A Mobile V2 physics step is a single graph launch:
//
//   begin (dt -> control block) -> ledger/prologue (static check, first dt)
//   -> WHILE(device flag) { fv_substep } -> ledger (after)
//
// so the substep loop that the reference drives from the host with two
// blocking synchronisations per substep (bulk_interaction/warp_mobile_v2.py:
// 181-216) runs entirely on the device; the host synchronises once per step.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/soilb200.h"
#include "sb_common.cuh"
#include "sb_fv.cuh"
#include "sb_ledger.cuh"

using namespace sb;

namespace {

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

struct MobileGraph {
  cudaGraphExec_t exec = nullptr;
  cudaGraph_t graph = nullptr;
  FvConst key{};
  double static_limit = 0.0;
  bool valid = false;
};

}  // namespace

struct sb_ctx {
  sb_grid_desc d{};
  int pitch = 0;        // elements per row
  size_t esize = 0;     // bytes per element of float-like fields
  cudaStream_t stream = nullptr;
  double quantum = 1.0;
  // fields (precision dependent element type)
  void* b = nullptr;
  void* z = nullptr;
  void* h[2] = {nullptr, nullptr};
  void* qx[2] = {nullptr, nullptr};
  void* qy[2] = {nullptr, nullptr};
  void* ext_x = nullptr;
  void* ext_y = nullptr;
  int32_t* reached = nullptr;
  // staging + control
  double* staging = nullptr;
  int* range_error = nullptr;
  FvControl* ctl = nullptr;
  StepIO* io = nullptr;
  double* partials = nullptr;
  long long* ipartials = nullptr;
  unsigned int* arrive = nullptr;
  double* dt_dev = nullptr;
  double* dt_host = nullptr;      // pinned
  FvControl* ctl_host = nullptr;  // pinned
  StepIO* io_host = nullptr;      // pinned
  int parity_host = 0;            // mirror of ctl->parity after the last sync
  CUtensorMap tm_b, tm_h[2], tm_qx[2], tm_qy[2];
  int fv_blocks = 0;
  int ledger_blocks = 0;
  MobileGraph mobile;
  long long launches = 0;
  char err[1024] = {0};
};

namespace {

int fail(sb_ctx* ctx, int code, const char* fmt, ...) {
  if (ctx) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(ctx->err, sizeof(ctx->err), fmt, ap);
    va_end(ap);
  }
  return code;
}

#define SB_CUDA(ctx, call)                                                                  \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess)                                                                  \
      return fail((ctx), SB_ERR_CUDA, "CUDA error %s at %s:%d (%s)", cudaGetErrorString(e_), \
                  __FILE__, __LINE__, #call);                                               \
  } while (0)

bool fx(const sb_ctx* c) { return c->d.precision == SB_FX32; }

int encode_2d(sb_ctx* ctx, CUtensorMap* map, void* base, CUtensorMapDataType dtype,
              size_t esize, int box_w, int box_h) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return fail(ctx, SB_ERR_CUDA, "cuTensorMapEncodeTiled entry point unavailable");
  cuuint64_t dims[2] = {(cuuint64_t)ctx->d.nx, (cuuint64_t)ctx->d.ny};
  cuuint64_t strides[1] = {(cuuint64_t)ctx->pitch * esize};
  cuuint32_t box[2] = {(cuuint32_t)box_w, (cuuint32_t)box_h};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = fn(map, dtype, 2, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                  CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(ctx, SB_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return SB_OK;
}

int grid_for(long long n) {
  long long b = (n + kThreads - 1) / kThreads;
  if (b > 148 * 8) b = 148 * 8;
  return (int)(b < 1 ? 1 : b);
}

void* field_ptr(sb_ctx* c, int field, int* is_int, int* is_height, int* is_support) {
  *is_int = 0;
  *is_height = 0;
  *is_support = 0;
  switch (field) {
    case SB_FIELD_Z_BASE: *is_support = 1; return c->z;
    case SB_FIELD_B_EFF: *is_support = 1; return c->b;
    case SB_FIELD_MOBILE: *is_height = 1; return c->h[c->parity_host];
    case SB_FIELD_MOMENTUM_X: return c->qx[c->parity_host];
    case SB_FIELD_MOMENTUM_Y: return c->qy[c->parity_host];
    case SB_FIELD_EXTERNAL_X: return c->ext_x;
    case SB_FIELD_EXTERNAL_Y: return c->ext_y;
    case SB_FIELD_FRONTIER_REACHED: *is_int = 1; return c->reached;
    default: return nullptr;
  }
}

FvConst make_const(const sb_ctx* ctx, const sb_mobile_params* p) {
  FvConst c{};
  c.ny = ctx->d.ny;
  c.nx = ctx->d.nx;
  c.pitch = ctx->pitch;
  c.tiles_x = (ctx->d.nx + kTileX - 1) / kTileX;
  c.nblocks = c.tiles_x * ((ctx->d.ny + kTileY - 1) / kTileY);
  c.dx = ctx->d.dx_m;
  c.dy = ctx->d.dy_m;
  c.K = p->earth_pressure_coefficient;
  c.g = p->gravity_m_s2;
  c.cfl = p->cfl;
  c.dry = p->dry_tolerance_m;
  c.mu_g = p->basal_friction_coefficient * p->gravity_m_s2;
  c.c_half = 0.5 * p->earth_pressure_coefficient * p->gravity_m_s2;
  c.kg = p->earth_pressure_coefficient * p->gravity_m_s2;
  c.min_spacing = ctx->d.dx_m < ctx->d.dy_m ? ctx->d.dx_m : ctx->d.dy_m;
  c.Q = ctx->quantum;
  c.Kf = (float)c.K;
  c.KGf = (float)c.kg;
  c.HKGf = (float)c.c_half;
  c.Qf = (float)ctx->quantum;
  c.invQf = (float)(1.0 / ctx->quantum);
  c.dryf = (float)c.dry;
  c.max_substeps = p->maximum_substeps;
  c.has_external = p->use_external ? 1 : 0;
  return c;
}

template <bool FX>
size_t fv_smem_bytes() {
  return sizeof(FvSmem<FX>) + 128;
}

template <bool FX>
void fv_args(sb_ctx* ctx, const FvConst& c, cudaGraphConditionalHandle* handle, int* use_handle,
             std::vector<void*>& args) {
  args = {(void*)&c,           (void*)&ctx->tm_b,     (void*)&ctx->tm_h[0], (void*)&ctx->tm_h[1],
          (void*)&ctx->tm_qx[0], (void*)&ctx->tm_qx[1], (void*)&ctx->tm_qy[0], (void*)&ctx->tm_qy[1],
          (void*)&ctx->h[0],   (void*)&ctx->h[1],     (void*)&ctx->qx[0],   (void*)&ctx->qx[1],
          (void*)&ctx->qy[0],  (void*)&ctx->qy[1],    (void*)&ctx->ext_x,   (void*)&ctx->ext_y,
          (void*)&ctx->ctl,    (void*)&ctx->partials, (void*)handle,        (void*)use_handle};
}

template <bool FX>
void ledger_args(sb_ctx* ctx, const FvConst& c, double* datum, double* static_limit, int* mode,
                 cudaGraphConditionalHandle* handle, int* use_handle, std::vector<void*>& args) {
  args = {(void*)&c,         (void*)&ctx->b,        (void*)&ctx->h[0],      (void*)&ctx->h[1],
          (void*)&ctx->qx[0], (void*)&ctx->qx[1],   (void*)&ctx->qy[0],     (void*)&ctx->qy[1],
          (void*)&ctx->ext_x, (void*)&ctx->ext_y,   (void*)datum,           (void*)static_limit,
          (void*)mode,        (void*)&ctx->ctl,     (void*)&ctx->io,        (void*)&ctx->partials,
          (void*)&ctx->ipartials, (void*)&ctx->arrive, (void*)handle,       (void*)use_handle};
}

int add_kernel(sb_ctx* ctx, cudaGraph_t g, cudaGraphNode_t* node, const cudaGraphNode_t* deps,
               size_t ndeps, void* func, dim3 grid, size_t smem, void** args) {
  cudaKernelNodeParams kp{};
  kp.func = func;
  kp.gridDim = grid;
  kp.blockDim = dim3(kThreads);
  kp.sharedMemBytes = (unsigned)smem;
  kp.kernelParams = args;
  SB_CUDA(ctx, cudaGraphAddKernelNode(node, g, deps, ndeps, &kp));
  return SB_OK;
}

template <bool FX>
int build_mobile_graph(sb_ctx* ctx, const FvConst& c, double static_limit) {
  MobileGraph& mg = ctx->mobile;
  if (mg.exec) {
    cudaGraphExecDestroy(mg.exec);
    mg.exec = nullptr;
  }
  if (mg.graph) {
    cudaGraphDestroy(mg.graph);
    mg.graph = nullptr;
  }
  mg.valid = false;
  cudaGraph_t g;
  SB_CUDA(ctx, cudaGraphCreate(&g, 0));
  mg.graph = g;
  cudaGraphConditionalHandle handle;
  SB_CUDA(ctx, cudaGraphConditionalHandleCreate(&handle, g, 0, cudaGraphCondAssignDefault));
  int use_handle = 1;
  double datum = ctx->d.datum_m;
  double limit = static_limit;
  int mode0 = 0, mode1 = 1;
  FvConst cc = c;

  cudaGraphNode_t n_begin, n_pro, n_loop, n_after, n_body;
  {
    void* args[] = {(void*)&ctx->ctl, (void*)&ctx->dt_dev};
    int rc = add_kernel(ctx, g, &n_begin, nullptr, 0, (void*)fv_begin_kernel, dim3(1), 0, args);
    if (rc) return rc;
  }
  {
    std::vector<void*> args;
    ledger_args<FX>(ctx, cc, &datum, &limit, &mode0, &handle, &use_handle, args);
    int rc = add_kernel(ctx, g, &n_pro, &n_begin, 1, (void*)ledger_kernel<FX>,
                        dim3(ctx->ledger_blocks), 0, args.data());
    if (rc) return rc;
  }
  {
    cudaGraphNodeParams cp{};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = handle;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    SB_CUDA(ctx, cudaGraphAddNode(&n_loop, g, &n_pro, 1, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    std::vector<void*> args;
    fv_args<FX>(ctx, cc, &handle, &use_handle, args);
    int rc = add_kernel(ctx, body, &n_body, nullptr, 0, (void*)fv_substep_kernel<FX>,
                        dim3(c.nblocks), fv_smem_bytes<FX>(), args.data());
    if (rc) return rc;
  }
  {
    int no_handle = 0;
    std::vector<void*> args;
    ledger_args<FX>(ctx, cc, &datum, &limit, &mode1, &handle, &no_handle, args);
    int rc = add_kernel(ctx, g, &n_after, &n_loop, 1, (void*)ledger_kernel<FX>,
                        dim3(ctx->ledger_blocks), 0, args.data());
    if (rc) return rc;
  }
  SB_CUDA(ctx, cudaGraphInstantiate(&mg.exec, g, 0));
  mg.key = c;
  mg.static_limit = static_limit;
  mg.valid = true;
  return SB_OK;
}

void fill_ledger(const sb_ctx* ctx, const LedgerOut& o, const sb_mobile_params* p,
                 sb_mobile_ledger* L) {
  const double dx = ctx->d.dx_m, dy = ctx->d.dy_m;
  const double area = dx * dy;
  const double f = dx * dy / 6.0;  // one weight unit
  const double rho = p->density_kg_m3;
  const double K = p->earth_pressure_coefficient, g = p->gravity_m_s2;
  double hsum, hsum_w;
  if (fx(ctx)) {
    hsum = (double)o.iq[0] * ctx->quantum;
    hsum_w = (double)o.iq[1] * ctx->quantum;
    L->mass_quanta = o.iq[0];
    L->volume_w_quanta = o.iq[1];
  } else {
    hsum = o.v[L_HSUM];
    hsum_w = o.v[L_HSUM_W];
    L->mass_quanta = 0;
    L->volume_w_quanta = 0;
  }
  L->mass_m3 = hsum * dx * dy;
  L->momentum_m4_s[0] = o.v[L_QX] * dx * dy;
  L->momentum_m4_s[1] = o.v[L_QY] * dx * dy;
  L->kinetic = 0.5 * o.v[L_HS2] * area;
  L->gravitational = g * o.v[L_HB] * area;
  L->internal = 0.5 * K * g * o.v[L_HH] * area;
  L->volume_w_m3 = hsum_w * f;
  L->momentum_w[0] = rho * o.v[L_QX_W] * f;
  L->momentum_w[1] = rho * o.v[L_QY_W] * f;
  L->kinetic_w_j = 0.5 * rho * o.v[L_HS2_W] * f;
  L->potential_w_j = rho * g * o.v[L_HB_W] * f;
  L->pressure_w_j = rho * 0.5 * K * g * o.v[L_HH_W] * f;
  L->max_speed_m_s = o.v[L_MAXSPEED];
  L->min_h_m = -o.v[L_NEGMINH];
}

}  // namespace

extern "C" {

const char* sb_version(void) { return "soilb200 0.1 (sm_100a)"; }

size_t sb_sizeof(const char* type_name) {
  if (!type_name) return 0;
  struct Entry { const char* name; size_t size; };
  static const Entry table[] = {
      {"sb_grid_desc", sizeof(sb_grid_desc)},
      {"sb_mobile_params", sizeof(sb_mobile_params)},
      {"sb_mobile_ledger", sizeof(sb_mobile_ledger)},
      {"sb_mobile_stats", sizeof(sb_mobile_stats)},
  };
  for (const Entry& e : table)
    if (std::strcmp(e.name, type_name) == 0) return e.size;
  return 0;
}

int sb_last_error(sb_ctx* ctx, char* buffer, size_t length) {
  if (!buffer || length == 0) return SB_ERR_BAD_ARG;
  const char* msg = ctx ? ctx->err : "";
  snprintf(buffer, length, "%s", msg);
  return SB_OK;
}

int64_t sb_kernel_launch_count(sb_ctx* ctx) { return ctx ? ctx->launches : 0; }

int sb_ctx_create(const sb_grid_desc* desc, sb_ctx** out) {
  if (!desc || !out) return SB_ERR_BAD_ARG;
  *out = nullptr;
  sb_ctx* ctx = new sb_ctx();
  ctx->d = *desc;
  const sb_grid_desc& d = *desc;
  if (d.ny < 2 || d.nx < 2 || !(d.dx_m > 0) || !(d.dy_m > 0) || !std::isfinite(d.dx_m) ||
      !std::isfinite(d.dy_m) || (d.precision != SB_FP64 && d.precision != SB_FX32) ||
      d.tile_size < 1) {
    int rc = fail(ctx, SB_ERR_BAD_ARG, "[soilb200] invalid grid description");
    *out = ctx;
    return rc;
  }
  if (d.precision == SB_FX32 && (d.height_exponent < 4 || d.height_exponent > 40)) {
    int rc = fail(ctx, SB_ERR_BAD_ARG, "[soilb200] height_exponent out of range");
    *out = ctx;
    return rc;
  }
  *out = ctx;
  SB_CUDA(ctx, cudaSetDevice(d.device));
  SB_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
  ctx->quantum = std::ldexp(1.0, -d.height_exponent);
  ctx->pitch = (d.nx + 31) / 32 * 32;
  ctx->esize = fx(ctx) ? 4 : 8;
  const size_t field_bytes = (size_t)ctx->pitch * d.ny * ctx->esize;
  void** all[] = {&ctx->b, &ctx->z, &ctx->h[0], &ctx->h[1], &ctx->qx[0],
                  &ctx->qx[1], &ctx->qy[0], &ctx->qy[1], &ctx->ext_x, &ctx->ext_y};
  for (void** p : all) {
    SB_CUDA(ctx, cudaMalloc(p, field_bytes));
    SB_CUDA(ctx, cudaMemsetAsync(*p, 0, field_bytes, ctx->stream));
  }
  SB_CUDA(ctx, cudaMalloc(&ctx->reached, (size_t)ctx->pitch * d.ny * sizeof(int32_t)));
  SB_CUDA(ctx, cudaMemsetAsync(ctx->reached, 0, (size_t)ctx->pitch * d.ny * 4, ctx->stream));
  SB_CUDA(ctx, cudaMalloc(&ctx->staging, (size_t)d.ny * d.nx * sizeof(double)));
  SB_CUDA(ctx, cudaMalloc(&ctx->range_error, sizeof(int)));
  SB_CUDA(ctx, cudaMalloc(&ctx->ctl, sizeof(FvControl)));
  SB_CUDA(ctx, cudaMemsetAsync(ctx->ctl, 0, sizeof(FvControl), ctx->stream));
  SB_CUDA(ctx, cudaMalloc(&ctx->io, sizeof(StepIO)));
  SB_CUDA(ctx, cudaMemsetAsync(ctx->io, 0, sizeof(StepIO), ctx->stream));
  const int tiles = ((d.nx + kTileX - 1) / kTileX) * ((d.ny + kTileY - 1) / kTileY);
  ctx->fv_blocks = tiles;
  ctx->ledger_blocks = grid_for((long long)d.ny * d.nx);
  const size_t np = (size_t)(tiles > ctx->ledger_blocks ? tiles : ctx->ledger_blocks) *
                    (kFvPartial > L_NP ? kFvPartial : L_NP);
  SB_CUDA(ctx, cudaMalloc(&ctx->partials, np * sizeof(double)));
  SB_CUDA(ctx, cudaMalloc(&ctx->ipartials, (size_t)ctx->ledger_blocks * kLedgerI64 * 8));
  SB_CUDA(ctx, cudaMalloc(&ctx->arrive, sizeof(unsigned)));
  SB_CUDA(ctx, cudaMemsetAsync(ctx->arrive, 0, sizeof(unsigned), ctx->stream));
  SB_CUDA(ctx, cudaMalloc(&ctx->dt_dev, sizeof(double)));
  SB_CUDA(ctx, cudaMallocHost(&ctx->dt_host, sizeof(double)));
  SB_CUDA(ctx, cudaMallocHost(&ctx->ctl_host, sizeof(FvControl)));
  SB_CUDA(ctx, cudaMallocHost(&ctx->io_host, sizeof(StepIO)));
  // TMA descriptors (box = halo tile of the FV kernel)
  int rc;
  if (fx(ctx)) {
    using Tl = FvTile<true>;
    if ((rc = encode_2d(ctx, &ctx->tm_b, ctx->b, CU_TENSOR_MAP_DATA_TYPE_INT32, 4, Tl::BW, Tl::BH)))
      return rc;
    for (int k = 0; k < 2; ++k) {
      if ((rc = encode_2d(ctx, &ctx->tm_h[k], ctx->h[k], CU_TENSOR_MAP_DATA_TYPE_INT32, 4, Tl::BW,
                          Tl::BH)))
        return rc;
      if ((rc = encode_2d(ctx, &ctx->tm_qx[k], ctx->qx[k], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4,
                          Tl::BW, Tl::BH)))
        return rc;
      if ((rc = encode_2d(ctx, &ctx->tm_qy[k], ctx->qy[k], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4,
                          Tl::BW, Tl::BH)))
        return rc;
    }
    SB_CUDA(ctx, cudaFuncSetAttribute(fv_substep_kernel<true>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)fv_smem_bytes<true>()));
  } else {
    using Tl = FvTile<false>;
    if ((rc = encode_2d(ctx, &ctx->tm_b, ctx->b, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8, Tl::BW,
                        Tl::BH)))
      return rc;
    for (int k = 0; k < 2; ++k) {
      if ((rc = encode_2d(ctx, &ctx->tm_h[k], ctx->h[k], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8,
                          Tl::BW, Tl::BH)))
        return rc;
      if ((rc = encode_2d(ctx, &ctx->tm_qx[k], ctx->qx[k], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8,
                          Tl::BW, Tl::BH)))
        return rc;
      if ((rc = encode_2d(ctx, &ctx->tm_qy[k], ctx->qy[k], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 8,
                          Tl::BW, Tl::BH)))
        return rc;
    }
    SB_CUDA(ctx, cudaFuncSetAttribute(fv_substep_kernel<false>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)fv_smem_bytes<false>()));
  }
  SB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return SB_OK;
}

int sb_ctx_destroy(sb_ctx* ctx) {
  if (!ctx) return SB_OK;
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->mobile.exec) cudaGraphExecDestroy(ctx->mobile.exec);
  if (ctx->mobile.graph) cudaGraphDestroy(ctx->mobile.graph);
  void* ptrs[] = {ctx->b, ctx->z, ctx->h[0], ctx->h[1], ctx->qx[0], ctx->qx[1], ctx->qy[0],
                  ctx->qy[1], ctx->ext_x, ctx->ext_y, ctx->reached, ctx->staging,
                  ctx->range_error, ctx->ctl, ctx->io, ctx->partials, ctx->ipartials,
                  ctx->arrive, ctx->dt_dev};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (ctx->dt_host) cudaFreeHost(ctx->dt_host);
  if (ctx->ctl_host) cudaFreeHost(ctx->ctl_host);
  if (ctx->io_host) cudaFreeHost(ctx->io_host);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return SB_OK;
}

int sb_synchronize(sb_ctx* ctx) {
  if (!ctx) return SB_ERR_BAD_ARG;
  SB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return SB_OK;
}

int sb_upload(sb_ctx* ctx, int field, const double* host) {
  if (!ctx || !host) return SB_ERR_BAD_ARG;
  int is_int, is_h, is_s;
  void* dst = field_ptr(ctx, field, &is_int, &is_h, &is_s);
  if (!dst || is_int) return fail(ctx, SB_ERR_BAD_ARG, "[soilb200] field %d is not a float field", field);
  const int ny = ctx->d.ny, nx = ctx->d.nx;
  if (!fx(ctx)) {
    SB_CUDA(ctx, cudaMemcpy2DAsync(dst, (size_t)ctx->pitch * 8, host, (size_t)nx * 8,
                                   (size_t)nx * 8, ny, cudaMemcpyHostToDevice, ctx->stream));
    SB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return SB_OK;
  }
  SB_CUDA(ctx, cudaMemcpyAsync(ctx->staging, host, (size_t)ny * nx * 8, cudaMemcpyHostToDevice,
                               ctx->stream));
  const int grid = grid_for((long long)ny * nx);
  if (is_h || is_s) {
    SB_CUDA(ctx, cudaMemsetAsync(ctx->range_error, 0, sizeof(int), ctx->stream));
    to_fixed_kernel<<<grid, kThreads, 0, ctx->stream>>>(ctx->staging, (int32_t*)dst, ny, nx,
                                                        ctx->pitch, is_s ? ctx->d.datum_m : 0.0,
                                                        std::ldexp(1.0, ctx->d.height_exponent),
                                                        ctx->range_error);
    ctx->launches++;
    int herr = 0;
    SB_CUDA(ctx, cudaGetLastError());
    SB_CUDA(ctx, cudaMemcpyAsync(&herr, ctx->range_error, sizeof(int), cudaMemcpyDeviceToHost,
                                 ctx->stream));
    SB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (herr)
      return fail(ctx, SB_ERR_RANGE,
                  "[soilb200] field %d exceeds the fixed-point range (2^31 quanta of 2^-%d m)",
                  field, ctx->d.height_exponent);
    return SB_OK;
  }
  to_float_kernel<<<grid, kThreads, 0, ctx->stream>>>(ctx->staging, (float*)dst, ny, nx, ctx->pitch);
  ctx->launches++;
  SB_CUDA(ctx, cudaGetLastError());
  SB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return SB_OK;
}

int sb_download(sb_ctx* ctx, int field, double* host) {
  if (!ctx || !host) return SB_ERR_BAD_ARG;
  int is_int, is_h, is_s;
  void* src = field_ptr(ctx, field, &is_int, &is_h, &is_s);
  if (!src || is_int) return fail(ctx, SB_ERR_BAD_ARG, "[soilb200] field %d is not a float field", field);
  const int ny = ctx->d.ny, nx = ctx->d.nx;
  if (!fx(ctx)) {
    SB_CUDA(ctx, cudaMemcpy2DAsync(host, (size_t)nx * 8, src, (size_t)ctx->pitch * 8,
                                   (size_t)nx * 8, ny, cudaMemcpyDeviceToHost, ctx->stream));
    SB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return SB_OK;
  }
  const int grid = grid_for((long long)ny * nx);
  if (is_h || is_s)
    from_fixed_kernel<<<grid, kThreads, 0, ctx->stream>>>((const int32_t*)src, ctx->staging, ny, nx,
                                                          ctx->pitch, is_s ? ctx->d.datum_m : 0.0,
                                                          ctx->quantum);
  else
    from_float_kernel<<<grid, kThreads, 0, ctx->stream>>>((const float*)src, ctx->staging, ny, nx,
                                                          ctx->pitch);
  ctx->launches++;
  SB_CUDA(ctx, cudaGetLastError());
  SB_CUDA(ctx, cudaMemcpyAsync(host, ctx->staging, (size_t)ny * nx * 8, cudaMemcpyDeviceToHost,
                               ctx->stream));
  SB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return SB_OK;
}

int sb_upload_i32(sb_ctx* ctx, int field, const int32_t* host) {
  if (!ctx || !host) return SB_ERR_BAD_ARG;
  int is_int, is_h, is_s;
  void* dst = field_ptr(ctx, field, &is_int, &is_h, &is_s);
  if (!dst || !is_int) return fail(ctx, SB_ERR_BAD_ARG, "[soilb200] field %d is not an int field", field);
  SB_CUDA(ctx, cudaMemcpy2DAsync(dst, (size_t)ctx->pitch * 4, host, (size_t)ctx->d.nx * 4,
                                 (size_t)ctx->d.nx * 4, ctx->d.ny, cudaMemcpyHostToDevice,
                                 ctx->stream));
  SB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return SB_OK;
}

int sb_download_i32(sb_ctx* ctx, int field, int32_t* host) {
  if (!ctx || !host) return SB_ERR_BAD_ARG;
  int is_int, is_h, is_s;
  void* src = field_ptr(ctx, field, &is_int, &is_h, &is_s);
  if (!src || !is_int) return fail(ctx, SB_ERR_BAD_ARG, "[soilb200] field %d is not an int field", field);
  SB_CUDA(ctx, cudaMemcpy2DAsync(host, (size_t)ctx->d.nx * 4, src, (size_t)ctx->pitch * 4,
                                 (size_t)ctx->d.nx * 4, ctx->d.ny, cudaMemcpyDeviceToHost,
                                 ctx->stream));
  SB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return SB_OK;
}

static int check_params(sb_ctx* ctx, const sb_mobile_params* p) {
  const double vals[] = {ctx->d.dx_m, ctx->d.dy_m, p->gravity_m_s2, p->earth_pressure_coefficient,
                         p->cfl, p->dry_tolerance_m, p->basal_friction_coefficient};
  for (double v : vals)
    if (!std::isfinite(v) || v <= 0.0)
      return fail(ctx, SB_ERR_BAD_ARG, "MobileV2 configuration must be finite/positive");
  return SB_OK;
}

int sb_mobile_step(sb_ctx* ctx, double dt_s, const sb_mobile_params* params, sb_mobile_stats* out) {
  if (!ctx || !params || !out) return SB_ERR_BAD_ARG;
  if (!std::isfinite(dt_s) || dt_s <= 0.0) return fail(ctx, SB_ERR_BAD_ARG, "dt must be finite/positive");
  int rc = check_params(ctx, params);
  if (rc) return rc;
  const FvConst c = make_const(ctx, params);
  const double static_limit =
      std::tan(params->start_angle_deg * (M_PI / 180.0)) + 1.0e-14;
  MobileGraph& mg = ctx->mobile;
  if (!mg.valid || std::memcmp(&mg.key, &c, sizeof(FvConst)) != 0 ||
      mg.static_limit != static_limit) {
    rc = fx(ctx) ? build_mobile_graph<true>(ctx, c, static_limit)
                 : build_mobile_graph<false>(ctx, c, static_limit);
    if (rc) return rc;
  }
  *ctx->dt_host = dt_s;
  SB_CUDA(ctx, cudaMemcpyAsync(ctx->dt_dev, ctx->dt_host, sizeof(double), cudaMemcpyHostToDevice,
                               ctx->stream));
  SB_CUDA(ctx, cudaGraphLaunch(mg.exec, ctx->stream));
  SB_CUDA(ctx, cudaMemcpyAsync(ctx->ctl_host, ctx->ctl, sizeof(FvControl), cudaMemcpyDeviceToHost,
                               ctx->stream));
  SB_CUDA(ctx, cudaMemcpyAsync(ctx->io_host, ctx->io, sizeof(StepIO), cudaMemcpyDeviceToHost,
                               ctx->stream));
  SB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  const FvControl& k = *ctx->ctl_host;
  ctx->parity_host = k.parity;
  ctx->launches += 3 + k.substeps;
  std::memset(out, 0, sizeof(*out));
  out->substeps = k.substeps;
  out->static_skip = k.static_skip;
  out->cfl_limited = k.cfl_limited;
  out->status = k.status;
  out->maximum_cfl = k.max_cfl;
  const double area = ctx->d.dx_m * ctx->d.dy_m;
  for (int i = 0; i < 2; ++i) {
    out->conservative_impulse_m4_s[i] = k.diag[i] * area;
    out->external_impulse_m4_s[i] = k.diag[2 + i] * area;
    out->friction_impulse_m4_s[i] = k.diag[4 + i] * area;
  }
  out->friction_dissipation = k.diag[6] * area;
  out->external_work = k.diag[7] * area;
  fill_ledger(ctx, ctx->io_host->before, params, &out->before);
  fill_ledger(ctx, ctx->io_host->after, params, &out->after);
  if (k.status == SB_ERR_POSITIVITY) return fail(ctx, SB_ERR_POSITIVITY, "MobileV2 positivity failure");
  if (k.status == SB_ERR_SUBSTEP_CAP)
    return fail(ctx, SB_ERR_SUBSTEP_CAP, "MobileV2 maximum_substeps exceeded");
  if (k.status == SB_ERR_WAIT_LIMIT)
    return fail(ctx, SB_ERR_WAIT_LIMIT, "[soilb200] a bounded device wait gave up (TMA tile load)");
  if (k.status != 0) return fail(ctx, k.status, "[soilb200] device status %d", k.status);
  return SB_OK;
}

int sb_mobile_ledger_of(sb_ctx* ctx, const sb_mobile_params* params, sb_mobile_ledger* out) {
  if (!ctx || !params || !out) return SB_ERR_BAD_ARG;
  int rc = check_params(ctx, params);
  if (rc) return rc;
  FvConst c = make_const(ctx, params);
  double datum = ctx->d.datum_m, limit = 0.0;
  int mode = 1, use_handle = 0;
  cudaGraphConditionalHandle handle{};
  std::vector<void*> args;
  if (fx(ctx))
    ledger_args<true>(ctx, c, &datum, &limit, &mode, &handle, &use_handle, args);
  else
    ledger_args<false>(ctx, c, &datum, &limit, &mode, &handle, &use_handle, args);
  void* fn = fx(ctx) ? (void*)ledger_kernel<true> : (void*)ledger_kernel<false>;
  SB_CUDA(ctx, cudaLaunchKernel(fn, dim3(ctx->ledger_blocks), dim3(kThreads), args.data(), 0,
                                ctx->stream));
  ctx->launches++;
  SB_CUDA(ctx, cudaMemcpyAsync(ctx->io_host, ctx->io, sizeof(StepIO), cudaMemcpyDeviceToHost,
                               ctx->stream));
  SB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  fill_ledger(ctx, ctx->io_host->after, params, out);
  return SB_OK;
}

}  // extern "C"
