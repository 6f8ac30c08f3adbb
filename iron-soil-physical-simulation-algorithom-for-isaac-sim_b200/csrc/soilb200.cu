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

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/soilb200.h"
#include "sb_common.cuh"
#include "sb_fv.cuh"
#include "sb_ledger.cuh"
#include "sb_labels.cuh"
#include "sb_relax.cuh"
#include "sb_exchange.cuh"
#include "sb_deposition.cuh"
#include "sb_avalanche.cuh"
#include "sb_surface.cuh"
#include "sb_path.cuh"
#include "sb_batch.cuh"
#include "sb_learned.cuh"
#include "sb_learned_net.cuh"

using namespace sb;

namespace sb {
// Address of fv_stream_kernel<true>, instantiated in sb_fv_fast.cu (compiled
// with FMA contraction); this file only ever instantiates the exact variant.
const void* fv_stream_fast_kernel();
const void* batch_fv_fast_kernel();  // batch_fv_kernel<true>, same translation unit
const void* fv_loop_fast_kernel();   // fv_loop_kernel<true>, same translation unit
}  // namespace sb

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

struct LoopGraph {  // graph whose key is a RelaxConst
  cudaGraphExec_t exec = nullptr;
  cudaGraph_t graph = nullptr;
  RelaxConst key{};
  bool valid = false;
  void reset() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
    valid = false;
  }
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
  double* fv_diag = nullptr;  // per-FV-block impulse/energy sums of the current step
  double* lpart_before = nullptr;       // "before" ledger block partials (folded at step end)
  long long* lipart_before = nullptr;
  unsigned int* arrive = nullptr;
  double* dt_dev = nullptr;
  double* dt_host = nullptr;      // pinned
  FvControl* ctl_host = nullptr;  // pinned
  StepIO* io_host = nullptr;      // pinned
  int parity_host = 0;            // mirror of ctl->parity after the last sync
  CUtensorMap tm_b, tm_h[2], tm_qx[2], tm_qy[2];
  int fv_blocks = 0;
  // FX32 substep kernel: register-streaming strips (default) or the TMA tile
  // kernel (SOILB200_FV_TILE=1); strips of 30 output columns, fv_rows row
  // chunks per strip
  int fv_stream = 0;
  int fv_exact = 0;  // 1: FX32 strip kernel with the CPU mirror's IEEE arithmetic
  int fv_persistent = 0;  // 1: step graphs run the substeps in one cooperative launch
  int fv_rows = 0;  // FX streaming kernel: row chunks per strip
  int fv_strips = 0;
  int fv_stream_blocks = 0;
  int ledger_blocks = 0;
  MobileGraph mobile;
  cudaEvent_t ev_loop[2] = {nullptr, nullptr};  // around the substep WHILE node
  cudaEvent_t ev_path[2] = {nullptr, nullptr};  // first and last node of the step graph
  // optional event nodes between the stages of the step graph's main chain
  // (SOILB200_STAGE_EVENTS=1): a device-time breakdown of one step
  static constexpr int kStages = 10;
  bool stage_events = false;
  cudaEvent_t ev_stage[kStages] = {};
  int n_stage = 0;
  float stage_ms[kStages] = {};
  bool use_graphs = true;  // false: host-driven launches (profilers that cannot see
                           // kernels inside conditional graphs)
  // labelling (flat ny*nx arrays)
  int* parent = nullptr;
  void* slope = nullptr;
  void* severity = nullptr;
  int* latch = nullptr;
  int* previous = nullptr;
  double* export_cum = nullptr;
  double* export_base = nullptr;
  LabelRoots roots{};
  int* root_list = nullptr;
  LabelOut* lout = nullptr;
  LabelOut* lout_host = nullptr;
  // relaxation
  void* b_alt = nullptr;
  CUtensorMap tm_relax[2];
  CUtensorMap tm_reached[2];  // frontier_reached and its ping-pong partner (reached-gated sweep)
  int* reached_alt = nullptr;
  int ftiles0 = 0, ftiles1 = 0;
  int* ftile_next = nullptr;   // next-round active tiles (seeded by labels / seeds)
  // residual frontier: phase[0] = the round's tile membership flags,
  // phase[1] = the round's compacted tile list (both ntiles ints)
  int* phase[2] = {nullptr, nullptr};
  int frontier_grid = 1;  // CTAs of the list-driven frontier kernels
  RelaxControl* rctl = nullptr;
  RelaxControl* rctl_host = nullptr;
  LoopGraph relax_full;
  LoopGraph relax_full2;  // second cached relaxation graph (e.g. short sweeps vs. to tolerance)
  LoopGraph relax_reached;  // reached-gated (event-driven) sweep to tolerance
  int relax_lru = 0;
  LoopGraph frontier;
  // fused plain-path step
  PathState* pstate = nullptr;
  PathState* pstate_host = nullptr;
  int* path_count = nullptr;       // device copy of the cut length (written by path_begin)
  PathInput* path_in = nullptr;     // pinned, mapped: dt + cut length of the next step
  int32_t* path_idx = nullptr;      // pinned, mapped: cut command of the next step
  double* path_val = nullptr;
  int path_cap = 0;                 // cells path_idx / path_val hold
  cudaGraphExec_t path_exec = nullptr;
  cudaGraph_t path_graph = nullptr;
  unsigned char path_key[512] = {0};
  bool path_valid = false;
  // exchange command buffers
  int32_t* xidx = nullptr;
  double* xval = nullptr;
  ExchangeOut* xout = nullptr;
  ExchangeOut* xout_host = nullptr;
  double* xpart = nullptr;  // exchange kernels' block partials (3 x grid_for max)
  // deposition: tool-forcing mask (int32, flat), per-cell settled volume
  // record (double m^3, flat), device/host result records
  int32_t* forcing = nullptr;
  double* m2r = nullptr;
  DepositionOut* dep_out = nullptr;
  DepositionOut* dep_out_host = nullptr;
  // large-avalanche activation history (flat) and lifecycle sums
  double* owned_surface = nullptr;
  int* act_count = nullptr;
  double* act_first = nullptr;
  double* act_last = nullptr;
  double* r2m = nullptr;
  void* initial_b = nullptr;   // b_eff at sb_avalanche_set_initial_resting (pitched)
  int* ptiles = nullptr;       // activity tile flags (tile_size tiles)
  MobilizeOut* mob_out = nullptr;
  MobilizeOut* mob_out_host = nullptr;
  double* pers_out = nullptr;
  double* pers_out_host = nullptr;
  // surface publication: captured free surface (flat double), dirty tile
  // flags, batched query buffers (grown on demand)
  double* surf_before = nullptr;
  int* dtiles = nullptr;
  double* q_rows = nullptr;
  double* q_cols = nullptr;
  double* q_out = nullptr;
  int q_cap = 0;
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
    if (e_ != cudaSuccess) {                                                                \
      cudaGetLastError(); /* a failed call must not surface again in a later check */      \
      return fail((ctx), SB_ERR_CUDA, "CUDA error %s at %s:%d (%s)", cudaGetErrorString(e_), \
                  __FILE__, __LINE__, #call);                                               \
    }                                                                                       \
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

void* field_ptr(sb_ctx* c, int field, int* is_int, int* is_height, int* is_support,
                int* is_flat = nullptr) {
  *is_int = 0;
  *is_height = 0;
  *is_support = 0;
  if (is_flat) *is_flat = 0;
  switch (field) {
    case SB_FIELD_LABELS: *is_int = 1; if (is_flat) *is_flat = 1; return c->parent;
    case SB_FIELD_LATCH: *is_int = 1; if (is_flat) *is_flat = 1; return c->latch;
    case SB_FIELD_PREVIOUS_COMPONENT: *is_int = 1; if (is_flat) *is_flat = 1; return c->previous;
    case SB_FIELD_SLOPE: if (is_flat) *is_flat = 1; return c->slope;
    case SB_FIELD_SEVERITY: if (is_flat) *is_flat = 1; return c->severity;
    case SB_FIELD_Z_BASE: *is_support = 1; return c->z;
    case SB_FIELD_B_EFF: *is_support = 1; return c->b;
    case SB_FIELD_MOBILE: *is_height = 1; return c->h[c->parity_host];
    case SB_FIELD_MOMENTUM_X: return c->qx[c->parity_host];
    case SB_FIELD_MOMENTUM_Y: return c->qy[c->parity_host];
    case SB_FIELD_EXTERNAL_X: return c->ext_x;
    case SB_FIELD_EXTERNAL_Y: return c->ext_y;
    case SB_FIELD_FRONTIER_REACHED: *is_int = 1; return c->reached;
    case SB_FIELD_FORCING: *is_int = 1; if (is_flat) *is_flat = 1; return c->forcing;
    case SB_FIELD_ACTIVATION_COUNT: *is_int = 1; if (is_flat) *is_flat = 1; return c->act_count;
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
  if (ctx->fv_stream) {
    c.tiles_x = ctx->fv_strips;
    c.nblocks = ctx->fv_stream_blocks;
    c.row_chunks = ctx->fv_rows;
  }
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
  c.gsx[0] = c.Q / (2.0 * c.dx);
  c.gsx[1] = c.Q / c.dx;
  c.gsy[0] = c.Q / (2.0 * c.dy);
  c.gsy[1] = c.Q / c.dy;
  c.Kf = (float)c.K;
  c.KGf = (float)c.kg;
  c.HKGf = (float)c.c_half;
  c.Qf = (float)ctx->quantum;
  c.invQf = (float)(1.0 / ctx->quantum);
  c.dryf = (float)c.dry;
  c.QKf = (float)(ctx->quantum / c.K);
  c.max_substeps = p->maximum_substeps;
  c.has_external = p->use_external ? 1 : 0;
  return c;
}

template <bool FX>
size_t fv_smem_bytes() {
  return sizeof(FvSmem<FX>) + 128;
}

// Kernel, grid, shared memory and argument list of one substep launch.
struct FvLaunch {
  void* func = nullptr;
  dim3 grid;
  size_t smem = 0;
  std::vector<void*> args;
};

template <bool FX>
void fv_launch(sb_ctx* ctx, const FvConst& c, cudaGraphConditionalHandle* handle, int* use_handle,
               FvLaunch& L) {
  if (FX && ctx->fv_stream) {
    L.func = ctx->fv_exact ? (void*)fv_stream_kernel<false>
                           : const_cast<void*>(fv_stream_fast_kernel());
    L.smem = 0;
    L.args = {(void*)&c,         (void*)&ctx->b,     (void*)&ctx->h[0],  (void*)&ctx->h[1],
              (void*)&ctx->qx[0], (void*)&ctx->qx[1], (void*)&ctx->qy[0], (void*)&ctx->qy[1],
              (void*)&ctx->ext_x, (void*)&ctx->ext_y, (void*)&ctx->ctl,   (void*)&ctx->fv_diag,
              (void*)handle,      (void*)use_handle};
  } else {
    L.func = (void*)fv_substep_kernel<FX>;
    L.smem = fv_smem_bytes<FX>();
    L.args = {(void*)&c,           (void*)&ctx->tm_b,     (void*)&ctx->tm_h[0], (void*)&ctx->tm_h[1],
              (void*)&ctx->tm_qx[0], (void*)&ctx->tm_qx[1], (void*)&ctx->tm_qy[0], (void*)&ctx->tm_qy[1],
              (void*)&ctx->h[0],   (void*)&ctx->h[1],     (void*)&ctx->qx[0],   (void*)&ctx->qx[1],
              (void*)&ctx->qy[0],  (void*)&ctx->qy[1],    (void*)&ctx->ext_x,   (void*)&ctx->ext_y,
              (void*)&ctx->ctl,    (void*)&ctx->fv_diag,  (void*)handle,        (void*)use_handle};
  }
  L.grid = dim3(c.nblocks);
}

int add_kernel(sb_ctx* ctx, cudaGraph_t g, cudaGraphNode_t* node, const cudaGraphNode_t* deps,
               size_t ndeps, void* func, dim3 grid, size_t smem, void** args,
               unsigned threads = kThreads);

// Adds a step graph's substep loop after `dep`: the persistent cooperative
// kernel (all substeps in one launch) when ctx->fv_persistent, else a WHILE
// conditional node whose body runs two substep launches per iteration (the
// second returns at once when the first ended the step).
template <bool FX>
int add_substep_loop(sb_ctx* ctx, cudaGraph_t g, cudaGraphNode_t dep, const FvConst& c,
                     cudaGraphConditionalHandle* handle, int* use_handle,
                     cudaGraphNode_t* out) {
  if (FX && ctx->fv_stream && ctx->fv_persistent) {
    FvConst cc = c;
    void* args[] = {(void*)&cc,         (void*)&ctx->b,     (void*)&ctx->h[0],  (void*)&ctx->h[1],
                    (void*)&ctx->qx[0], (void*)&ctx->qx[1], (void*)&ctx->qy[0], (void*)&ctx->qy[1],
                    (void*)&ctx->ext_x, (void*)&ctx->ext_y, (void*)&ctx->ctl,   (void*)&ctx->fv_diag};
    void* fn = ctx->fv_exact ? (void*)fv_loop_kernel<false>
                             : const_cast<void*>(fv_loop_fast_kernel());
    int rc = add_kernel(ctx, g, out, &dep, 1, fn, dim3(ctx->fv_stream_blocks), 0, args, kThreads);
    if (rc) return rc;
    cudaLaunchAttributeValue v{};
    v.cooperative = 1;
    SB_CUDA(ctx, cudaGraphKernelNodeSetAttribute(*out, cudaLaunchAttributeCooperative, &v));
    return SB_OK;
  }
  cudaGraphNodeParams cp{};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = *handle;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  SB_CUDA(ctx, cudaGraphAddNode(out, g, &dep, 1, &cp));
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  FvLaunch L;
  fv_launch<FX>(ctx, c, handle, use_handle, L);
  cudaGraphNode_t n1, n2;
  int rc = add_kernel(ctx, body, &n1, nullptr, 0, L.func, L.grid, L.smem, L.args.data(), kThreads);
  if (rc) return rc;
  return add_kernel(ctx, body, &n2, &n1, 1, L.func, L.grid, L.smem, L.args.data(), kThreads);
}

template <bool FX>
void ledger_args(sb_ctx* ctx, const FvConst& c, double* datum, double* static_limit, int* mode,
                 cudaGraphConditionalHandle* handle, int* use_handle, std::vector<void*>& args) {
  args = {(void*)&c,         (void*)&ctx->b,        (void*)&ctx->z,  (void*)&ctx->h[0],      (void*)&ctx->h[1],
          (void*)&ctx->qx[0], (void*)&ctx->qx[1],   (void*)&ctx->qy[0],     (void*)&ctx->qy[1],
          (void*)&ctx->ext_x, (void*)&ctx->ext_y,   (void*)datum,           (void*)static_limit,
          (void*)mode,        (void*)&ctx->ctl,     (void*)&ctx->io,        (void*)&ctx->partials,
          (void*)&ctx->ipartials, (void*)&ctx->arrive, (void*)&ctx->fv_diag,
          (void*)&ctx->lpart_before, (void*)&ctx->lipart_before, (void*)handle,
          (void*)use_handle};
}

int add_kernel(sb_ctx* ctx, cudaGraph_t g, cudaGraphNode_t* node, const cudaGraphNode_t* deps,
               size_t ndeps, void* func, dim3 grid, size_t smem, void** args,
               unsigned threads) {
  cudaKernelNodeParams kp{};
  kp.func = func;
  kp.gridDim = grid;
  kp.blockDim = dim3(threads);
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
  // a conditional handle without a conditional node can fail instantiation:
  // the persistent substep loop needs none
  handle = 0;
  if (!(FX && ctx->fv_stream && ctx->fv_persistent))
    SB_CUDA(ctx, cudaGraphConditionalHandleCreate(&handle, g, 0, cudaGraphCondAssignDefault));
  int use_handle = 1;
  double datum = ctx->d.datum_m;
  double limit = static_limit;
  int mode0 = 0, mode1 = 2;  // 2: after-step ledger + substep diagnostics fold
  FvConst cc = c;

  cudaGraphNode_t n_begin, n_pro, n_loop, n_after;
  {
    void* dt_mapped = nullptr;
    SB_CUDA(ctx, cudaHostGetDevicePointer(&dt_mapped, ctx->dt_host, 0));
    void* args[] = {(void*)&ctx->ctl, &dt_mapped, (void*)&ctx->dt_dev};
    int rc = add_kernel(ctx, g, &n_begin, nullptr, 0, (void*)fv_begin_mapped_kernel, dim3(1), 0,
                        args);
    if (rc) return rc;
  }
  {
    std::vector<void*> args;
    // the prologue sets the WHILE condition only when the loop is one
    int pro_handle = (FX && ctx->fv_stream && ctx->fv_persistent) ? 0 : use_handle;
    ledger_args<FX>(ctx, cc, &datum, &limit, &mode0, &handle, &pro_handle, args);
    int rc = add_kernel(ctx, g, &n_pro, &n_begin, 1, (void*)ledger_kernel<FX>,
                        dim3(ctx->ledger_blocks), 0, args.data());
    if (rc) return rc;
  }
  cudaGraphNode_t n_ev0, n_ev1;
  SB_CUDA(ctx, cudaGraphAddEventRecordNode(&n_ev0, g, &n_pro, 1, ctx->ev_loop[0]));
  {
    int rc = add_substep_loop<FX>(ctx, g, n_ev0, cc, &handle, &use_handle, &n_loop);
    if (rc) return rc;
  }
  {
    int no_handle = 0;
    std::vector<void*> args;
    ledger_args<FX>(ctx, cc, &datum, &limit, &mode1, &handle, &no_handle, args);
    SB_CUDA(ctx, cudaGraphAddEventRecordNode(&n_ev1, g, &n_loop, 1, ctx->ev_loop[1]));
    int rc = add_kernel(ctx, g, &n_after, &n_ev1, 1, (void*)ledger_kernel<FX>,
                        dim3(ctx->ledger_blocks), 0, args.data());
    if (rc) return rc;
  }
  {
    // loop control and step ledgers straight into the pinned host copies
    PathRecordPtrs rp{};
    void *ctl_dst = nullptr, *io_dst = nullptr;
    SB_CUDA(ctx, cudaHostGetDevicePointer(&ctl_dst, ctx->ctl_host, 0));
    SB_CUDA(ctx, cudaHostGetDevicePointer(&io_dst, ctx->io_host, 0));
    rp.src[0] = ctx->ctl;
    rp.dst[0] = ctl_dst;
    rp.bytes[0] = (int)sizeof(FvControl);
    rp.src[1] = ctx->io;
    rp.dst[1] = io_dst;
    rp.bytes[1] = (int)sizeof(StepIO);
    int nrec = 2;
    void* args[] = {&rp, &nrec};
    cudaGraphNode_t n_rec;
    int rc = add_kernel(ctx, g, &n_rec, &n_after, 1, (void*)records_copy_kernel, dim3(1), 0, args);
    if (rc) return rc;
  }
  SB_CUDA(ctx, cudaGraphInstantiate(&mg.exec, g, 0));
  mg.key = c;
  mg.static_limit = static_limit;
  mg.valid = true;
  return SB_OK;
}

// Host form of a device ledger for a grid of spacing dx, dy; fixed-point
// grids (fxp) convert their exact quanta sums with the grid's quantum.
void fill_ledger_geom(bool fxp, double dx, double dy, double quantum, const LedgerOut& o,
                      const sb_mobile_params* p, sb_mobile_ledger* L) {
  const double area = dx * dy;
  const double f = dx * dy / 6.0;  // one weight unit
  const double rho = p->density_kg_m3;
  const double K = p->earth_pressure_coefficient, g = p->gravity_m_s2;
  double hsum, hsum_w;
  if (fxp) {
    hsum = (double)o.iq[0] * quantum;
    hsum_w = (double)o.iq[1] * quantum;
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
  L->resting_volume_w_m3 = fxp ? (double)o.iq[2] * quantum * f : o.v[L_REST_W] * f;
  L->resting_w_quanta = fxp ? o.iq[2] : 0;
}

void fill_ledger(const sb_ctx* ctx, const LedgerOut& o, const sb_mobile_params* p,
                 sb_mobile_ledger* L) {
  fill_ledger_geom(fx(ctx), ctx->d.dx_m, ctx->d.dy_m, ctx->quantum, o, p, L);
}

template <bool FX>
static int mobile_step_host_loop(sb_ctx* ctx, const FvConst& c, double static_limit) {
  // Same kernels as the graph, launched from the host; the loop flag is read
  // back after every substep (one synchronisation per substep).
  double datum = ctx->d.datum_m, limit = static_limit;
  int mode0 = 0, mode1 = 2, no_handle = 0;  // 2: after-step ledger + diagnostics fold
  cudaGraphConditionalHandle handle{};
  FvConst cc = c;
  {
    void* args[] = {(void*)&ctx->ctl, (void*)&ctx->dt_dev};
    SB_CUDA(ctx, cudaLaunchKernel((void*)fv_begin_kernel, dim3(1), dim3(kThreads), args, 0,
                                  ctx->stream));
  }
  std::vector<void*> args;
  ledger_args<FX>(ctx, cc, &datum, &limit, &mode0, &handle, &no_handle, args);
  SB_CUDA(ctx, cudaLaunchKernel((void*)ledger_kernel<FX>, dim3(ctx->ledger_blocks), dim3(kThreads),
                                args.data(), 0, ctx->stream));
  SB_CUDA(ctx, cudaEventRecord(ctx->ev_loop[0], ctx->stream));
  if (FX && ctx->fv_stream && ctx->fv_persistent) {
    // the step graph's persistent substep loop, as one cooperative launch
    void* pargs[] = {(void*)&cc,         (void*)&ctx->b,     (void*)&ctx->h[0],  (void*)&ctx->h[1],
                     (void*)&ctx->qx[0], (void*)&ctx->qx[1], (void*)&ctx->qy[0], (void*)&ctx->qy[1],
                     (void*)&ctx->ext_x, (void*)&ctx->ext_y, (void*)&ctx->ctl,   (void*)&ctx->fv_diag};
    void* fn = ctx->fv_exact ? (void*)fv_loop_kernel<false>
                             : const_cast<void*>(fv_loop_fast_kernel());
    SB_CUDA(ctx, cudaLaunchCooperativeKernel(fn, dim3(ctx->fv_stream_blocks), dim3(kThreads),
                                             pargs, 0, ctx->stream));
  }
  FvLaunch L;
  fv_launch<FX>(ctx, cc, &handle, &no_handle, L);
  for (int it = 0; it <= c.max_substeps; ++it) {
    SB_CUDA(ctx, cudaMemcpyAsync(ctx->ctl_host, ctx->ctl, sizeof(FvControl), cudaMemcpyDeviceToHost,
                                 ctx->stream));
    SB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (ctx->ctl_host->done) break;
    SB_CUDA(ctx, cudaLaunchKernel(L.func, L.grid, dim3(kThreads), L.args.data(), L.smem,
                                  ctx->stream));
  }
  SB_CUDA(ctx, cudaEventRecord(ctx->ev_loop[1], ctx->stream));
  std::vector<void*> a2;
  ledger_args<FX>(ctx, cc, &datum, &limit, &mode1, &handle, &no_handle, a2);
  SB_CUDA(ctx, cudaLaunchKernel((void*)ledger_kernel<FX>, dim3(ctx->ledger_blocks), dim3(kThreads),
                                a2.data(), 0, ctx->stream));
  return SB_OK;
}

int fill_mobile_stats(sb_ctx* ctx, const sb_mobile_params* params, sb_mobile_stats* out) {
  const FvControl& k = *ctx->ctl_host;
  ctx->parity_host = k.parity;
  float loop_ms = 0.f;
  SB_CUDA(ctx, cudaEventElapsedTime(&loop_ms, ctx->ev_loop[0], ctx->ev_loop[1]));
  std::memset(out, 0, sizeof(*out));
  out->substep_loop_ms = loop_ms;
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
  return SB_OK;
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
      {"sb_label_params", sizeof(sb_label_params)},
      {"sb_label_stats", sizeof(sb_label_stats)},
      {"sb_relax_params", sizeof(sb_relax_params)},
      {"sb_relax_stats", sizeof(sb_relax_stats)},
      {"sb_path_params", sizeof(sb_path_params)},
      {"sb_path_stats", sizeof(sb_path_stats)},
      {"sb_patch_desc", sizeof(sb_patch_desc)},
      {"sb_deposition_params", sizeof(sb_deposition_params)},
      {"sb_deposition_stats", sizeof(sb_deposition_stats)},
      {"sb_mobilize_stats", sizeof(sb_mobilize_stats)},
      {"sb_persistence_stats", sizeof(sb_persistence_stats)},
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

void* sb_stream(sb_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

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
  {
    const char* env = std::getenv("SOILB200_NO_GRAPH");
    ctx->use_graphs = !(env && env[0] == '1');
  }
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
  if (d.precision == SB_FX32) {
    const char* tile_env = std::getenv("SOILB200_FV_TILE");
    ctx->fv_stream = (tile_env && tile_env[0] == '1') ? 0 : 1;
    const char* exact_env = std::getenv("SOILB200_FV_EXACT");
    ctx->fv_exact = (exact_env && exact_env[0] == '1') ? 1 : 0;
    ctx->fv_strips = (d.nx + kStripOut - 1) / kStripOut;
    // row chunks per strip: at most one wave of warps (4 CTAs of 8 warps on
    // each SM of this device) and at least kMinChunkRows rows per chunk (every
    // chunk pays one extra row of loads, two cell preparations and one face);
    // the chunks split the rows evenly (sizes differ by at most one row)
    int sms = 0;
    SB_CUDA(ctx, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, d.device));
    const long long want_warps = (long long)std::max(sms, 1) * 32;
    long long chunks = want_warps / ctx->fv_strips;
    chunks = std::min<long long>(chunks, d.ny / kMinChunkRows);
    chunks = std::max<long long>(chunks, 1);
    if (const char* rows_env = std::getenv("SOILB200_FV_ROWS")) {
      const long long r = std::atoll(rows_env);
      if (r >= 1 && r <= 4096) chunks = (d.ny + r - 1) / r;
    }
    ctx->fv_rows = (int)chunks;
    const long long warps = (long long)ctx->fv_strips * chunks;
    ctx->fv_stream_blocks = (int)((warps + kThreads / 32 - 1) / (kThreads / 32));
    // the persistent substep loop needs every CTA resident at once
    const void* loop_fn = ctx->fv_exact ? (const void*)fv_loop_kernel<false> : fv_loop_fast_kernel();
    int per_sm = 0;
    SB_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, loop_fn, kThreads, 0));
    const char* pers_env = std::getenv("SOILB200_FV_PERSISTENT");
    ctx->fv_persistent = (!(pers_env && pers_env[0] == '0') &&
                          (long long)per_sm * sms >= ctx->fv_stream_blocks)
                             ? 1
                             : 0;
  }
  // grid-stride reductions: three CTAs per SM (the ledger kernel's register
  // bound) keep the final fold short
  ctx->ledger_blocks = std::min(grid_for((long long)d.ny * d.nx), 3 * 148);
  const size_t np = (size_t)std::max({tiles, ctx->ledger_blocks, ctx->fv_stream_blocks}) *
                    (kFvPartial > L_NP ? kFvPartial : L_NP);
  SB_CUDA(ctx, cudaMalloc(&ctx->partials, np * sizeof(double)));
  SB_CUDA(ctx, cudaMalloc(&ctx->ipartials, (size_t)ctx->ledger_blocks * kLedgerI64 * 8));
  SB_CUDA(ctx, cudaMalloc(&ctx->lpart_before, (size_t)ctx->ledger_blocks * L_NP * sizeof(double)));
  SB_CUDA(ctx, cudaMalloc(&ctx->lipart_before, (size_t)ctx->ledger_blocks * kLedgerI64 * 8));
  {
    const size_t nd = (size_t)kFvDiag * std::max(tiles, ctx->fv_stream_blocks);
    SB_CUDA(ctx, cudaMalloc(&ctx->fv_diag, nd * sizeof(double)));
    SB_CUDA(ctx, cudaMemsetAsync(ctx->fv_diag, 0, nd * sizeof(double), ctx->stream));
  }
  SB_CUDA(ctx, cudaMalloc(&ctx->arrive, sizeof(unsigned)));
  SB_CUDA(ctx, cudaMemsetAsync(ctx->arrive, 0, sizeof(unsigned), ctx->stream));
  SB_CUDA(ctx, cudaMalloc(&ctx->dt_dev, sizeof(double)));
  SB_CUDA(ctx, cudaMallocHost(&ctx->dt_host, sizeof(double)));
  SB_CUDA(ctx, cudaMallocHost(&ctx->ctl_host, sizeof(FvControl)));
  SB_CUDA(ctx, cudaMallocHost(&ctx->io_host, sizeof(StepIO)));
  SB_CUDA(ctx, cudaEventCreate(&ctx->ev_loop[0]));
  SB_CUDA(ctx, cudaEventCreate(&ctx->ev_loop[1]));
  SB_CUDA(ctx, cudaEventCreate(&ctx->ev_path[0]));
  SB_CUDA(ctx, cudaEventCreate(&ctx->ev_path[1]));
  {
    const char* env = std::getenv("SOILB200_STAGE_EVENTS");
    ctx->stage_events = env && env[0] == '1';
    if (ctx->stage_events)
      for (cudaEvent_t& e : ctx->ev_stage) SB_CUDA(ctx, cudaEventCreate(&e));
  }
  // labelling buffers (flat ny*nx)
  const size_t n = (size_t)d.ny * d.nx;
  SB_CUDA(ctx, cudaMalloc(&ctx->parent, n * 4));
  SB_CUDA(ctx, cudaMalloc(&ctx->slope, n * ctx->esize));
  SB_CUDA(ctx, cudaMalloc(&ctx->severity, n * ctx->esize));
  SB_CUDA(ctx, cudaMalloc(&ctx->latch, n * 4));
  SB_CUDA(ctx, cudaMalloc(&ctx->previous, n * 4));
  SB_CUDA(ctx, cudaMalloc(&ctx->export_cum, n * 8));
  SB_CUDA(ctx, cudaMalloc(&ctx->export_base, n * 8));
  SB_CUDA(ctx, cudaMalloc(&ctx->roots.count, n * 4));
  SB_CUDA(ctx, cudaMalloc(&ctx->roots.area6, n * 8));
  SB_CUDA(ctx, cudaMalloc(&ctx->roots.volume, n * 8));
  SB_CUDA(ctx, cudaMalloc(&ctx->roots.exc_start, n * 8));
  SB_CUDA(ctx, cudaMalloc(&ctx->roots.exc_stop, n * 8));
  SB_CUDA(ctx, cudaMalloc(&ctx->roots.max_exc_start, n * 8));
  SB_CUDA(ctx, cudaMalloc(&ctx->roots.max_exc_stop, n * 8));
  SB_CUDA(ctx, cudaMalloc(&ctx->roots.prev_overlap, n * 4));
  SB_CUDA(ctx, cudaMalloc(&ctx->root_list, n * 4));
  SB_CUDA(ctx, cudaMalloc(&ctx->lout, sizeof(LabelOut)));
  SB_CUDA(ctx, cudaMallocHost(&ctx->lout_host, sizeof(LabelOut)));
  SB_CUDA(ctx, cudaMalloc(&ctx->forcing, n * 4));
  SB_CUDA(ctx, cudaMalloc(&ctx->m2r, n * 8));
  SB_CUDA(ctx, cudaMemsetAsync(ctx->forcing, 0, n * 4, ctx->stream));
  SB_CUDA(ctx, cudaMemsetAsync(ctx->m2r, 0, n * 8, ctx->stream));
  SB_CUDA(ctx, cudaMalloc(&ctx->surf_before, n * 8));
  SB_CUDA(ctx, cudaMemsetAsync(ctx->surf_before, 0, n * 8, ctx->stream));
  SB_CUDA(ctx, cudaMalloc(&ctx->owned_surface, n * 8));
  SB_CUDA(ctx, cudaMalloc(&ctx->act_count, n * 4));
  SB_CUDA(ctx, cudaMalloc(&ctx->act_first, n * 8));
  SB_CUDA(ctx, cudaMalloc(&ctx->act_last, n * 8));
  SB_CUDA(ctx, cudaMalloc(&ctx->r2m, n * 8));
  {
    void* hist[] = {ctx->owned_surface, ctx->act_first, ctx->act_last, ctx->r2m};
    for (void* p : hist) SB_CUDA(ctx, cudaMemsetAsync(p, 0, n * 8, ctx->stream));
    SB_CUDA(ctx, cudaMemsetAsync(ctx->act_count, 0, n * 4, ctx->stream));
  }
  SB_CUDA(ctx, cudaMalloc(&ctx->initial_b, (size_t)ctx->pitch * d.ny * ctx->esize));
  SB_CUDA(ctx, cudaMemsetAsync(ctx->initial_b, 0, (size_t)ctx->pitch * d.ny * ctx->esize, ctx->stream));
  SB_CUDA(ctx, cudaMalloc(&ctx->mob_out, sizeof(MobilizeOut)));
  SB_CUDA(ctx, cudaMallocHost(&ctx->mob_out_host, sizeof(MobilizeOut)));
  SB_CUDA(ctx, cudaMalloc(&ctx->pers_out, kPersistSlots * sizeof(double)));
  SB_CUDA(ctx, cudaMallocHost(&ctx->pers_out_host, kPersistSlots * sizeof(double)));
  SB_CUDA(ctx, cudaMalloc(&ctx->dep_out, sizeof(DepositionOut)));
  SB_CUDA(ctx, cudaMallocHost(&ctx->dep_out_host, sizeof(DepositionOut)));
  void* zero_init[] = {ctx->parent, ctx->latch, ctx->previous, ctx->export_cum, ctx->export_base};
  size_t zero_size[] = {n * 4, n * 4, n * 4, n * 8, n * 8};
  for (int k = 0; k < 5; ++k) SB_CUDA(ctx, cudaMemsetAsync(zero_init[k], 0, zero_size[k], ctx->stream));
  // relaxation buffers
  SB_CUDA(ctx, cudaMalloc(&ctx->b_alt, field_bytes));
  SB_CUDA(ctx, cudaMemsetAsync(ctx->b_alt, 0, field_bytes, ctx->stream));
  ctx->ftiles0 = (d.ny + d.tile_size - 1) / d.tile_size;
  ctx->ftiles1 = (d.nx + d.tile_size - 1) / d.tile_size;
  {
    // list-driven frontier kernels: eight 256-thread CTAs per SM stride over
    // the active tiles (never more CTAs than tiles)
    int sms = 0;
    SB_CUDA(ctx, cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, d.device));
    ctx->frontier_grid =
        (int)std::min<long long>((long long)ctx->ftiles0 * ctx->ftiles1, 8LL * std::max(sms, 1));
  }
  const size_t nt = (size_t)ctx->ftiles0 * ctx->ftiles1;
  SB_CUDA(ctx, cudaMalloc(&ctx->ptiles, nt * sizeof(int)));
  SB_CUDA(ctx, cudaMalloc(&ctx->dtiles, nt * sizeof(int)));
  SB_CUDA(ctx, cudaMalloc(&ctx->ftile_next, nt * 4));
  SB_CUDA(ctx, cudaMalloc(&ctx->phase[0], nt * 4));
  SB_CUDA(ctx, cudaMalloc(&ctx->phase[1], nt * 4));
  SB_CUDA(ctx, cudaMemsetAsync(ctx->ftile_next, 0, nt * 4, ctx->stream));
  SB_CUDA(ctx, cudaMalloc(&ctx->rctl, sizeof(RelaxControl)));
  SB_CUDA(ctx, cudaMemsetAsync(ctx->rctl, 0, sizeof(RelaxControl), ctx->stream));
  SB_CUDA(ctx, cudaMallocHost(&ctx->rctl_host, sizeof(RelaxControl)));
  SB_CUDA(ctx, cudaMalloc(&ctx->xidx, n * 4));
  SB_CUDA(ctx, cudaMalloc(&ctx->xval, n * 8));
  SB_CUDA(ctx, cudaMalloc(&ctx->xout, sizeof(ExchangeOut)));
  SB_CUDA(ctx, cudaMemsetAsync(ctx->xout, 0, sizeof(ExchangeOut), ctx->stream));  // arrive = 0
  static_assert(offsetof(ExchangeOut, momentum_w) == offsetof(ExchangeOut, volume_w_fp64) + 8,
                "exchange_fold writes volume and momentum sums as one array");
  SB_CUDA(ctx, cudaMalloc(&ctx->xpart, 3 * 148 * 8 * sizeof(double)));
  SB_CUDA(ctx, cudaMallocHost(&ctx->xout_host, sizeof(ExchangeOut)));
  SB_CUDA(ctx, cudaMalloc(&ctx->pstate, sizeof(PathState)));
  SB_CUDA(ctx, cudaMemsetAsync(ctx->pstate, 0, sizeof(PathState), ctx->stream));
  SB_CUDA(ctx, cudaMallocHost(&ctx->pstate_host, sizeof(PathState)));
  SB_CUDA(ctx, cudaMalloc(&ctx->path_count, sizeof(int)));
  SB_CUDA(ctx, cudaHostAlloc(&ctx->path_in, sizeof(PathInput), cudaHostAllocMapped));
  // TMA descriptors (box = halo tile of the FV kernel)
  int rc;
  {
    const CUtensorMapDataType dt =
        fx(ctx) ? CU_TENSOR_MAP_DATA_TYPE_INT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
    if ((rc = encode_2d(ctx, &ctx->tm_relax[0], ctx->b, dt, ctx->esize, kRelaxBox, kRelaxBox)))
      return rc;
    if ((rc = encode_2d(ctx, &ctx->tm_relax[1], ctx->b_alt, dt, ctx->esize, kRelaxBox, kRelaxBox)))
      return rc;
    SB_CUDA(ctx, cudaMalloc(&ctx->reached_alt, (size_t)ctx->pitch * d.ny * sizeof(int32_t)));
    SB_CUDA(ctx, cudaMemsetAsync(ctx->reached_alt, 0, (size_t)ctx->pitch * d.ny * 4, ctx->stream));
    if ((rc = encode_2d(ctx, &ctx->tm_reached[0], ctx->reached, CU_TENSOR_MAP_DATA_TYPE_INT32, 4,
                        kRelaxBox, kRelaxBox)))
      return rc;
    if ((rc = encode_2d(ctx, &ctx->tm_reached[1], ctx->reached_alt, CU_TENSOR_MAP_DATA_TYPE_INT32,
                        4, kRelaxBox, kRelaxBox)))
      return rc;
  }
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
  ctx->relax_full.reset();
  ctx->relax_full2.reset();
  ctx->relax_reached.reset();
  ctx->frontier.reset();
  void* ptrs[] = {ctx->b, ctx->z, ctx->h[0], ctx->h[1], ctx->qx[0], ctx->qx[1], ctx->qy[0],
                  ctx->qy[1], ctx->ext_x, ctx->ext_y, ctx->reached, ctx->staging,
                  ctx->range_error, ctx->ctl, ctx->io, ctx->partials, ctx->ipartials, ctx->fv_diag,
                  ctx->lpart_before, ctx->lipart_before,
                  ctx->arrive, ctx->dt_dev, ctx->parent, ctx->slope, ctx->severity, ctx->latch,
                  ctx->previous, ctx->export_cum, ctx->export_base, ctx->roots.count,
                  ctx->roots.area6, ctx->roots.volume, ctx->roots.exc_start, ctx->roots.exc_stop,
                  ctx->roots.max_exc_start, ctx->roots.max_exc_stop, ctx->roots.prev_overlap,
                  ctx->root_list, ctx->lout, ctx->b_alt, ctx->ftile_next, ctx->phase[0],
                  ctx->phase[1], ctx->rctl, ctx->xidx, ctx->xval, ctx->xout, ctx->xpart, ctx->pstate,
                  ctx->path_count, ctx->forcing, ctx->m2r, ctx->dep_out, ctx->owned_surface,
                  ctx->act_count, ctx->act_first, ctx->act_last, ctx->r2m, ctx->initial_b,
                  ctx->ptiles, ctx->mob_out, ctx->pers_out, ctx->surf_before, ctx->dtiles,
                  ctx->q_rows, ctx->q_cols, ctx->q_out, ctx->reached_alt};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (ctx->lout_host) cudaFreeHost(ctx->lout_host);
  if (ctx->rctl_host) cudaFreeHost(ctx->rctl_host);
  for (cudaEvent_t e : ctx->ev_loop)
    if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : ctx->ev_path)
    if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : ctx->ev_stage)
    if (e) cudaEventDestroy(e);
  if (ctx->xout_host) cudaFreeHost(ctx->xout_host);
  if (ctx->dep_out_host) cudaFreeHost(ctx->dep_out_host);
  if (ctx->mob_out_host) cudaFreeHost(ctx->mob_out_host);
  if (ctx->pers_out_host) cudaFreeHost(ctx->pers_out_host);
  if (ctx->pstate_host) cudaFreeHost(ctx->pstate_host);
  if (ctx->path_in) cudaFreeHost(ctx->path_in);
  if (ctx->path_idx) cudaFreeHost(ctx->path_idx);
  if (ctx->path_val) cudaFreeHost(ctx->path_val);
  if (ctx->path_exec) cudaGraphExecDestroy(ctx->path_exec);
  if (ctx->path_graph) cudaGraphDestroy(ctx->path_graph);
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

}  // extern "C"

// Per-cell float64 records (flat ny*nx, float64 in both precisions).
static double* flat_f64_field(sb_ctx* ctx, int field) {
  switch (field) {
    case SB_FIELD_M2R_CUMULATIVE: return ctx->m2r;
    case SB_FIELD_R2M_CUMULATIVE: return ctx->r2m;
    case SB_FIELD_FIRST_ACTIVATION_TIME: return ctx->act_first;
    case SB_FIELD_LAST_ACTIVATION_TIME: return ctx->act_last;
    case SB_FIELD_OWNED_SURFACE: return ctx->owned_surface;
    case SB_FIELD_OWNED_EXPORT_BASELINE: return ctx->export_base;
    case SB_FIELD_EXPORT_CUMULATIVE: return ctx->export_cum;
    default: return nullptr;
  }
}

extern "C" {

int sb_upload(sb_ctx* ctx, int field, const double* host) {
  if (!ctx || !host) return SB_ERR_BAD_ARG;
  if (double* rec = flat_f64_field(ctx, field)) {  // checkpoint restore of a record
    SB_CUDA(ctx, cudaMemcpyAsync(rec, host, (size_t)ctx->d.ny * ctx->d.nx * 8,
                                 cudaMemcpyHostToDevice, ctx->stream));
    SB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return SB_OK;
  }
  int is_int, is_h, is_s, is_flat;
  void* dst = field_ptr(ctx, field, &is_int, &is_h, &is_s, &is_flat);
  if (!dst || is_int) return fail(ctx, SB_ERR_BAD_ARG, "[soilb200] field %d is not a float field", field);
  if (is_flat) return fail(ctx, SB_ERR_BAD_ARG, "[soilb200] field %d is read-only", field);
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
  if (double* rec = flat_f64_field(ctx, field)) {
    SB_CUDA(ctx, cudaMemcpyAsync(host, rec, (size_t)ctx->d.ny * ctx->d.nx * 8,
                                 cudaMemcpyDeviceToHost, ctx->stream));
    SB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return SB_OK;
  }
  int is_int, is_h, is_s, is_flat;
  void* src = field_ptr(ctx, field, &is_int, &is_h, &is_s, &is_flat);
  if (!src || is_int) return fail(ctx, SB_ERR_BAD_ARG, "[soilb200] field %d is not a float field", field);
  const int ny = ctx->d.ny, nx = ctx->d.nx;
  if (is_flat) {
    if (!fx(ctx)) {
      SB_CUDA(ctx, cudaMemcpyAsync(host, src, (size_t)ny * nx * 8, cudaMemcpyDeviceToHost, ctx->stream));
    } else {
      from_float_kernel<<<grid_for((long long)ny * nx), kThreads, 0, ctx->stream>>>(
          (const float*)src, ctx->staging, ny, nx, nx);
      ctx->launches++;
      SB_CUDA(ctx, cudaGetLastError());
      SB_CUDA(ctx, cudaMemcpyAsync(host, ctx->staging, (size_t)ny * nx * 8, cudaMemcpyDeviceToHost,
                                   ctx->stream));
    }
    SB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return SB_OK;
  }
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
  int is_int, is_h, is_s, is_flat;
  void* dst = field_ptr(ctx, field, &is_int, &is_h, &is_s, &is_flat);
  if (!dst || !is_int) return fail(ctx, SB_ERR_BAD_ARG, "[soilb200] field %d is not an int field", field);
  if (field == SB_FIELD_LABELS)
    return fail(ctx, SB_ERR_BAD_ARG, "[soilb200] labels are read-only");
  if (is_flat) {
    SB_CUDA(ctx, cudaMemcpyAsync(dst, host, (size_t)ctx->d.ny * ctx->d.nx * 4,
                                 cudaMemcpyHostToDevice, ctx->stream));
    SB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return SB_OK;
  }
  SB_CUDA(ctx, cudaMemcpy2DAsync(dst, (size_t)ctx->pitch * 4, host, (size_t)ctx->d.nx * 4,
                                 (size_t)ctx->d.nx * 4, ctx->d.ny, cudaMemcpyHostToDevice,
                                 ctx->stream));
  SB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return SB_OK;
}

int sb_download_i32(sb_ctx* ctx, int field, int32_t* host) {
  if (!ctx || !host) return SB_ERR_BAD_ARG;
  int is_int, is_h, is_s, is_flat;
  void* src = field_ptr(ctx, field, &is_int, &is_h, &is_s, &is_flat);
  if (!src || !is_int) return fail(ctx, SB_ERR_BAD_ARG, "[soilb200] field %d is not an int field", field);
  if (is_flat) {
    SB_CUDA(ctx, cudaMemcpyAsync(host, src, (size_t)ctx->d.ny * ctx->d.nx * 4,
                                 cudaMemcpyDeviceToHost, ctx->stream));
    SB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return SB_OK;
  }
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
  if (ctx->use_graphs && (!mg.valid || std::memcmp(&mg.key, &c, sizeof(FvConst)) != 0 ||
                          mg.static_limit != static_limit)) {
    rc = fx(ctx) ? build_mobile_graph<true>(ctx, c, static_limit)
                 : build_mobile_graph<false>(ctx, c, static_limit);
    if (rc) return rc;
  }
  // the previous call ended synchronised, so the mapped dt is free to rewrite
  *ctx->dt_host = dt_s;
  if (ctx->use_graphs) {
    // the graph reads dt from the mapped pinned copy and writes its records
    // back into mapped pinned memory: no copy-engine operations per step
    SB_CUDA(ctx, cudaGraphLaunch(mg.exec, ctx->stream));
  } else {
    SB_CUDA(ctx, cudaMemcpyAsync(ctx->dt_dev, ctx->dt_host, sizeof(double),
                                 cudaMemcpyHostToDevice, ctx->stream));
    rc = fx(ctx) ? mobile_step_host_loop<true>(ctx, c, static_limit)
                 : mobile_step_host_loop<false>(ctx, c, static_limit);
    if (rc) return rc;
    SB_CUDA(ctx, cudaMemcpyAsync(ctx->ctl_host, ctx->ctl, sizeof(FvControl),
                                 cudaMemcpyDeviceToHost, ctx->stream));
    SB_CUDA(ctx, cudaMemcpyAsync(ctx->io_host, ctx->io, sizeof(StepIO), cudaMemcpyDeviceToHost,
                                 ctx->stream));
  }
  SB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  const FvControl& k = *ctx->ctl_host;
  // graph: begin, two ledgers, records + two substep launches per loop
  // iteration; host loop: begin, two ledgers + one launch per substep; the
  // persistent loop is one launch either way
  const bool pers = fx(ctx) && ctx->fv_stream && ctx->fv_persistent;
  ctx->launches += !ctx->use_graphs ? 3 + (pers ? 1 : k.substeps)
                   : pers           ? 5
                                    : 4 + (k.substeps + 1) / 2 * 2;
  rc = fill_mobile_stats(ctx, params, out);
  if (rc) return rc;
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

// ---------------------------------------------------------------------------
// Labelling
// ---------------------------------------------------------------------------
static LabelConst make_label_const(const sb_ctx* ctx, const sb_label_params* p) {
  LabelConst c{};
  c.ny = ctx->d.ny;
  c.nx = ctx->d.nx;
  c.pitch = ctx->pitch;
  c.tiles_x = (ctx->d.nx + kLabelTile - 1) / kLabelTile;
  c.connectivity = p->connectivity;
  c.dx = ctx->d.dx_m;
  c.dy = ctx->d.dy_m;
  c.tan_start = p->tan_start;
  c.tan_stop = p->tan_stop;
  c.density = p->density_kg_m3;
  c.gravity = p->gravity_m_s2;
  c.cohesion = p->cohesion_pa;
  c.mob_depth = p->mobilization_depth_m;
  c.dry = p->dry_tolerance_m;
  c.activity_speed = p->activity_speed_m_s;
  c.start_rad = p->start_rad;
  c.stop_rad = p->stop_rad;
  c.Q = ctx->quantum;
  c.datum = ctx->d.datum_m;
  c.release_latches = p->release_settled_latches ? 1 : 0;
  c.tile_size = ctx->d.tile_size;
  c.frontier_tiles_x = ctx->ftiles1;
  return c;
}

template <bool FX>
static int run_label(sb_ctx* ctx, const LabelConst& c) {
  using T = FvTypes<FX>;
  const int tiles = c.tiles_x * ((c.ny + kLabelTile - 1) / kLabelTile);
  SB_CUDA(ctx, cudaMemsetAsync(ctx->lout, 0, sizeof(LabelOut), ctx->stream));
  label_init_local_kernel<FX><<<tiles, kLabelInitThreads, 0, ctx->stream>>>(
      c, (const typename T::B*)ctx->b, (const typename T::B*)ctx->z,
      (const typename T::H*)ctx->h[0], (const typename T::H*)ctx->h[1],
      (const typename T::R*)ctx->qx[0], (const typename T::R*)ctx->qx[1],
      (const typename T::R*)ctx->qy[0], (const typename T::R*)ctx->qy[1], ctx->ctl, ctx->parent,
      (typename T::R*)ctx->slope, (typename T::R*)ctx->severity, ctx->latch, ctx->export_cum,
      ctx->export_base, ctx->roots);
  label_merge_kernel<<<tiles, kThreads, 0, ctx->stream>>>(c, ctx->parent, ctx->lout);
  const int g = grid_for((long long)c.ny * c.nx);
  label_compress_kernel<FX><<<g, kThreads, 0, ctx->stream>>>(
      c, ctx->parent, (const typename T::B*)ctx->b, (const typename T::B*)ctx->z,
      (const typename T::R*)ctx->slope, (const typename T::R*)ctx->severity, ctx->latch,
      ctx->previous, ctx->roots, ctx->root_list, ctx->lout, 0);
  label_reduce_kernel<<<32, kThreads, 0, ctx->stream>>>(ctx->roots, ctx->root_list, ctx->lout,
                                                         ctx->arrive);
  ctx->launches += 4;
  SB_CUDA(ctx, cudaGetLastError());
  SB_CUDA(ctx, cudaMemcpyAsync(ctx->lout_host, ctx->lout, sizeof(LabelOut), cudaMemcpyDeviceToHost,
                               ctx->stream));
  SB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return SB_OK;
}

extern "C" int sb_label(sb_ctx* ctx, const sb_label_params* p, sb_label_stats* out) {
  if (!ctx || !p || !out) return SB_ERR_BAD_ARG;
  if (p->connectivity != 4 && p->connectivity != 8)
    return fail(ctx, SB_ERR_BAD_ARG, "[LargeAvalanche] connectivity must be 4 or 8");
  if ((long long)ctx->d.ny * ctx->d.nx >= 0x7fffffffLL)
    return fail(ctx, SB_ERR_BAD_ARG, "[soilb200] grid too large for int32 labels");
  const LabelConst c = make_label_const(ctx, p);
  int rc = fx(ctx) ? run_label<true>(ctx, c) : run_label<false>(ctx, c);
  if (rc) return rc;
  const LabelOut& o = *ctx->lout_host;
  std::memset(out, 0, sizeof(*out));
  out->status = o.status;
  out->unstable_cell_count = o.total_unstable;
  out->connected_region_count = o.regions;
  out->largest_connected_cell_count = o.largest;
  out->winner_root = o.winner;
  out->union_passes = 2;
  out->previous_overlap = o.prev_overlap;
  const double f = ctx->d.dx_m * ctx->d.dy_m / 6.0;
  out->largest_connected_area_m2 = (double)o.area6 * f;
  out->largest_connected_mobilizable_volume_m3 =
      fx(ctx) ? (double)o.volume * ctx->quantum * f : (double)o.volume / kVolumeScaleFp64 * f;
  out->excess_start_sum_rad = (double)o.exc_start / kExcessScale;
  out->excess_start_max_rad = (double)o.max_exc_start / kExcessScale;
  out->excess_stop_sum_rad = (double)o.exc_stop / kExcessScale;
  out->excess_stop_max_rad = (double)o.max_exc_stop / kExcessScale;
  if (o.status)
    return fail(ctx, SB_ERR_NONCONVERGENCE,
                "NUMERICAL_NONCONVERGENCE: device avalanche connected components");
  return SB_OK;
}

extern "C" int sb_label_mask(sb_ctx* ctx, const int32_t* mask, int connectivity,
                             sb_label_stats* out) {
  if (!ctx || !mask || !out) return SB_ERR_BAD_ARG;
  if (connectivity != 4 && connectivity != 8)
    return fail(ctx, SB_ERR_BAD_ARG, "[LargeAvalanche] connectivity must be 4 or 8");
  LabelConst c{};
  c.ny = ctx->d.ny;
  c.nx = ctx->d.nx;
  c.pitch = ctx->pitch;
  c.tiles_x = (ctx->d.nx + kLabelTile - 1) / kLabelTile;
  c.connectivity = connectivity;
  const size_t n = (size_t)c.ny * c.nx;
  int32_t* dmask = (int32_t*)ctx->staging;  // 8*n bytes of scratch >= 4*n
  SB_CUDA(ctx, cudaMemcpyAsync(dmask, mask, n * 4, cudaMemcpyHostToDevice, ctx->stream));
  SB_CUDA(ctx, cudaMemsetAsync(ctx->lout, 0, sizeof(LabelOut), ctx->stream));
  const int tiles = c.tiles_x * ((c.ny + kLabelTile - 1) / kLabelTile);
  label_mask_local_kernel<<<tiles, kThreads, 0, ctx->stream>>>(c, dmask, ctx->parent, ctx->roots);
  label_merge_kernel<<<tiles, kThreads, 0, ctx->stream>>>(c, ctx->parent, ctx->lout);
  const int g = grid_for((long long)n);
  if (fx(ctx))
    label_compress_kernel<true><<<g, kThreads, 0, ctx->stream>>>(
        c, ctx->parent, nullptr, nullptr, nullptr, nullptr, ctx->latch, ctx->previous, ctx->roots,
        ctx->root_list, ctx->lout, 1);
  else
    label_compress_kernel<false><<<g, kThreads, 0, ctx->stream>>>(
        c, ctx->parent, nullptr, nullptr, nullptr, nullptr, ctx->latch, ctx->previous, ctx->roots,
        ctx->root_list, ctx->lout, 1);
  label_reduce_kernel<<<32, kThreads, 0, ctx->stream>>>(ctx->roots, ctx->root_list, ctx->lout,
                                                         ctx->arrive);
  ctx->launches += 4;
  SB_CUDA(ctx, cudaGetLastError());
  SB_CUDA(ctx, cudaMemcpyAsync(ctx->lout_host, ctx->lout, sizeof(LabelOut), cudaMemcpyDeviceToHost,
                               ctx->stream));
  SB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  const LabelOut& o = *ctx->lout_host;
  std::memset(out, 0, sizeof(*out));
  out->status = o.status;
  out->unstable_cell_count = o.total_unstable;
  out->connected_region_count = o.regions;
  out->largest_connected_cell_count = o.largest;
  out->winner_root = o.winner;
  out->union_passes = 2;
  out->largest_connected_area_m2 = (double)o.area6 * (ctx->d.dx_m * ctx->d.dy_m / 6.0);
  if (o.status)
    return fail(ctx, SB_ERR_NONCONVERGENCE,
                "NUMERICAL_NONCONVERGENCE: device avalanche connected components");
  return SB_OK;
}

extern "C" int sb_label_commit(sb_ctx* ctx, int keep_candidate, int seed_frontier) {
  if (!ctx) return SB_ERR_BAD_ARG;
  LabelConst c{};
  c.ny = ctx->d.ny;
  c.nx = ctx->d.nx;
  c.pitch = ctx->pitch;
  c.tile_size = ctx->d.tile_size;
  c.frontier_tiles_x = ctx->ftiles1;
  label_update_previous_kernel<<<grid_for((long long)c.ny * c.nx), kThreads, 0, ctx->stream>>>(
      c, ctx->parent, ctx->previous, ctx->reached, ctx->ftile_next, ctx->lout,
      keep_candidate ? 1 : 0, seed_frontier ? 1 : 0);
  ctx->launches++;
  SB_CUDA(ctx, cudaGetLastError());
  SB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return SB_OK;
}

// ---------------------------------------------------------------------------
// Relaxation
// ---------------------------------------------------------------------------
static int relax_const(sb_ctx* ctx, const sb_relax_params* p, RelaxConst* c, int tile) {
  if (!(p->spacing0_m > 0) || !(p->spacing1_m > 0) || !std::isfinite(p->spacing0_m) ||
      !std::isfinite(p->spacing1_m))
    return fail(ctx, SB_ERR_BAD_ARG, "grid spacing must be positive");
  if (!(p->critical_slope > 0) || !std::isfinite(p->critical_slope))
    return fail(ctx, SB_ERR_BAD_ARG, "critical slope must be finite/positive");
  if (!(p->tolerance_m >= 0) || p->max_iterations < 1)
    return fail(ctx, SB_ERR_BAD_ARG, "tolerance/max_iterations invalid");
  std::memset(c, 0, sizeof(*c));
  c->n0 = ctx->d.ny;
  c->n1 = ctx->d.nx;
  c->pitch = ctx->pitch;
  c->tiles1 = (ctx->d.nx + tile - 1) / tile;
  c->ntiles = c->tiles1 * ((ctx->d.ny + tile - 1) / tile);
  c->s0 = p->spacing0_m;
  c->s1 = p->spacing1_m;
  const double diag = std::hypot(p->spacing0_m, p->spacing1_m);
  const double dist[4] = {p->spacing0_m, p->spacing1_m, diag, diag};
  for (int k = 0; k < 4; ++k) {
    c->crit[k] = p->critical_slope * dist[k];
    c->crit_q[k] = c->crit[k] / ctx->quantum;
  }
  c->tol = p->tolerance_m;
  c->tol_q = p->tolerance_m / ctx->quantum;
  c->max_iterations = p->max_iterations;
  c->weighted = p->weighted ? 1 : 0;
  c->ftile = tile;
  c->f = p->spacing0_m * p->spacing1_m / 6.0;
  if (fx(ctx)) {
    // the rounded-up transfer rule needs crit*L >= 8 quanta (no overshoot past level)
    for (int k = 0; k < 2; ++k)
      if (c->crit_q[k] < 8.0)
        return fail(ctx, SB_ERR_BAD_ARG,
                    "[soilb200] critical height difference below 8 quanta; use a finer quantum");
  }
  return SB_OK;
}

__global__ void relax_reset_kernel(RelaxControl* ctl) {
  if (threadIdx.x == 0) {
    ctl->confirm = 0;
    ctl->bb[0] = INT_MAX;
    ctl->bb[1] = INT_MIN;
    ctl->bb[2] = INT_MAX;
    ctl->bb[3] = INT_MIN;
    ctl->iterations = 0;
    ctl->done = 0;
    ctl->converged = 0;
    ctl->status = 0;
    ctl->max_excess_bits = 0;
    ctl->arrive = 0;
    ctl->parity = 0;
    ctl->n_active = 0;
    ctl->rounds = 0;
    ctl->moved_edges = 0;
    ctl->list_len = 0;
    ctl->sub_len = 0;
  }
}

template <bool FX>
static int build_relax_full(sb_ctx* ctx, const RelaxConst& c, LoopGraph& lg) {
  lg.reset();
  cudaGraph_t g;
  SB_CUDA(ctx, cudaGraphCreate(&g, 0));
  lg.graph = g;
  cudaGraphConditionalHandle handle;
  SB_CUDA(ctx, cudaGraphConditionalHandleCreate(&handle, g, 1, cudaGraphCondAssignDefault));
  cudaGraphNode_t n_reset, n_loop, n_body;
  {
    void* args[] = {(void*)&ctx->rctl};
    int rc = add_kernel(ctx, g, &n_reset, nullptr, 0, (void*)relax_reset_kernel, dim3(1), 0, args);
    if (rc) return rc;
  }
  cudaGraphNodeParams cp{};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = handle;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  SB_CUDA(ctx, cudaGraphAddNode(&n_loop, g, &n_reset, 1, &cp));
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  RelaxConst cc = c;
  int use_handle = 1;
  const int tiles1 = (c.n1 + kRelaxTile - 1) / kRelaxTile;
  const int tiles0 = (c.n0 + kRelaxTile - 1) / kRelaxTile;
  RelaxConst ck = cc;
  ck.tiles1 = tiles1;
  void* args[] = {(void*)&ck, (void*)&ctx->tm_relax[0], (void*)&ctx->tm_relax[1],
                  (void*)&ctx->b, (void*)&ctx->b_alt, (void*)&ctx->rctl, (void*)&handle,
                  (void*)&use_handle};
  int rc = add_kernel(ctx, body, &n_body, nullptr, 0, (void*)relax_full_kernel<FX>,
                      dim3(tiles0 * tiles1), 0, args);
  if (rc) return rc;
  // leave the result in b_eff whichever ping-pong buffer it ended in
  cudaGraphNode_t n_copy, n_par;
  {
    long long count = (long long)ctx->pitch * ctx->d.ny;
    void* cargs[] = {(void*)&ctx->b_alt, (void*)&ctx->b, (void*)&count, (void*)&ctx->rctl};
    if ((rc = add_kernel(ctx, g, &n_copy, &n_loop, 1, (void*)relax_copyback_kernel<FX>,
                         dim3(grid_for(count)), 0, cargs)))
      return rc;
    void* pargs[] = {(void*)&ctx->rctl};
    if ((rc = add_kernel(ctx, g, &n_par, &n_copy, 1, (void*)relax_parity_clear_kernel, dim3(1), 0,
                         pargs)))
      return rc;
  }
  SB_CUDA(ctx, cudaGraphInstantiate(&lg.exec, g, 0));
  lg.key = c;
  lg.valid = true;
  return SB_OK;
}

// Cached graph for these parameters (two slots, least recently used replaced).
static int relax_graph_for(sb_ctx* ctx, const RelaxConst& c, LoopGraph** out) {
  LoopGraph* slots[2] = {&ctx->relax_full, &ctx->relax_full2};
  for (int i = 0; i < 2; ++i)
    if (slots[i]->valid && std::memcmp(&slots[i]->key, &c, sizeof(RelaxConst)) == 0) {
      ctx->relax_lru = i ^ 1;
      *out = slots[i];
      return SB_OK;
    }
  const int victim = ctx->relax_lru;
  const int rc = fx(ctx) ? build_relax_full<true>(ctx, c, *slots[victim])
                         : build_relax_full<false>(ctx, c, *slots[victim]);
  if (rc) return rc;
  ctx->relax_lru = victim ^ 1;
  *out = slots[victim];
  return SB_OK;
}

// SOILB200_NO_GRAPH=1 (profilers that cannot see kernel nodes of a graph
// with conditional nodes): the sweep graph's kernels launched from the host,
// the loop flag read back after every sweep.
template <bool FX>
static int relax_full_host_loop(sb_ctx* ctx, const RelaxConst& c) {
  void* rargs[] = {(void*)&ctx->rctl};
  SB_CUDA(ctx, cudaLaunchKernel((void*)relax_reset_kernel, dim3(1), dim3(kThreads), rargs, 0,
                                ctx->stream));
  RelaxConst ck = c;
  ck.tiles1 = (c.n1 + kRelaxTile - 1) / kRelaxTile;
  const int tiles0 = (c.n0 + kRelaxTile - 1) / kRelaxTile;
  cudaGraphConditionalHandle handle{};
  int no_handle = 0;
  void* args[] = {(void*)&ck, (void*)&ctx->tm_relax[0], (void*)&ctx->tm_relax[1],
                  (void*)&ctx->b, (void*)&ctx->b_alt, (void*)&ctx->rctl, (void*)&handle,
                  (void*)&no_handle};
  for (long long it = 0; it <= (long long)c.max_iterations; ++it) {
    SB_CUDA(ctx, cudaLaunchKernel((void*)relax_full_kernel<FX>, dim3(tiles0 * ck.tiles1),
                                  dim3(kThreads), args, 0, ctx->stream));
    SB_CUDA(ctx, cudaMemcpyAsync(ctx->rctl_host, ctx->rctl, sizeof(RelaxControl),
                                 cudaMemcpyDeviceToHost, ctx->stream));
    SB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (ctx->rctl_host->done) break;
  }
  long long count = (long long)ctx->pitch * ctx->d.ny;
  void* cargs[] = {(void*)&ctx->b_alt, (void*)&ctx->b, (void*)&count, (void*)&ctx->rctl};
  SB_CUDA(ctx, cudaLaunchKernel((void*)relax_copyback_kernel<FX>, dim3(grid_for(count)),
                                dim3(kThreads), cargs, 0, ctx->stream));
  SB_CUDA(ctx, cudaLaunchKernel((void*)relax_parity_clear_kernel, dim3(1), dim3(kThreads), rargs,
                                0, ctx->stream));
  return SB_OK;
}

// Queues max_iterations (or fewer, if converged) sweeps without waiting for
// them or reading their statistics back.
extern "C" int sb_relax_sweeps(sb_ctx* ctx, const sb_relax_params* p) {
  if (!ctx || !p) return SB_ERR_BAD_ARG;
  RelaxConst c;
  int rc = relax_const(ctx, p, &c, kRelaxTile);
  if (rc) return rc;
  if (!ctx->use_graphs) {
    rc = fx(ctx) ? relax_full_host_loop<true>(ctx, c) : relax_full_host_loop<false>(ctx, c);
    ctx->launches += 3 + ctx->rctl_host->iterations;
    return rc;
  }
  LoopGraph* lg = nullptr;
  if ((rc = relax_graph_for(ctx, c, &lg))) return rc;
  SB_CUDA(ctx, cudaGraphLaunch(lg->exec, ctx->stream));
  ctx->launches += 3;
  return SB_OK;
}

extern "C" int sb_relax_full(sb_ctx* ctx, const sb_relax_params* p, sb_relax_stats* out) {
  if (!ctx || !p || !out) return SB_ERR_BAD_ARG;
  RelaxConst c;
  int rc = relax_const(ctx, p, &c, kRelaxTile);
  if (rc) return rc;
  if (!ctx->use_graphs) {
    rc = fx(ctx) ? relax_full_host_loop<true>(ctx, c) : relax_full_host_loop<false>(ctx, c);
    if (rc) return rc;
  } else {
    LoopGraph* lg = nullptr;
    if ((rc = relax_graph_for(ctx, c, &lg))) return rc;
    SB_CUDA(ctx, cudaGraphLaunch(lg->exec, ctx->stream));
  }
  SB_CUDA(ctx, cudaMemcpyAsync(ctx->rctl_host, ctx->rctl, sizeof(RelaxControl),
                               cudaMemcpyDeviceToHost, ctx->stream));
  SB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  const RelaxControl& k = *ctx->rctl_host;
  ctx->launches += 3 + k.iterations;
  std::memset(out, 0, sizeof(*out));
  out->iterations = k.iterations;
  out->converged = k.converged;
  out->status = k.status;
  if (k.status == SB_ERR_WAIT_LIMIT)
    return fail(ctx, SB_ERR_WAIT_LIMIT, "[soilb200] a bounded device wait gave up (TMA tile load)");
  return SB_OK;
}

// Reached-gated sweep graph: reset + begin (equal ping-pong buffers, seed
// bounding box), a WHILE loop over relax_reached_kernel (iterations and
// confirming scans), then heights and reached mask back into b_eff /
// frontier_reached.
template <bool FX>
static int build_relax_reached(sb_ctx* ctx, const RelaxConst& c, LoopGraph& lg) {
  lg.reset();
  cudaGraph_t g;
  SB_CUDA(ctx, cudaGraphCreate(&g, 0));
  lg.graph = g;
  cudaGraphConditionalHandle handle;
  SB_CUDA(ctx, cudaGraphConditionalHandleCreate(&handle, g, 1, cudaGraphCondAssignDefault));
  cudaGraphNode_t n_reset, n_begin, n_loop, n_body;
  int rc;
  {
    void* args[] = {(void*)&ctx->rctl};
    if ((rc = add_kernel(ctx, g, &n_reset, nullptr, 0, (void*)relax_reset_kernel, dim3(1), 0,
                         args)))
      return rc;
  }
  RelaxConst ck = c;
  ck.tiles1 = (c.n1 + kRelaxTile - 1) / kRelaxTile;
  const int tiles0 = (c.n0 + kRelaxTile - 1) / kRelaxTile;
  {
    void* args[] = {(void*)&ck, (void*)&ctx->b, (void*)&ctx->b_alt, (void*)&ctx->reached,
                    (void*)&ctx->reached_alt, (void*)&ctx->rctl};
    if ((rc = add_kernel(ctx, g, &n_begin, &n_reset, 1, (void*)relax_reached_begin_kernel<FX>,
                         dim3(grid_for((long long)c.n0 * c.n1)), 0, args)))
      return rc;
  }
  cudaGraphNodeParams cp{};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = handle;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  SB_CUDA(ctx, cudaGraphAddNode(&n_loop, g, &n_begin, 1, &cp));
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  int use_handle = 1;
  {
    void* args[] = {(void*)&ck, (void*)&ctx->tm_relax[0], (void*)&ctx->tm_relax[1],
                    (void*)&ctx->tm_reached[0], (void*)&ctx->tm_reached[1], (void*)&ctx->b,
                    (void*)&ctx->b_alt, (void*)&ctx->reached, (void*)&ctx->reached_alt,
                    (void*)&ctx->rctl, (void*)&handle, (void*)&use_handle};
    if ((rc = add_kernel(ctx, body, &n_body, nullptr, 0, (void*)relax_reached_kernel<FX>,
                         dim3(tiles0 * ck.tiles1), 0, args)))
      return rc;
  }
  cudaGraphNode_t n_copy, n_rcopy, n_par;
  long long count = (long long)ctx->pitch * ctx->d.ny;
  {
    void* cargs[] = {(void*)&ctx->b_alt, (void*)&ctx->b, (void*)&count, (void*)&ctx->rctl};
    if ((rc = add_kernel(ctx, g, &n_copy, &n_loop, 1, (void*)relax_copyback_kernel<FX>,
                         dim3(grid_for(count)), 0, cargs)))
      return rc;
  }
  {
    void* cargs[] = {(void*)&ctx->reached_alt, (void*)&ctx->reached, (void*)&count,
                     (void*)&ctx->rctl};
    if ((rc = add_kernel(ctx, g, &n_rcopy, &n_copy, 1, (void*)reached_copyback_kernel,
                         dim3(grid_for(count)), 0, cargs)))
      return rc;
  }
  {
    void* pargs[] = {(void*)&ctx->rctl};
    if ((rc = add_kernel(ctx, g, &n_par, &n_rcopy, 1, (void*)relax_parity_clear_kernel, dim3(1),
                         0, pargs)))
      return rc;
  }
  SB_CUDA(ctx, cudaGraphInstantiate(&lg.exec, g, 0));
  lg.key = c;
  lg.valid = true;
  return SB_OK;
}

extern "C" int sb_relax_reached(sb_ctx* ctx, const sb_relax_params* p, sb_relax_stats* out) {
  if (!ctx || !p || !out) return SB_ERR_BAD_ARG;
  RelaxConst c;
  int rc = relax_const(ctx, p, &c, kRelaxTile);
  if (rc) return rc;
  LoopGraph& lg = ctx->relax_reached;
  if (!lg.valid || std::memcmp(&lg.key, &c, sizeof(RelaxConst)) != 0) {
    rc = fx(ctx) ? build_relax_reached<true>(ctx, c, lg) : build_relax_reached<false>(ctx, c, lg);
    if (rc) return rc;
  }
  SB_CUDA(ctx, cudaGraphLaunch(lg.exec, ctx->stream));
  SB_CUDA(ctx, cudaMemcpyAsync(ctx->rctl_host, ctx->rctl, sizeof(RelaxControl),
                               cudaMemcpyDeviceToHost, ctx->stream));
  SB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  const RelaxControl& k = *ctx->rctl_host;
  ctx->launches += 5 + k.iterations;
  std::memset(out, 0, sizeof(*out));
  out->iterations = k.iterations;
  out->converged = k.converged;
  out->status = k.status;
  if (k.status == SB_ERR_WAIT_LIMIT)
    return fail(ctx, SB_ERR_WAIT_LIMIT, "[soilb200] a bounded device wait gave up (TMA tile load)");
  if (k.status == SB_ERR_NONCONVERGENCE)
    return fail(ctx, SB_ERR_NONCONVERGENCE,
                "NUMERICAL_NONCONVERGENCE: reached-bbox MiniSlope exceeded the numerical safety "
                "limit");
  return SB_OK;
}

__global__ void frontier_seed_cells_kernel(const int32_t* __restrict__ idx, int count, int ny,
                                           int nx, int pitch, int tile, int tiles1,
                                           int* __restrict__ reached, int* __restrict__ flags,
                                           int* bad) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x) {
    const int i = idx[k];
    if (i < 0 || i >= ny * nx) {
      atomicExch(bad, 1);
      continue;
    }
    const int r = i / nx, c = i % nx;
    reached[(size_t)r * pitch + c] = 1;
    for (int o0 = -1; o0 <= 1; ++o0)
      for (int o1 = -1; o1 <= 1; ++o1) {
        const int q0 = r + o0, q1 = c + o1;
        if (q0 < 0 || q1 < 0 || q0 >= ny || q1 >= nx) continue;
        flags[(q0 / tile) * tiles1 + q1 / tile] = 1;
      }
  }
}

__global__ void frontier_seed_tiles_kernel(const int32_t* __restrict__ ids, int count, int ntiles,
                                           int* __restrict__ flags, int* bad) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x) {
    const int t = ids[k];
    if (t < 0 || t >= ntiles) {
      atomicExch(bad, 1);
      continue;
    }
    flags[t] = 1;
  }
}

static int upload_ints(sb_ctx* ctx, const int32_t* host, int count) {
  // staging holds ny*nx doubles = 2*ny*nx int32 >= count for any valid request
  if ((long long)count > 2LL * ctx->d.ny * ctx->d.nx)
    return fail(ctx, SB_ERR_BAD_ARG, "[soilb200] seed list longer than the grid");
  SB_CUDA(ctx, cudaMemcpyAsync(ctx->staging, host, (size_t)count * 4, cudaMemcpyHostToDevice,
                               ctx->stream));
  SB_CUDA(ctx, cudaMemsetAsync(ctx->range_error, 0, sizeof(int), ctx->stream));
  return SB_OK;
}

static int check_bad(sb_ctx* ctx, const char* what) {
  int herr = 0;
  SB_CUDA(ctx, cudaGetLastError());
  SB_CUDA(ctx, cudaMemcpyAsync(&herr, ctx->range_error, sizeof(int), cudaMemcpyDeviceToHost,
                               ctx->stream));
  SB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (herr) return fail(ctx, SB_ERR_BAD_ARG, "[soilb200] %s index outside state", what);
  return SB_OK;
}

extern "C" int sb_frontier_seed_cells(sb_ctx* ctx, const int32_t* flat, int count) {
  if (!ctx || (!flat && count)) return SB_ERR_BAD_ARG;
  if (count <= 0) return SB_OK;
  int rc = upload_ints(ctx, flat, count);
  if (rc) return rc;
  frontier_seed_cells_kernel<<<grid_for(count), kThreads, 0, ctx->stream>>>(
      (const int32_t*)ctx->staging, count, ctx->d.ny, ctx->d.nx, ctx->pitch, ctx->d.tile_size,
      ctx->ftiles1, ctx->reached, ctx->ftile_next, ctx->range_error);
  ctx->launches++;
  return check_bad(ctx, "frontier seed");
}

extern "C" int sb_frontier_seed_tiles(sb_ctx* ctx, const int32_t* ids, int count) {
  if (!ctx || (!ids && count)) return SB_ERR_BAD_ARG;
  if (count <= 0) return SB_OK;
  int rc = upload_ints(ctx, ids, count);
  if (rc) return rc;
  frontier_seed_tiles_kernel<<<grid_for(count), kThreads, 0, ctx->stream>>>(
      (const int32_t*)ctx->staging, count, ctx->ftiles0 * ctx->ftiles1, ctx->ftile_next,
      ctx->range_error);
  ctx->launches++;
  return check_bad(ctx, "frontier tile");
}

extern "C" int sb_frontier_tile_count(sb_ctx* ctx) { return ctx ? ctx->ftiles0 * ctx->ftiles1 : 0; }

extern "C" int sb_frontier_active_tiles(sb_ctx* ctx, int32_t* flags, int capacity) {
  if (!ctx || !flags) return SB_ERR_BAD_ARG;
  const int nt = ctx->ftiles0 * ctx->ftiles1;
  if (capacity < nt) return fail(ctx, SB_ERR_BAD_ARG, "[soilb200] tile flag buffer too small");
  SB_CUDA(ctx, cudaMemcpyAsync(flags, ctx->ftile_next, (size_t)nt * 4, cudaMemcpyDeviceToHost,
                               ctx->stream));
  SB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return SB_OK;
}

template <bool FX>
static int build_frontier(sb_ctx* ctx, const RelaxConst& c) {
  LoopGraph& lg = ctx->frontier;
  lg.reset();
  cudaGraph_t g;
  SB_CUDA(ctx, cudaGraphCreate(&g, 0));
  lg.graph = g;
  cudaGraphConditionalHandle handle;
  SB_CUDA(ctx, cudaGraphConditionalHandleCreate(&handle, g, 0, cudaGraphCondAssignDefault));
  RelaxConst cc;  // copied into the node parameters at add time
  cc = c;
  cudaGraphNode_t n_reset, n_begin0, n_loop, n_finish;
  int rc;
  {
    void* args[] = {(void*)&ctx->rctl};
    if ((rc = add_kernel(ctx, g, &n_reset, nullptr, 0, (void*)relax_reset_kernel, dim3(1), 0, args)))
      return rc;
  }
  void* begin_args[] = {(void*)&cc, (void*)&ctx->ftile_next, (void*)&ctx->phase[0],
                        (void*)&ctx->phase[1], (void*)&ctx->rctl, (void*)&handle};
  if ((rc = add_kernel(ctx, g, &n_begin0, &n_reset, 1, (void*)frontier_begin_kernel, dim3(1), 0,
                       begin_args)))
    return rc;
  cudaGraphNodeParams cp{};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = handle;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  SB_CUDA(ctx, cudaGraphAddNode(&n_loop, g, &n_begin0, 1, &cp));
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  cudaGraphNode_t prev = nullptr;
  int dirs[8], pars[8];
  for (int k = 0; k < 8; ++k) {
    dirs[k] = k / 2;
    pars[k] = k % 2;
  }
  typename FvTypes<FX>::H* hf = (typename FvTypes<FX>::H*)ctx->b;
  for (int k = 0; k < 8; ++k) {
    cudaGraphNode_t node;
    void* args[] = {(void*)&cc, (void*)&dirs[k], (void*)&pars[k], (void*)&hf,
                    (void*)&ctx->reached, (void*)&ctx->phase[0], (void*)&ctx->phase[1],
                    (void*)&ctx->rctl};
    if ((rc = add_kernel(ctx, body, &node, prev ? &prev : nullptr, prev ? 1 : 0,
                         (void*)frontier_subphase_kernel<FX>, dim3(ctx->frontier_grid), 0,
                         args)))
      return rc;
    prev = node;
  }
  cudaGraphNode_t n_scan, n_begin;
  {
    void* args[] = {(void*)&cc, (void*)&hf, (void*)&ctx->reached, (void*)&ctx->phase[1],
                    (void*)&ctx->ftile_next, (void*)&ctx->rctl};
    if ((rc = add_kernel(ctx, body, &n_scan, &prev, 1, (void*)frontier_scan_kernel<FX>,
                         dim3(ctx->frontier_grid), 0, args)))
      return rc;
  }
  if ((rc = add_kernel(ctx, body, &n_begin, &n_scan, 1, (void*)frontier_begin_kernel, dim3(1), 0,
                       begin_args)))
    return rc;
  {
    void* args[] = {(void*)&cc, (void*)&ctx->reached, (void*)&ctx->rctl};
    if ((rc = add_kernel(ctx, g, &n_finish, &n_loop, 1, (void*)frontier_finish_kernel,
                         dim3(grid_for((long long)c.n0 * c.pitch)), 0, args)))
      return rc;
  }
  SB_CUDA(ctx, cudaGraphInstantiate(&lg.exec, g, 0));
  lg.key = c;
  lg.valid = true;
  return SB_OK;
}

extern "C" int sb_frontier_run(sb_ctx* ctx, const sb_relax_params* p, sb_relax_stats* out) {
  if (!ctx || !p || !out) return SB_ERR_BAD_ARG;
  RelaxConst c;
  int rc = relax_const(ctx, p, &c, ctx->d.tile_size);
  if (rc) return rc;
  LoopGraph& lg = ctx->frontier;
  if (!lg.valid || std::memcmp(&lg.key, &c, sizeof(RelaxConst)) != 0) {
    rc = fx(ctx) ? build_frontier<true>(ctx, c) : build_frontier<false>(ctx, c);
    if (rc) return rc;
  }
  SB_CUDA(ctx, cudaGraphLaunch(lg.exec, ctx->stream));
  SB_CUDA(ctx, cudaMemcpyAsync(ctx->rctl_host, ctx->rctl, sizeof(RelaxControl),
                               cudaMemcpyDeviceToHost, ctx->stream));
  SB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  const RelaxControl& k = *ctx->rctl_host;
  ctx->launches += 3 + 10LL * k.rounds;
  std::memset(out, 0, sizeof(*out));
  out->iterations = k.rounds;
  out->converged = k.converged;
  out->status = k.status;
  out->active_tiles = k.n_active;
  out->moved_edges = k.moved_edges;
  if (k.status == SB_ERR_NONCONVERGENCE)
    return fail(ctx, SB_ERR_NONCONVERGENCE,
                "NUMERICAL_NONCONVERGENCE: GPU residual MiniSlope exceeded the numerical safety limit");
  return SB_OK;
}

extern "C" int sb_field_stats(sb_ctx* ctx, int field, double spacing0, double spacing1,
                              double* out4) {
  if (!ctx || !out4) return SB_ERR_BAD_ARG;
  if (field != SB_FIELD_B_EFF && field != SB_FIELD_Z_BASE)
    return fail(ctx, SB_ERR_BAD_ARG, "[soilb200] field statistics support b_eff / z_base");
  void* f = field == SB_FIELD_B_EFF ? ctx->b : ctx->z;
  const int g = ctx->ledger_blocks;
  double* dout = (double*)ctx->staging;  // 4 doubles of scratch
  if (fx(ctx))
    field_stats_kernel<true><<<g, kThreads, 0, ctx->stream>>>(
        ctx->d.ny, ctx->d.nx, ctx->pitch, spacing0, spacing1, ctx->quantum, ctx->d.datum_m,
        (const int32_t*)f, ctx->partials, ctx->ipartials, ctx->arrive, dout);
  else
    field_stats_kernel<false><<<g, kThreads, 0, ctx->stream>>>(
        ctx->d.ny, ctx->d.nx, ctx->pitch, spacing0, spacing1, ctx->quantum, ctx->d.datum_m,
        (const double*)f, ctx->partials, ctx->ipartials, ctx->arrive, dout);
  ctx->launches++;
  SB_CUDA(ctx, cudaGetLastError());
  SB_CUDA(ctx, cudaMemcpyAsync(out4, dout, 4 * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  SB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return SB_OK;
}

// ---------------------------------------------------------------------------
// Resting <-> Mobile exchange
// ---------------------------------------------------------------------------
static int exchange_upload(sb_ctx* ctx, const int32_t* idx, const double* val, int count) {
  if (count < 0 || (long long)count > (long long)ctx->d.ny * ctx->d.nx)
    return fail(ctx, SB_ERR_BAD_ARG, "[DeviceBulkState] invalid exchange request size");
  for (int k = 0; k < count; ++k)
    if (!std::isfinite(val[k]))
      return fail(ctx, SB_ERR_BAD_ARG, "[DeviceBulkState] invalid exchange request");
  SB_CUDA(ctx, cudaMemcpyAsync(ctx->xidx, idx, (size_t)count * 4, cudaMemcpyHostToDevice, ctx->stream));
  SB_CUDA(ctx, cudaMemcpyAsync(ctx->xval, val, (size_t)count * 8, cudaMemcpyHostToDevice, ctx->stream));
  SB_CUDA(ctx, cudaMemsetAsync(ctx->xout, 0, sizeof(ExchangeOut), ctx->stream));
  return SB_OK;
}

static int exchange_finish(sb_ctx* ctx) {
  SB_CUDA(ctx, cudaGetLastError());
  SB_CUDA(ctx, cudaMemcpyAsync(ctx->xout_host, ctx->xout, sizeof(ExchangeOut),
                               cudaMemcpyDeviceToHost, ctx->stream));
  SB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (ctx->xout_host->bad_index)
    return fail(ctx, SB_ERR_BAD_ARG, "[DeviceBulkState] exchange index outside state");
  return SB_OK;
}

static int entrain_common(sb_ctx* ctx, const int32_t* idx, const double* val, int count, int mode,
                          double* volume_m3) {
  if (!ctx || (count > 0 && (!idx || !val))) return SB_ERR_BAD_ARG;
  if (volume_m3) *volume_m3 = 0.0;
  if (count == 0) return SB_OK;
  int rc = exchange_upload(ctx, idx, val, count);
  if (rc) return rc;
  const int P = ctx->parity_host;
  const double f = ctx->d.dx_m * ctx->d.dy_m / 6.0;
  if (fx(ctx))
    entrain_kernel<true><<<grid_for(count), kThreads, 0, ctx->stream>>>(
        ctx->d.ny, ctx->d.nx, ctx->pitch, ctx->quantum, ctx->d.datum_m, f, (int32_t*)ctx->b,
        (const int32_t*)ctx->z, (int32_t*)ctx->h[P], ctx->xidx, ctx->xval, count, mode, ctx->xout,
        ctx->xpart);
  else
    entrain_kernel<false><<<grid_for(count), kThreads, 0, ctx->stream>>>(
        ctx->d.ny, ctx->d.nx, ctx->pitch, ctx->quantum, ctx->d.datum_m, f, (double*)ctx->b,
        (const double*)ctx->z, (double*)ctx->h[P], ctx->xidx, ctx->xval, count, mode, ctx->xout,
        ctx->xpart);
  ctx->launches++;
  if ((rc = exchange_finish(ctx))) return rc;
  if (volume_m3)
    *volume_m3 = fx(ctx) ? (double)ctx->xout_host->volume_w6_quanta * ctx->quantum * f
                         : ctx->xout_host->volume_w_fp64;
  return SB_OK;
}

extern "C" int sb_entrain(sb_ctx* ctx, const int32_t* flat_indices, const double* depth_m,
                          int count, double* volume_m3) {
  return entrain_common(ctx, flat_indices, depth_m, count, 0, volume_m3);
}

extern "C" int sb_entrain_to_surface(sb_ctx* ctx, const int32_t* flat_indices,
                                     const double* target_m, int count, double* volume_m3) {
  return entrain_common(ctx, flat_indices, target_m, count, 1, volume_m3);
}

extern "C" int sb_deposit(sb_ctx* ctx, const int32_t* flat_indices, const double* depth_m,
                          int count, double density_kg_m3, double* out3) {
  if (!ctx || (count > 0 && (!flat_indices || !depth_m)) || !out3) return SB_ERR_BAD_ARG;
  if (!(density_kg_m3 > 0.0)) return fail(ctx, SB_ERR_BAD_ARG, "[DeviceBulkState] invalid deposition indices/density");
  out3[0] = out3[1] = out3[2] = 0.0;
  if (count == 0) return SB_OK;
  int rc = exchange_upload(ctx, flat_indices, depth_m, count);
  if (rc) return rc;
  const int P = ctx->parity_host;
  const double f = ctx->d.dx_m * ctx->d.dy_m / 6.0;
  if (fx(ctx))
    deposit_kernel<true><<<grid_for(count), kThreads, 0, ctx->stream>>>(
        ctx->d.ny, ctx->d.nx, ctx->pitch, ctx->quantum, f, (int32_t*)ctx->b, (int32_t*)ctx->h[P],
        (float*)ctx->qx[P], (float*)ctx->qy[P], ctx->xidx, ctx->xval, count, ctx->xout,
        ctx->xpart);
  else
    deposit_kernel<false><<<grid_for(count), kThreads, 0, ctx->stream>>>(
        ctx->d.ny, ctx->d.nx, ctx->pitch, ctx->quantum, f, (double*)ctx->b, (double*)ctx->h[P],
        (double*)ctx->qx[P], (double*)ctx->qy[P], ctx->xidx, ctx->xval, count, ctx->xout,
        ctx->xpart);
  ctx->launches++;
  if ((rc = exchange_finish(ctx))) return rc;
  const ExchangeOut& o = *ctx->xout_host;
  out3[0] = fx(ctx) ? (double)o.volume_w6_quanta * ctx->quantum * f : o.volume_w_fp64;
  out3[1] = density_kg_m3 * o.momentum_w[0];
  out3[2] = density_kg_m3 * o.momentum_w[1];
  return SB_OK;
}

extern "C" int sb_deposition_step(sb_ctx* ctx, double dt_s, const sb_deposition_params* p,
                                  sb_deposition_stats* out) {
  if (!ctx || !p || !out) return SB_ERR_BAD_ARG;
  if (!(p->settling_rate_m_s > 0.0) || !(p->speed_threshold_m_s >= 0.0) ||
      !std::isfinite(p->settling_rate_m_s) || !std::isfinite(p->speed_threshold_m_s))
    return fail(ctx, SB_ERR_BAD_ARG, "[WarpDeposition] invalid configuration");
  if (!std::isfinite(dt_s) || dt_s <= 0.0)
    return fail(ctx, SB_ERR_BAD_ARG, "[WarpDeposition] dt_s must be finite/positive");
  if (!(p->density_kg_m3 > 0.0) || !std::isfinite(p->gravity_m_s2) || !std::isfinite(p->cohesion_pa))
    return fail(ctx, SB_ERR_BAD_ARG, "[WarpDeposition] invalid material");
  DepositionConst c{};
  c.ny = ctx->d.ny;
  c.nx = ctx->d.nx;
  c.pitch = ctx->pitch;
  c.dx = ctx->d.dx_m;
  c.dy = ctx->d.dy_m;
  c.dt = dt_s;
  c.rate = p->settling_rate_m_s;
  c.speed_threshold = p->speed_threshold_m_s;
  c.density = p->density_kg_m3;
  c.gravity = p->gravity_m_s2;
  c.cohesion = p->cohesion_pa;
  c.stop_tan = std::tan(p->stop_angle_deg * (M_PI / 180.0));
  c.settle_tail = p->settle_subcell_tail ? 1 : 0;
  c.Q = ctx->quantum;
  c.Qf = (float)ctx->quantum;
  const double rq = std::floor(p->settling_rate_m_s * dt_s / ctx->quantum);
  c.rate_q = rq > 2147483647.0 ? 2147483647LL : (long long)rq;
  const int P = ctx->parity_host;
  const int grid = ctx->ledger_blocks;
  double* amount = ctx->staging;
  if (fx(ctx)) {
    deposition_decide_kernel<true><<<grid, kThreads, 0, ctx->stream>>>(
        c, (const int32_t*)ctx->b, (const int32_t*)ctx->h[P], (const float*)ctx->qx[P],
        (const float*)ctx->qy[P], ctx->forcing, amount);
    deposition_apply_kernel<true><<<grid, kThreads, 0, ctx->stream>>>(
        c, (int32_t*)ctx->b, (int32_t*)ctx->h[P], (float*)ctx->qx[P], (float*)ctx->qy[P], amount,
        ctx->m2r, ctx->partials, ctx->arrive, ctx->dep_out);
  } else {
    deposition_decide_kernel<false><<<grid, kThreads, 0, ctx->stream>>>(
        c, (const double*)ctx->b, (const double*)ctx->h[P], (const double*)ctx->qx[P],
        (const double*)ctx->qy[P], ctx->forcing, amount);
    deposition_apply_kernel<false><<<grid, kThreads, 0, ctx->stream>>>(
        c, (double*)ctx->b, (double*)ctx->h[P], (double*)ctx->qx[P], (double*)ctx->qy[P], amount,
        ctx->m2r, ctx->partials, ctx->arrive, ctx->dep_out);
  }
  ctx->launches += 2;
  SB_CUDA(ctx, cudaGetLastError());
  SB_CUDA(ctx, cudaMemcpyAsync(ctx->dep_out_host, ctx->dep_out, sizeof(DepositionOut),
                               cudaMemcpyDeviceToHost, ctx->stream));
  SB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  const DepositionOut& o = *ctx->dep_out_host;
  const double f = ctx->d.dx_m * ctx->d.dy_m / 6.0;
  out->deposited_volume_m3 = fx(ctx) ? (double)o.volume_w6_quanta * ctx->quantum * f : o.volume_w;
  out->removed_momentum_kg_m_s[0] = o.momentum_w[0];
  out->removed_momentum_kg_m_s[1] = o.momentum_w[1];
  out->deposited_w6_quanta = fx(ctx) ? o.volume_w6_quanta : 0;
  out->cells = o.cells;
  out->pad = 0;
  return SB_OK;
}

extern "C" int sb_avalanche_set_initial_resting(sb_ctx* ctx) {
  if (!ctx) return SB_ERR_BAD_ARG;
  SB_CUDA(ctx, cudaMemcpyAsync(ctx->initial_b, ctx->b, (size_t)ctx->pitch * ctx->d.ny * ctx->esize,
                               cudaMemcpyDeviceToDevice, ctx->stream));
  SB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return SB_OK;
}

extern "C" int sb_avalanche_mobilize(sb_ctx* ctx, double activation_time_s,
                                     double mobilization_depth_m, double dry_tolerance_m,
                                     sb_mobilize_stats* out) {
  if (!ctx || !out) return SB_ERR_BAD_ARG;
  if (!std::isfinite(activation_time_s) || !(mobilization_depth_m > 0.0) ||
      !(dry_tolerance_m >= 0.0))
    return fail(ctx, SB_ERR_BAD_ARG, "[GpuLargeAvalanche] invalid mobilization parameters");
  MobilizeConst c{ctx->d.ny, ctx->d.nx, ctx->pitch, ctx->quantum, ctx->d.datum_m,
                  ctx->d.dx_m * ctx->d.dy_m / 6.0, mobilization_depth_m, dry_tolerance_m,
                  activation_time_s};
  const int P = ctx->parity_host;
  const int grid = ctx->ledger_blocks;
  if (fx(ctx))
    mobilize_kernel<true><<<grid, kThreads, 0, ctx->stream>>>(
        c, (const int32_t*)ctx->z, (int32_t*)ctx->b, (int32_t*)ctx->h[P], ctx->parent, ctx->latch,
        (const float*)ctx->severity, ctx->owned_surface, ctx->export_base, ctx->export_cum,
        ctx->act_count, ctx->act_first, ctx->act_last, ctx->r2m, ctx->lout, ctx->partials,
        ctx->arrive, ctx->mob_out);
  else
    mobilize_kernel<false><<<grid, kThreads, 0, ctx->stream>>>(
        c, (const double*)ctx->z, (double*)ctx->b, (double*)ctx->h[P], ctx->parent, ctx->latch,
        (const double*)ctx->severity, ctx->owned_surface, ctx->export_base, ctx->export_cum,
        ctx->act_count, ctx->act_first, ctx->act_last, ctx->r2m, ctx->lout, ctx->partials,
        ctx->arrive, ctx->mob_out);
  ctx->launches++;
  SB_CUDA(ctx, cudaGetLastError());
  SB_CUDA(ctx, cudaMemcpyAsync(ctx->mob_out_host, ctx->mob_out, sizeof(MobilizeOut),
                               cudaMemcpyDeviceToHost, ctx->stream));
  SB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  const MobilizeOut& o = *ctx->mob_out_host;
  const double f = ctx->d.dx_m * ctx->d.dy_m / 6.0;
  out->transferred_volume_m3 = fx(ctx) ? (double)o.transferred_w6_quanta * ctx->quantum * f : o.v[0];
  out->newly_activated_volume_m3 = o.v[1];
  out->reactivated_volume_m3 = o.v[2];
  out->newly_activated_area_m2 = o.v[3];
  out->reactivated_area_step_m2 = o.v[4];
  out->transferred_w6_quanta = fx(ctx) ? o.transferred_w6_quanta : 0;
  out->cells = (int)o.v[5];
  out->pad = 0;
  return SB_OK;
}

extern "C" int sb_avalanche_persistence(sb_ctx* ctx, double start_angle_rad, double stop_angle_rad,
                                        double dry_tolerance_m, double activity_speed_m_s,
                                        sb_persistence_stats* out) {
  if (!ctx || !out) return SB_ERR_BAD_ARG;
  PersistConst c{ctx->d.ny, ctx->d.nx, ctx->pitch, ctx->d.tile_size, ctx->ftiles1, ctx->quantum,
                 ctx->d.datum_m, ctx->d.dx_m * ctx->d.dy_m / 6.0, start_angle_rad, stop_angle_rad,
                 dry_tolerance_m, activity_speed_m_s};
  const size_t nt = (size_t)ctx->ftiles0 * ctx->ftiles1;
  SB_CUDA(ctx, cudaMemsetAsync(ctx->ptiles, 0, nt * sizeof(int), ctx->stream));
  const int P = ctx->parity_host;
  const int grid = ctx->ledger_blocks;
  if (fx(ctx))
    persistence_kernel<true><<<grid, kThreads, 0, ctx->stream>>>(
        c, (const int32_t*)ctx->initial_b, (const int32_t*)ctx->b, (const int32_t*)ctx->h[P],
        (const float*)ctx->qx[P], (const float*)ctx->qy[P], (const float*)ctx->slope, ctx->parent,
        ctx->latch, ctx->act_count, ctx->r2m, ctx->m2r, ctx->ptiles, ctx->partials, ctx->arrive,
        ctx->pers_out);
  else
    persistence_kernel<false><<<grid, kThreads, 0, ctx->stream>>>(
        c, (const double*)ctx->initial_b, (const double*)ctx->b, (const double*)ctx->h[P],
        (const double*)ctx->qx[P], (const double*)ctx->qy[P], (const double*)ctx->slope,
        ctx->parent, ctx->latch, ctx->act_count, ctx->r2m, ctx->m2r, ctx->ptiles, ctx->partials,
        ctx->arrive, ctx->pers_out);
  ctx->launches++;
  SB_CUDA(ctx, cudaGetLastError());
  std::vector<int> flags(nt);
  SB_CUDA(ctx, cudaMemcpyAsync(ctx->pers_out_host, ctx->pers_out, kPersistSlots * sizeof(double),
                               cudaMemcpyDeviceToHost, ctx->stream));
  SB_CUDA(ctx, cudaMemcpyAsync(flags.data(), ctx->ptiles, nt * sizeof(int), cudaMemcpyDeviceToHost,
                               ctx->stream));
  SB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  const double* v = ctx->pers_out_host;
  out->unique_cells_ever_activated = (int)v[14];
  out->cells_activated_more_than_once = (int)v[15];
  out->current_mobile_cell_count = (int)v[16];
  out->retired_candidate_cell_count = (int)v[17];
  out->active_tile_count = (int)std::count_if(flags.begin(), flags.end(), [](int f) { return f != 0; });
  out->pad = 0;
  out->cumulative_r2m_m3 = v[0];
  out->cumulative_m2r_m3 = v[1];
  out->unique_activated_area_m2 = v[2];
  out->reactivated_area_m2 = v[3];
  out->current_mobile_volume_m3 = v[4];
  out->maximum_mobile_speed_m_s = v[5];
  out->net_terrain_volume_change_m3 = v[6];
  out->net_spatial_transfer_m3 = v[7];
  out->activated_slope_sum_rad = v[8];
  out->activated_slope_max_rad = v[9];
  out->slope_minus_stop_sum_rad = v[10];
  out->start_minus_slope_sum_rad = v[11];
  out->retired_candidate_area_m2 = v[12];
  out->moving_mobile_volume_m3 = v[13];
  return SB_OK;
}

extern "C" int sb_surface_capture(sb_ctx* ctx) {
  if (!ctx) return SB_ERR_BAD_ARG;
  const int P = ctx->parity_host;
  const int g = grid_for((long long)ctx->d.ny * ctx->d.nx);
  if (fx(ctx))
    surface_capture_kernel<true><<<g, kThreads, 0, ctx->stream>>>(
        ctx->d.ny, ctx->d.nx, ctx->pitch, ctx->quantum, ctx->d.datum_m, (const int32_t*)ctx->b,
        (const int32_t*)ctx->h[P], ctx->surf_before);
  else
    surface_capture_kernel<false><<<g, kThreads, 0, ctx->stream>>>(
        ctx->d.ny, ctx->d.nx, ctx->pitch, 0.0, 0.0, (const double*)ctx->b, (const double*)ctx->h[P],
        ctx->surf_before);
  ctx->launches++;
  SB_CUDA(ctx, cudaGetLastError());
  SB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return SB_OK;
}

extern "C" int sb_surface_dirty_tiles(sb_ctx* ctx, double tolerance_m, int32_t* flags, int ntiles) {
  if (!ctx || !flags) return SB_ERR_BAD_ARG;
  if (!std::isfinite(tolerance_m) || tolerance_m < 0.0)
    return fail(ctx, SB_ERR_BAD_ARG, "[DeviceBulkState] dirty tolerance must be finite/non-negative");
  const size_t nt = (size_t)ctx->ftiles0 * ctx->ftiles1;
  if ((size_t)ntiles < nt) return fail(ctx, SB_ERR_CAPACITY, "[soilb200] tile flag buffer too small");
  SB_CUDA(ctx, cudaMemsetAsync(ctx->dtiles, 0, nt * sizeof(int), ctx->stream));
  const int P = ctx->parity_host;
  const int g = grid_for((long long)ctx->d.ny * ctx->d.nx);
  if (fx(ctx))
    surface_flag_kernel<true><<<g, kThreads, 0, ctx->stream>>>(
        ctx->d.ny, ctx->d.nx, ctx->pitch, ctx->quantum, ctx->d.datum_m, (const int32_t*)ctx->b,
        (const int32_t*)ctx->h[P], ctx->surf_before, ctx->d.tile_size, ctx->ftiles1, tolerance_m,
        ctx->dtiles);
  else
    surface_flag_kernel<false><<<g, kThreads, 0, ctx->stream>>>(
        ctx->d.ny, ctx->d.nx, ctx->pitch, 0.0, 0.0, (const double*)ctx->b, (const double*)ctx->h[P],
        ctx->surf_before, ctx->d.tile_size, ctx->ftiles1, tolerance_m, ctx->dtiles);
  ctx->launches++;
  SB_CUDA(ctx, cudaGetLastError());
  SB_CUDA(ctx, cudaMemcpyAsync(flags, ctx->dtiles, nt * sizeof(int), cudaMemcpyDeviceToHost,
                               ctx->stream));
  SB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return SB_OK;
}

extern "C" int sb_surface_region(sb_ctx* ctx, int r0, int r1, int c0, int c1, double* out) {
  if (!ctx || !out) return SB_ERR_BAD_ARG;
  if (r0 < 0 || c0 < 0 || r1 > ctx->d.ny || c1 > ctx->d.nx || r1 <= r0 || c1 <= c0)
    return fail(ctx, SB_ERR_BAD_ARG, "[DeviceBulkState] region outside grid");
  const int count = (r1 - r0) * (c1 - c0);
  const int P = ctx->parity_host;
  const int g = grid_for(count);
  if (fx(ctx))
    surface_region_kernel<true><<<g, kThreads, 0, ctx->stream>>>(
        c1 - c0, count, r0, c0, ctx->pitch, ctx->quantum, ctx->d.datum_m, (const int32_t*)ctx->b,
        (const int32_t*)ctx->h[P], ctx->staging);
  else
    surface_region_kernel<false><<<g, kThreads, 0, ctx->stream>>>(
        c1 - c0, count, r0, c0, ctx->pitch, 0.0, 0.0, (const double*)ctx->b,
        (const double*)ctx->h[P], ctx->staging);
  ctx->launches++;
  SB_CUDA(ctx, cudaGetLastError());
  SB_CUDA(ctx, cudaMemcpyAsync(out, ctx->staging, (size_t)count * 8, cudaMemcpyDeviceToHost,
                               ctx->stream));
  SB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return SB_OK;
}

extern "C" int sb_surface_sample_bilinear(sb_ctx* ctx, const double* rows, const double* cols,
                                          int count, double* out) {
  if (!ctx || count < 0 || (count > 0 && (!rows || !cols || !out))) return SB_ERR_BAD_ARG;
  if (count == 0) return SB_OK;
  for (int i = 0; i < count; ++i)
    if (!std::isfinite(rows[i]) || !std::isfinite(cols[i]))
      return fail(ctx, SB_ERR_BAD_ARG, "[DeviceBulkState] terrain queries must be finite [N,2]");
  if (count > ctx->q_cap) {
    cudaFree(ctx->q_rows);
    cudaFree(ctx->q_cols);
    cudaFree(ctx->q_out);
    ctx->q_rows = ctx->q_cols = ctx->q_out = nullptr;
    ctx->q_cap = 0;
    SB_CUDA(ctx, cudaMalloc(&ctx->q_rows, (size_t)count * 8));
    SB_CUDA(ctx, cudaMalloc(&ctx->q_cols, (size_t)count * 8));
    SB_CUDA(ctx, cudaMalloc(&ctx->q_out, (size_t)count * 8));
    ctx->q_cap = count;
  }
  SB_CUDA(ctx, cudaMemcpyAsync(ctx->q_rows, rows, (size_t)count * 8, cudaMemcpyHostToDevice, ctx->stream));
  SB_CUDA(ctx, cudaMemcpyAsync(ctx->q_cols, cols, (size_t)count * 8, cudaMemcpyHostToDevice, ctx->stream));
  const int P = ctx->parity_host;
  const int g = grid_for(count);
  if (fx(ctx))
    surface_bilinear_kernel<true><<<g, kThreads, 0, ctx->stream>>>(
        ctx->d.ny, ctx->d.nx, ctx->pitch, ctx->quantum, ctx->d.datum_m, (const int32_t*)ctx->b,
        (const int32_t*)ctx->h[P], ctx->q_rows, ctx->q_cols, count, ctx->q_out);
  else
    surface_bilinear_kernel<false><<<g, kThreads, 0, ctx->stream>>>(
        ctx->d.ny, ctx->d.nx, ctx->pitch, 0.0, 0.0, (const double*)ctx->b, (const double*)ctx->h[P],
        ctx->q_rows, ctx->q_cols, count, ctx->q_out);
  ctx->launches++;
  SB_CUDA(ctx, cudaGetLastError());
  SB_CUDA(ctx, cudaMemcpyAsync(out, ctx->q_out, (size_t)count * 8, cudaMemcpyDeviceToHost, ctx->stream));
  SB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return SB_OK;
}

// ---------------------------------------------------------------------------
// Fused plain terrain step (one graph per step)
// ---------------------------------------------------------------------------
namespace {

template <bool FX>
int build_path_graph(sb_ctx* ctx, const sb_path_params* p) {
  using T = FvTypes<FX>;
  if (ctx->path_exec) cudaGraphExecDestroy(ctx->path_exec);
  if (ctx->path_graph) cudaGraphDestroy(ctx->path_graph);
  ctx->path_exec = nullptr;
  ctx->path_graph = nullptr;
  ctx->path_valid = false;
  cudaGraph_t g;
  SB_CUDA(ctx, cudaGraphCreate(&g, 0));
  ctx->path_graph = g;
  cudaGraphConditionalHandle h_mob, h_front;
  // a conditional handle without a conditional node can fail instantiation:
  // the persistent substep loop needs none
  h_mob = 0;
  if (!(FX && ctx->fv_stream && ctx->fv_persistent))
    SB_CUDA(ctx, cudaGraphConditionalHandleCreate(&h_mob, g, 0, cudaGraphCondAssignDefault));
  SB_CUDA(ctx, cudaGraphConditionalHandleCreate(&h_front, g, 0, cudaGraphCondAssignDefault));
  int rc, one = 1, zero = 0;
  const int ny = ctx->d.ny, nx = ctx->d.nx;
  double Q = ctx->quantum, datum = ctx->d.datum_m, f = ctx->d.dx_m * ctx->d.dy_m / 6.0;
  cudaGraphNode_t prev, node;
  SB_CUDA(ctx, cudaGraphAddEventRecordNode(&prev, g, nullptr, 0, ctx->ev_path[0]));
  ctx->n_stage = 0;
  // stage boundary on the main chain (only with stage events enabled)
  auto mark = [&]() -> int {
    if (!ctx->stage_events || ctx->n_stage >= sb_ctx::kStages) return SB_OK;
    cudaGraphNode_t ev;
    SB_CUDA(ctx, cudaGraphAddEventRecordNode(&ev, g, &prev, 1, ctx->ev_stage[ctx->n_stage++]));
    prev = ev;
    return SB_OK;
  };
  // 1. step start (loop control, cleared records), cut entrainment: one
  // block when the command buffer holds at most kPathStartCells cells (the
  // entrainment stage is then part of the start stage), else a start kernel
  // and a 64-block entrainment kernel
  if (ctx->path_cap <= kPathStartCells) {
    int pitch = ctx->pitch;
    int nyv = ny, nxv = nx;
    void *in_dev = nullptr, *idx_dev = nullptr, *val_dev = nullptr;
    SB_CUDA(ctx, cudaHostGetDevicePointer(&in_dev, ctx->path_in, 0));
    SB_CUDA(ctx, cudaHostGetDevicePointer(&idx_dev, ctx->path_idx, 0));
    SB_CUDA(ctx, cudaHostGetDevicePointer(&val_dev, ctx->path_val, 0));
    int cap = ctx->path_cap;
    void* args[] = {&nyv, &nxv, &pitch, &Q, &datum, &f, &ctx->b, &ctx->z, &ctx->h[0], &ctx->h[1],
                    &ctx->ctl, &in_dev, (void*)&ctx->dt_dev, &idx_dev, &val_dev, &cap, &ctx->xout,
                    &ctx->lout};
    if ((rc = add_kernel(ctx, g, &node, &prev, 1, (void*)path_start_kernel<FX>, dim3(1), 0, args)))
      return rc;
    prev = node;
    if ((rc = mark())) return rc;
    if ((rc = mark())) return rc;
  } else {
  {
    void* in_dev = nullptr;
    SB_CUDA(ctx, cudaHostGetDevicePointer(&in_dev, ctx->path_in, 0));
    void* args[] = {(void*)&ctx->ctl, &in_dev, (void*)&ctx->dt_dev, (void*)&ctx->path_count,
                    (void*)&ctx->xout, (void*)&ctx->lout};
    if ((rc = add_kernel(ctx, g, &node, &prev, 1, (void*)path_begin_kernel, dim3(1), 0, args)))
      return rc;
    prev = node;
    if ((rc = mark())) return rc;
  }
  {
    int pitch = ctx->pitch;
    int nyv = ny, nxv = nx;
    void *idx_dev = nullptr, *val_dev = nullptr;
    SB_CUDA(ctx, cudaHostGetDevicePointer(&idx_dev, ctx->path_idx, 0));
    SB_CUDA(ctx, cudaHostGetDevicePointer(&val_dev, ctx->path_val, 0));
    void* args[] = {&nyv, &nxv, &pitch, &Q, &datum, &f, &ctx->b, &ctx->z, &ctx->h[0], &ctx->h[1],
                    &ctx->ctl, &idx_dev, &val_dev, &ctx->path_count, &ctx->xout, &ctx->xpart};
    if ((rc = add_kernel(ctx, g, &node, &prev, 1, (void*)path_entrain_kernel<FX>, dim3(64), 0, args)))
      return rc;
    prev = node;
    if ((rc = mark())) return rc;
  }
  }
  // 2. Mobile V2 (same kernels as the standalone step graph)
  FvConst fc;
  fc = make_const(ctx, &p->mobile);
  double static_limit, dat;
  static_limit = std::tan(p->mobile.start_angle_deg * (M_PI / 180.0)) + 1.0e-14;
  dat = ctx->d.datum_m;
  int mode0 = 0, mode1 = 2, use_h = 1, no_h = 0;  // 2: after + diagnostics fold
  {
    // the prologue sets the WHILE condition only when the loop is one
    int pro_h = (FX && ctx->fv_stream && ctx->fv_persistent) ? 0 : use_h;
    std::vector<void*> args;
    ledger_args<FX>(ctx, fc, &dat, &static_limit, &mode0, &h_mob, &pro_h, args);
    if ((rc = add_kernel(ctx, g, &node, &prev, 1, (void*)ledger_kernel<FX>, dim3(ctx->ledger_blocks),
                         0, args.data())))
      return rc;
    prev = node;
    if ((rc = mark())) return rc;
  }
  SB_CUDA(ctx, cudaGraphAddEventRecordNode(&node, g, &prev, 1, ctx->ev_loop[0]));
  prev = node;
  if ((rc = add_substep_loop<FX>(ctx, g, prev, fc, &h_mob, &use_h, &node))) return rc;
  prev = node;
  SB_CUDA(ctx, cudaGraphAddEventRecordNode(&node, g, &prev, 1, ctx->ev_loop[1]));
  prev = node;
  // The after-step ledger and the labelling chain both only read the final
  // state: the ledger runs as a second branch that starts after the yield /
  // tile union-find pass (which fills the SMs on its own) and overlaps the
  // border merge and compression (short dependent chains that leave the SMs
  // idle); the branches join at the component reduction.
  cudaGraphNode_t n_after;
  // 3. labelling
  LabelConst lc;
  lc = make_label_const(ctx, &p->label);
  const int ltiles = lc.tiles_x * ((ny + kLabelTile - 1) / kLabelTile);
  {
    void* args[] = {&lc, &ctx->b, &ctx->z, &ctx->h[0], &ctx->h[1], &ctx->qx[0], &ctx->qx[1],
                    &ctx->qy[0], &ctx->qy[1], &ctx->ctl, &ctx->parent, &ctx->slope, &ctx->severity,
                    &ctx->latch, &ctx->export_cum, &ctx->export_base, &ctx->roots};
    if ((rc = add_kernel(ctx, g, &node, &prev, 1, (void*)label_init_local_kernel<FX>, dim3(ltiles),
                         0, args, kLabelInitThreads)))
      return rc;
    prev = node;
  }
  {
    std::vector<void*> args;
    ledger_args<FX>(ctx, fc, &dat, &static_limit, &mode1, &h_mob, &no_h, args);
    if ((rc = add_kernel(ctx, g, &n_after, &prev, 1, (void*)ledger_kernel<FX>,
                         dim3(ctx->ledger_blocks), 0, args.data())))
      return rc;
    if ((rc = mark())) return rc;
  }
  {
    void* args[] = {&lc, &ctx->parent, &ctx->lout};
    if ((rc = add_kernel(ctx, g, &node, &prev, 1, (void*)label_merge_kernel, dim3(ltiles), 0, args)))
      return rc;
    prev = node;
    if ((rc = mark())) return rc;
  }
  {
    int mask_only = 0;
    void* args[] = {&lc, &ctx->parent, &ctx->b, &ctx->z, &ctx->slope, &ctx->severity, &ctx->latch,
                    &ctx->previous, &ctx->roots, &ctx->root_list, &ctx->lout, &mask_only};
    if ((rc = add_kernel(ctx, g, &node, &prev, 1, (void*)label_compress_kernel<FX>,
                         dim3(grid_for((long long)ny * nx)), 0, args)))
      return rc;
    prev = node;
    if ((rc = mark())) return rc;
  }
  // 4. component reduction + classification / persistence / gate, then
  // previous mask + seeding
  PathConst pc;
  pc = PathConst{};
  pc.f = f;
  pc.Q = ctx->quantum;
  pc.dx = ctx->d.dx_m;
  pc.dy = ctx->d.dy_m;
  pc.min_cells = p->minimum_connected_cells;
  pc.min_area = p->minimum_connected_area_m2;
  pc.min_volume = p->minimum_mobilizable_volume_m3;
  pc.min_mean_excess_deg = p->minimum_mean_excess_start_deg;
  pc.persistence_time = p->persistence_time_s;
  pc.settled_volume = p->settled_mobile_volume_m3;
  pc.settled_speed = p->settled_speed_m_s;
  pc.dry_tol = p->label.dry_tolerance_m;
  pc.residual_mode = p->residual_mode;
  pc.fx = FX ? 1 : 0;
  RelaxConst rcn;
  if ((rc = relax_const(ctx, &p->relax, &rcn, ctx->d.tile_size))) return rc;
  {
    void* args[] = {&ctx->roots, &ctx->root_list, &ctx->lout, &ctx->arrive, &pc,
                    &ctx->io,    &ctx->xout,      &ctx->pstate, &ctx->dt_dev, &ctx->rctl};
    const cudaGraphNode_t deps[2] = {prev, n_after};
    if ((rc = add_kernel(ctx, g, &node, deps, 2, (void*)path_reduce_classify_kernel, dim3(32), 0,
                         args)))
      return rc;
    prev = node;
    if ((rc = mark())) return rc;
  }
  // 5. previous mask + frontier seeds; its last block opens the gated
  // residual frontier loop (same kernels as sb_frontier_run)
  void* begin_args[] = {&rcn, &ctx->ftile_next, &ctx->phase[0], &ctx->phase[1], &ctx->rctl,
                        &h_front};
  {
    void* args[] = {&lc, &ctx->parent, &ctx->previous, &ctx->reached, &ctx->ftile_next, &ctx->lout,
                    &ctx->pstate, &rcn, &ctx->phase[0], &ctx->phase[1], &ctx->rctl, &h_front};
    if ((rc = add_kernel(ctx, g, &node, &prev, 1, (void*)path_update_previous_kernel,
                         dim3(grid_for((long long)ny * nx)), 0, args)))
      return rc;
    prev = node;
    if ((rc = mark())) return rc;
  }
  {
    cudaGraphNodeParams cp{};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h_front;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    SB_CUDA(ctx, cudaGraphAddNode(&node, g, &prev, 1, &cp));
    prev = node;
    if ((rc = mark())) return rc;
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    int dirs[8], pars[8];
    typename T::H* hf;
    hf = (typename T::H*)ctx->b;
    cudaGraphNode_t bprev = nullptr, bnode;
    for (int k = 0; k < 8; ++k) {
      dirs[k] = k / 2;
      pars[k] = k % 2;
      void* args[] = {&rcn, &dirs[k], &pars[k], &hf, &ctx->reached, &ctx->phase[0],
                      &ctx->phase[1], &ctx->rctl};
      if ((rc = add_kernel(ctx, body, &bnode, bprev ? &bprev : nullptr, bprev ? 1 : 0,
                           (void*)frontier_subphase_kernel<FX>, dim3(ctx->frontier_grid), 0,
                           args)))
        return rc;
      bprev = bnode;
    }
    void* sargs[] = {&rcn, &hf, &ctx->reached, &ctx->phase[1], &ctx->ftile_next, &ctx->rctl};
    if ((rc = add_kernel(ctx, body, &bnode, &bprev, 1, (void*)frontier_scan_kernel<FX>,
                         dim3(ctx->frontier_grid), 0, sargs)))
      return rc;
    bprev = bnode;
    if ((rc = add_kernel(ctx, body, &bnode, &bprev, 1, (void*)frontier_begin_kernel, dim3(1), 0,
                         begin_args)))
      return rc;
  }
  // 6. records to the pinned host copies (+ frontier_finish)
  {
    PathRecordPtrs rp;
    const void* srcs[6] = {ctx->ctl, ctx->io, ctx->lout, ctx->rctl, ctx->pstate, ctx->xout};
    void* hosts[6] = {ctx->ctl_host, ctx->io_host, ctx->lout_host, ctx->rctl_host,
                      ctx->pstate_host, ctx->xout_host};
    const int sizes[6] = {(int)sizeof(FvControl), (int)sizeof(StepIO), (int)sizeof(LabelOut),
                          (int)sizeof(RelaxControl), (int)sizeof(PathState),
                          (int)sizeof(ExchangeOut)};
    for (int k = 0; k < 6; ++k) {
      static_assert(sizeof(FvControl) % 4 == 0 && sizeof(StepIO) % 4 == 0 &&
                        sizeof(LabelOut) % 4 == 0 && sizeof(RelaxControl) % 4 == 0 &&
                        sizeof(PathState) % 4 == 0 && sizeof(ExchangeOut) % 4 == 0,
                    "records are copied as 32-bit words");
      void* dptr = nullptr;
      SB_CUDA(ctx, cudaHostGetDevicePointer(&dptr, hosts[k], 0));
      rp.src[k] = srcs[k];
      rp.dst[k] = dptr;
      rp.bytes[k] = sizes[k];
    }
    void* args[] = {&rp, &rcn, &ctx->reached, &ctx->rctl};
    if ((rc = add_kernel(ctx, g, &node, &prev, 1, (void*)path_records_kernel,
                         dim3(std::min(grid_for((long long)rcn.n0 * rcn.pitch), 2 * 148)), 0, args)))
      return rc;
    prev = node;
  }
  SB_CUDA(ctx, cudaGraphAddEventRecordNode(&node, g, &prev, 1, ctx->ev_path[1]));
  (void)one;
  (void)zero;
  SB_CUDA(ctx, cudaGraphInstantiate(&ctx->path_exec, g, 0));
  ctx->path_valid = true;
  return SB_OK;
}

}  // namespace

// Device-time breakdown of the last sb_path_step (SOILB200_STAGE_EVENTS=1 at
// context creation): out[k] = ms from the previous boundary to stage k's end.
extern "C" int sb_path_stage_times(sb_ctx* ctx, float* out_ms, int capacity) {
  if (!ctx || !out_ms || capacity < 0) return -SB_ERR_BAD_ARG;
  const int n = ctx->stage_events ? std::min(ctx->n_stage, capacity) : 0;
  for (int k = 0; k < n; ++k) out_ms[k] = ctx->stage_ms[k];
  return n;
}

extern "C" int sb_path_reset(sb_ctx* ctx) {
  if (!ctx) return SB_ERR_BAD_ARG;
  SB_CUDA(ctx, cudaMemsetAsync(ctx->pstate, 0, sizeof(PathState), ctx->stream));
  SB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return SB_OK;
}

extern "C" int sb_path_step(sb_ctx* ctx, double dt_s, const int32_t* cut_idx,
                            const double* cut_target, int cut_count, const sb_path_params* p,
                            sb_path_stats* out) {
  if (!ctx || !p || !out) return SB_ERR_BAD_ARG;
  if (!std::isfinite(dt_s) || dt_s <= 0.0) return fail(ctx, SB_ERR_BAD_ARG, "dt must be finite/positive");
  if (cut_count < 0 || (cut_count > 0 && (!cut_idx || !cut_target)) ||
      (long long)cut_count > (long long)ctx->d.ny * ctx->d.nx)
    return fail(ctx, SB_ERR_BAD_ARG, "[DeviceBulkState] invalid entrainment request");
  if (p->label.connectivity != 4 && p->label.connectivity != 8)
    return fail(ctx, SB_ERR_BAD_ARG, "[LargeAvalanche] connectivity must be 4 or 8");
  int rc = check_params(ctx, &p->mobile);
  if (rc) return rc;
  if (!ctx->use_graphs)
    return fail(ctx, SB_ERR_STATE, "[soilb200] the fused step needs CUDA graphs (unset SOILB200_NO_GRAPH)");
  if (cut_count > ctx->path_cap || !ctx->path_idx) {
    // the graph reads the command from these buffers: grow them (rare; the
    // cut footprint changes little between steps) and rebuild the graph
    const long long cells = (long long)ctx->d.ny * ctx->d.nx;
    const int cap = (int)std::min<long long>(
        cells, std::max<long long>({(long long)cut_count, 2LL * ctx->path_cap, 4096LL}));
    SB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (ctx->path_idx) cudaFreeHost(ctx->path_idx);
    if (ctx->path_val) cudaFreeHost(ctx->path_val);
    ctx->path_idx = nullptr;
    ctx->path_val = nullptr;
    ctx->path_cap = 0;
    ctx->path_valid = false;
    SB_CUDA(ctx, cudaHostAlloc(&ctx->path_idx, (size_t)cap * 4, cudaHostAllocMapped));
    SB_CUDA(ctx, cudaHostAlloc(&ctx->path_val, (size_t)cap * 8, cudaHostAllocMapped));
    ctx->path_cap = cap;
  }
  if (!ctx->path_valid || std::memcmp(ctx->path_key, p, sizeof(*p)) != 0) {
    static_assert(sizeof(sb_path_params) <= sizeof(((sb_ctx*)nullptr)->path_key), "key size");
    rc = fx(ctx) ? build_path_graph<true>(ctx, p) : build_path_graph<false>(ctx, p);
    if (rc) return rc;
    std::memcpy(ctx->path_key, p, sizeof(*p));
    // the standalone Mobile graph shares the control block; force its rebuild check
    ctx->mobile.valid = false;
  }
  // the previous step's graph has finished (every call ends synchronised), so
  // the mapped inputs are free to overwrite; the launch publishes them
  ctx->path_in->dt = dt_s;
  ctx->path_in->count = cut_count;
  if (cut_count > 0) {
    for (int k = 0; k < cut_count; ++k)
      if (!std::isfinite(cut_target[k]))
        return fail(ctx, SB_ERR_BAD_ARG, "[DeviceBulkState] invalid entrainment request");
    std::memcpy(ctx->path_idx, cut_idx, (size_t)cut_count * 4);
    std::memcpy(ctx->path_val, cut_target, (size_t)cut_count * 8);
  }
  SB_CUDA(ctx, cudaGraphLaunch(ctx->path_exec, ctx->stream));
  SB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  std::memset(out, 0, sizeof(*out));
  if ((rc = fill_mobile_stats(ctx, &p->mobile, &out->mobile))) return rc;
  const LabelOut& o = *ctx->lout_host;
  out->label.status = o.status;
  out->label.unstable_cell_count = o.total_unstable;
  out->label.connected_region_count = o.regions;
  out->label.largest_connected_cell_count = o.largest;
  out->label.winner_root = o.winner;
  out->label.union_passes = 2;
  out->label.previous_overlap = o.prev_overlap;
  const double f = ctx->d.dx_m * ctx->d.dy_m / 6.0;
  out->label.largest_connected_area_m2 = (double)o.area6 * f;
  out->label.largest_connected_mobilizable_volume_m3 =
      fx(ctx) ? (double)o.volume * ctx->quantum * f : (double)o.volume / kVolumeScaleFp64 * f;
  out->label.excess_start_sum_rad = (double)o.exc_start / kExcessScale;
  out->label.excess_start_max_rad = (double)o.max_exc_start / kExcessScale;
  out->label.excess_stop_sum_rad = (double)o.exc_stop / kExcessScale;
  out->label.excess_stop_max_rad = (double)o.max_exc_stop / kExcessScale;
  const RelaxControl& r = *ctx->rctl_host;
  out->relax.iterations = r.rounds;
  out->relax.converged = r.converged;
  out->relax.status = r.status;
  out->relax.active_tiles = r.n_active;
  out->relax.moved_edges = r.moved_edges;
  const PathState& ps = *ctx->pstate_host;
  out->entrained_m3 = ps.entrained_m3;
  out->persistence_s = ps.persistence_s;
  out->mean_excess_start_deg = ps.mean_excess_start_deg;
  out->classification = ps.classification;
  out->candidate = ps.candidate;
  out->transition_ready = ps.ready;
  out->residual_ran = ps.residual_enable;
  float step_ms = 0.f;
  SB_CUDA(ctx, cudaEventElapsedTime(&step_ms, ctx->ev_path[0], ctx->ev_path[1]));
  out->device_ms = step_ms;
  if (ctx->stage_events) {
    cudaEvent_t prev_ev = ctx->ev_path[0];
    for (int k = 0; k < ctx->n_stage; ++k) {
      SB_CUDA(ctx, cudaEventElapsedTime(&ctx->stage_ms[k], prev_ev, ctx->ev_stage[k]));
      prev_ev = ctx->ev_stage[k];
    }
  }
  const FvControl& k = *ctx->ctl_host;
  // ten kernels outside the loops, two substep launches per loop iteration,
  // ten kernels per residual round
  ctx->launches += 10 +
                   ((fx(ctx) && ctx->fv_stream && ctx->fv_persistent) ? 1
                                                                      : (k.substeps + 1) / 2 * 2) +
                   10LL * r.rounds;
  if (ctx->xout_host->bad_index)
    return fail(ctx, SB_ERR_BAD_ARG, "[DeviceBulkState] entrainment index outside state");
  if (k.status == SB_ERR_POSITIVITY) return fail(ctx, SB_ERR_POSITIVITY, "MobileV2 positivity failure");
  if (k.status == SB_ERR_SUBSTEP_CAP)
    return fail(ctx, SB_ERR_SUBSTEP_CAP, "MobileV2 maximum_substeps exceeded");
  if (k.status) return fail(ctx, k.status, "[soilb200] device status %d", k.status);
  if (o.status)
    return fail(ctx, SB_ERR_NONCONVERGENCE, "NUMERICAL_NONCONVERGENCE: device avalanche connected components");
  if (r.status == SB_ERR_NONCONVERGENCE)
    return fail(ctx, SB_ERR_NONCONVERGENCE,
                "NUMERICAL_NONCONVERGENCE: GPU residual MiniSlope exceeded the numerical safety limit");
  return SB_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free connected components (sb_label_mask_static).
//
// For callers that may not allocate device memory themselves or through this
// library: the union-find needs per-root counters and a root list beyond its
// input mask and output labels, and here that scratch lives in one file-scope
// static device array sized for kStaticLabelMaxCells cells (8 MiB + header,
// reserved on every GPU that loads the library, until process exit).
// ---------------------------------------------------------------------------
namespace {

constexpr int kStaticLabelMaxCells = 1 << 19;  // 524288 cells (701 x 701 fits)
constexpr size_t kStaticHeaderBytes = 256;     // LabelOut + arrive counter, zeroed per call
constexpr size_t kStaticCountOffset = kStaticHeaderBytes;
constexpr size_t kStaticAreaOffset = kStaticCountOffset + (size_t)kStaticLabelMaxCells * 4;
constexpr size_t kStaticRootOffset = kStaticAreaOffset + (size_t)kStaticLabelMaxCells * 8;
constexpr size_t kStaticScratchBytes = kStaticRootOffset + (size_t)kStaticLabelMaxCells * 4;
static_assert(sizeof(LabelOut) + sizeof(unsigned int) <= kStaticHeaderBytes, "header too small");

static __device__ __align__(256) unsigned char g_label_scratch[kStaticScratchBytes];

constexpr int kMaxDevices = 64;
// Device address of g_label_scratch per device ordinal, looked up once; the
// mutex makes a first call from two host threads at once safe.
unsigned char* g_label_scratch_ptr[kMaxDevices] = {nullptr};
std::mutex g_label_scratch_mutex;

// Per-cell init of the static variant: only the counters it uses are cleared.
__global__ void __launch_bounds__(kThreads)
    label_mask_local_static_kernel(const LabelConst c, const int* __restrict__ mask,
                                   int* __restrict__ parent, int* __restrict__ count,
                                   long long* __restrict__ area6) {
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
        count[flat] = 0;
        area6[flat] = 0;
      }
    }
    lab[li] = u ? li : -1;
  }
  local_ccl(lab, c.connectivity, gy0, gx0, c.nx, parent);
}

// Region count / total / winner over the root list (count and area only).
__global__ void __launch_bounds__(kThreads)
    label_reduce_static_kernel(const int* __restrict__ count, const long long* __restrict__ area6,
                               const int* __restrict__ root_list, LabelOut* out,
                               unsigned int* arrive) {
  const int nroots = out->root_count;
  unsigned long long best = 0;
  int total = 0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nroots; k += gridDim.x * blockDim.x) {
    const int root = root_list[k];
    const int cnt = count[root];
    total += cnt;
    const unsigned long long key = ((unsigned long long)(unsigned)cnt << 32) |
                                   (unsigned long long)(0x7fffffffu - (unsigned)root);
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
  if (!last || threadIdx.x != 0) return;
  __threadfence();
  *arrive = 0;
  out->regions = nroots;
  const unsigned long long key = *(volatile unsigned long long*)&out->best_key;
  if (key == 0) {
    out->largest = 0;
    out->winner = -1;
    return;
  }
  const int winner = (int)(0x7fffffffu - (unsigned)(key & 0xffffffffu));
  out->largest = (int)(key >> 32);
  out->winner = winner;
  out->area6 = area6[winner];
}

}  // namespace

extern "C" int sb_label_mask_static(const int32_t* d_mask, int32_t* d_labels, int ny, int nx,
                                    int connectivity, double dx_m, double dy_m, void* stream,
                                    sb_label_stats* out) {
  if (!d_mask || !d_labels || !out || ny < 1 || nx < 1) return SB_ERR_BAD_ARG;
  if (connectivity != 4 && connectivity != 8) return SB_ERR_BAD_ARG;
  if ((long long)ny * nx > kStaticLabelMaxCells) return SB_ERR_CAPACITY;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return SB_ERR_CUDA;
  unsigned char* base = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_label_scratch_mutex);
    if (!g_label_scratch_ptr[dev]) {
      // one-time set-up on this device (the device is current): the host-side
      // symbol is only a stand-in, the kernels need its device address
      void* p = nullptr;
      if (cudaGetSymbolAddress(&p, g_label_scratch) != cudaSuccess || !p) return SB_ERR_CUDA;
      g_label_scratch_ptr[dev] = static_cast<unsigned char*>(p);
    }
    base = g_label_scratch_ptr[dev];
  }
  LabelOut* lout = reinterpret_cast<LabelOut*>(base);
  unsigned int* arrive = reinterpret_cast<unsigned int*>(base + sizeof(LabelOut));
  int* count = reinterpret_cast<int*>(base + kStaticCountOffset);
  long long* area6 = reinterpret_cast<long long*>(base + kStaticAreaOffset);
  int* root_list = reinterpret_cast<int*>(base + kStaticRootOffset);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  LabelConst c{};
  c.ny = ny;
  c.nx = nx;
  c.pitch = nx;
  c.tiles_x = (nx + kLabelTile - 1) / kLabelTile;
  c.connectivity = connectivity;
  LabelRoots roots{};
  roots.count = count;
  roots.area6 = area6;
  if (cudaMemsetAsync(base, 0, kStaticHeaderBytes, s) != cudaSuccess) return SB_ERR_CUDA;
  const int tiles = c.tiles_x * ((ny + kLabelTile - 1) / kLabelTile);
  label_mask_local_static_kernel<<<tiles, kThreads, 0, s>>>(c, d_mask, d_labels, count, area6);
  label_merge_kernel<<<tiles, kThreads, 0, s>>>(c, d_labels, lout);
  label_compress_kernel<true><<<grid_for((long long)ny * nx), kThreads, 0, s>>>(
      c, d_labels, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, roots, root_list, lout, 1);
  label_reduce_static_kernel<<<148, kThreads, 0, s>>>(count, area6, root_list, lout, arrive);
  if (cudaGetLastError() != cudaSuccess) return SB_ERR_CUDA;
  LabelOut host;
  if (cudaMemcpyAsync(&host, lout, sizeof(LabelOut), cudaMemcpyDeviceToHost, s) != cudaSuccess)
    return SB_ERR_CUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return SB_ERR_CUDA;
  std::memset(out, 0, sizeof(*out));
  out->status = host.status;
  out->unstable_cell_count = host.total_unstable;
  out->connected_region_count = host.regions;
  out->largest_connected_cell_count = host.largest;
  out->winner_root = host.winner;
  out->union_passes = 2;
  out->largest_connected_area_m2 = (double)host.area6 * (dx_m * dy_m / 6.0);
  return host.status ? SB_ERR_NONCONVERGENCE : SB_OK;
}

#include "sb_batch_host.cuh"
#include "sb_learned_host.cuh"
