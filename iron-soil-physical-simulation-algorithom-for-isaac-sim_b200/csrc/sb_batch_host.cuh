// Host side of the batched patch runtime (C ABI sb_batch_*), included by
// soilb200.cu after the single-grid entry points so that it shares their
// helpers (fill_ledger_geom, grid_for, the field conversion kernels).
#pragma once

struct sb_batch {
  int device = 0;
  int npatch = 0;
  cudaStream_t stream = nullptr;
  std::vector<sb_patch_desc> desc;
  std::vector<long long> base;
  std::vector<int> pitch, rows, parity;
  long long elems = 0;
  int32_t* b = nullptr;
  int32_t* z = nullptr;
  int32_t* h[2] = {nullptr, nullptr};
  float* qx[2] = {nullptr, nullptr};
  float* qy[2] = {nullptr, nullptr};
  double* staging = nullptr;
  int* range_error = nullptr;
  sb::BatchPatch* d_patches = nullptr;
  int* d_item_patch = nullptr;
  int* d_band_patch = nullptr;
  int nitems = 0, nbands = 0, item_cap = 0, band_cap = 0;
  sb::BatchCtl* d_ctl = nullptr;
  sb::BatchCtl* h_ctl = nullptr;
  sb::BatchGlobal* d_g = nullptr;
  double* d_item_partials = nullptr;
  double* d_band_partials = nullptr;
  long long* d_band_ipartials = nullptr;
  double* dt_dev = nullptr;
  double* dt_host = nullptr;
  cudaEvent_t ev[2] = {nullptr, nullptr};
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  sb_mobile_params key{};
  int rows_version = 0;
  int graph_rows_version = -1;
  long long launches = 0;
  // per-patch labelling (sb_batch_label): scratch for the largest patch,
  // reused patch by patch, and the labels of every patch (flat ny*nx each)
  long long max_cells = 0;
  int* lab_parent = nullptr;
  float* lab_slope = nullptr;
  float* lab_severity = nullptr;
  int* lab_zero_i = nullptr;        // latch / previous component: all zero in a batch
  double* lab_zero_d = nullptr;     // export ledgers: all zero
  sb::LabelRoots lab_roots{};
  int* lab_root_list = nullptr;
  sb::LabelOut* lab_out = nullptr;  // one record per patch
  sb::LabelOut* lab_out_host = nullptr;
  unsigned int* lab_arrive = nullptr;
  int32_t* labels = nullptr;
  std::vector<long long> label_base;
  char err[512] = {0};
};

namespace {

using namespace sb;

int bfail(sb_batch* bt, int code, const char* fmt, ...) {
  if (bt) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(bt->err, sizeof(bt->err), fmt, ap);
    va_end(ap);
  }
  return code;
}

#define SB_BCUDA(bt, call)                                                                   \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess) {                                                                 \
      cudaGetLastError(); /* a failed call must not surface again in a later check */       \
      return bfail((bt), SB_ERR_CUDA, "CUDA error %s at %s:%d (%s)", cudaGetErrorString(e_), \
                   __FILE__, __LINE__, #call);                                               \
    }                                                                                        \
  } while (0)

constexpr int kBatchMinRows = 4;
constexpr int kBatchMaxRows = 256;

FvConst batch_patch_const(const sb_patch_desc& d, int pitch, int rows, const sb_mobile_params* p) {
  FvConst c{};
  c.ny = d.ny;
  c.nx = d.nx;
  c.pitch = pitch;
  c.tiles_x = (d.nx + kStripOut - 1) / kStripOut;
  c.rows_per_warp = rows;
  c.dx = d.dx_m;
  c.dy = d.dy_m;
  c.K = p->earth_pressure_coefficient;
  c.g = p->gravity_m_s2;
  c.cfl = p->cfl;
  c.dry = p->dry_tolerance_m;
  c.mu_g = p->basal_friction_coefficient * p->gravity_m_s2;
  c.c_half = 0.5 * p->earth_pressure_coefficient * p->gravity_m_s2;
  c.kg = p->earth_pressure_coefficient * p->gravity_m_s2;
  c.min_spacing = d.dx_m < d.dy_m ? d.dx_m : d.dy_m;
  c.Q = std::ldexp(1.0, -d.height_exponent);
  c.gsx[0] = c.Q / (2.0 * c.dx);
  c.gsx[1] = c.Q / c.dx;
  c.gsy[0] = c.Q / (2.0 * c.dy);
  c.gsy[1] = c.Q / c.dy;
  c.Kf = (float)c.K;
  c.KGf = (float)c.kg;
  c.HKGf = (float)c.c_half;
  c.Qf = (float)c.Q;
  c.invQf = (float)(1.0 / c.Q);
  c.dryf = (float)c.dry;
  c.QKf = (float)(c.Q / c.K);
  c.max_substeps = p->maximum_substeps;
  c.has_external = 0;
  return c;
}

// Patch table, FV work items and ledger bands for the current rows and params.
int batch_tables(sb_batch* bt, const sb_mobile_params* p) {
  std::vector<BatchPatch> table(bt->npatch);
  std::vector<int> item_patch, band_patch;
  const double static_limit = std::tan(p->start_angle_deg * (M_PI / 180.0)) + 1.0e-14;
  for (int i = 0; i < bt->npatch; ++i) {
    const sb_patch_desc& d = bt->desc[i];
    BatchPatch& P = table[i];
    P.c = batch_patch_const(d, bt->pitch[i], bt->rows[i], p);
    P.base = bt->base[i];
    P.datum = d.datum_m;
    P.static_limit = static_limit;
    const int chunks = (d.ny + bt->rows[i] - 1) / bt->rows[i];
    P.first_item = (int)item_patch.size();
    P.n_items = P.c.tiles_x * chunks;
    item_patch.insert(item_patch.end(), P.n_items, i);
    P.first_band = (int)band_patch.size();
    P.n_bands = (d.ny + kBandRows - 1) / kBandRows;
    band_patch.insert(band_patch.end(), P.n_bands, i);
  }
  bt->nitems = (int)item_patch.size();
  bt->nbands = (int)band_patch.size();
  if (bt->nitems > bt->item_cap) {
    cudaFree(bt->d_item_patch);
    cudaFree(bt->d_item_partials);
    bt->d_item_patch = nullptr;
    bt->d_item_partials = nullptr;
    SB_BCUDA(bt, cudaMalloc(&bt->d_item_patch, (size_t)bt->nitems * sizeof(int)));
    SB_BCUDA(bt, cudaMalloc(&bt->d_item_partials, (size_t)bt->nitems * (kFvDiag + 1) * sizeof(double)));
    bt->item_cap = bt->nitems;
  }
  if (bt->nbands > bt->band_cap) {
    cudaFree(bt->d_band_patch);
    cudaFree(bt->d_band_partials);
    cudaFree(bt->d_band_ipartials);
    bt->d_band_patch = nullptr;
    bt->d_band_partials = nullptr;
    bt->d_band_ipartials = nullptr;
    SB_BCUDA(bt, cudaMalloc(&bt->d_band_patch, (size_t)bt->nbands * sizeof(int)));
    SB_BCUDA(bt, cudaMalloc(&bt->d_band_partials, (size_t)bt->nbands * L_NP * sizeof(double)));
    SB_BCUDA(bt, cudaMalloc(&bt->d_band_ipartials, (size_t)bt->nbands * kLedgerI64 * sizeof(long long)));
    bt->band_cap = bt->nbands;
  }
  SB_BCUDA(bt, cudaMemcpyAsync(bt->d_patches, table.data(), table.size() * sizeof(BatchPatch),
                               cudaMemcpyHostToDevice, bt->stream));
  SB_BCUDA(bt, cudaMemcpyAsync(bt->d_item_patch, item_patch.data(), item_patch.size() * sizeof(int),
                               cudaMemcpyHostToDevice, bt->stream));
  SB_BCUDA(bt, cudaMemcpyAsync(bt->d_band_patch, band_patch.data(), band_patch.size() * sizeof(int),
                               cudaMemcpyHostToDevice, bt->stream));
  SB_BCUDA(bt, cudaStreamSynchronize(bt->stream));
  return SB_OK;
}

int badd_kernel(sb_batch* bt, cudaGraph_t g, cudaGraphNode_t* node, const cudaGraphNode_t* deps,
                size_t ndeps, void* func, dim3 grid, void** args) {
  cudaKernelNodeParams kp{};
  kp.func = func;
  kp.gridDim = grid;
  kp.blockDim = dim3(kThreads);
  kp.sharedMemBytes = 0;
  kp.kernelParams = args;
  SB_BCUDA(bt, cudaGraphAddKernelNode(node, g, deps, ndeps, &kp));
  return SB_OK;
}

// begin -> ledger(before) -> finish(prologue, sets the loop condition) -> ev0
// -> while { strips of all active patches -> per-patch round } -> ev1
// -> ledger(after) -> finish
int batch_build_graph(sb_batch* bt) {
  if (bt->exec) cudaGraphExecDestroy(bt->exec);
  if (bt->graph) cudaGraphDestroy(bt->graph);
  bt->exec = nullptr;
  bt->graph = nullptr;
  cudaGraph_t g;
  SB_BCUDA(bt, cudaGraphCreate(&g, 0));
  bt->graph = g;
  cudaGraphConditionalHandle handle;
  SB_BCUDA(bt, cudaGraphConditionalHandleCreate(&handle, g, 0, cudaGraphCondAssignDefault));
  BatchArena a{bt->b, bt->z, {bt->h[0], bt->h[1]}, {bt->qx[0], bt->qx[1]}, {bt->qy[0], bt->qy[1]}};
  int npatch = bt->npatch, nbands = bt->nbands, nitems = bt->nitems;
  int mode0 = 0, mode1 = 1, use1 = 1, use0 = 0;
  const dim3 gp((npatch + kThreads - 1) / kThreads);
  const dim3 gw((npatch + kThreads / 32 - 1) / (kThreads / 32));
  const dim3 gb(nbands);
  const dim3 gi((nitems + kThreads / 32 - 1) / (kThreads / 32));
  cudaGraphNode_t n0, n1, n2, ne0, nloop, ne1, n3, n4, nb1, nb2;
  int rc;
  {
    void* args[] = {&npatch, &bt->d_ctl, &bt->dt_dev};
    if ((rc = badd_kernel(bt, g, &n0, nullptr, 0, (void*)batch_begin_kernel, gp, args))) return rc;
  }
  {
    void* args[] = {&bt->d_patches, &bt->d_band_patch, &nbands, &a, &bt->d_ctl,
                    &bt->d_band_partials, &bt->d_band_ipartials};
    if ((rc = badd_kernel(bt, g, &n1, &n0, 1, (void*)batch_ledger_kernel, gb, args))) return rc;
  }
  {
    void* args[] = {&npatch, &bt->d_patches, &bt->d_ctl, &bt->d_band_partials,
                    &bt->d_band_ipartials, &mode0, &bt->d_g, &handle, &use1};
    if ((rc = badd_kernel(bt, g, &n2, &n1, 1, (void*)batch_ledger_finish_kernel, gw, args)))
      return rc;
  }
  SB_BCUDA(bt, cudaGraphAddEventRecordNode(&ne0, g, &n2, 1, bt->ev[0]));
  {
    cudaGraphNodeParams cp{};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = handle;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    SB_BCUDA(bt, cudaGraphAddNode(&nloop, g, &ne0, 1, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    void* fargs[] = {&bt->d_patches, &bt->d_item_patch, &nitems, &a, &bt->d_ctl,
                     &bt->d_item_partials};
    // production: the FMA-contracted fast kernel; SOILB200_FV_EXACT=1 selects
    // the CPU mirror's IEEE arithmetic (as for the single-grid kernel)
    const char* exact_env = std::getenv("SOILB200_FV_EXACT");
    void* fv = (exact_env && exact_env[0] == '1') ? (void*)batch_fv_kernel<false>
                                                  : const_cast<void*>(batch_fv_fast_kernel());
    if ((rc = badd_kernel(bt, body, &nb1, nullptr, 0, fv, gi, fargs))) return rc;
    void* rargs[] = {&npatch, &bt->d_patches, &bt->d_ctl, &bt->d_item_partials, &bt->d_g,
                     &handle, &use1};
    if ((rc = badd_kernel(bt, body, &nb2, &nb1, 1, (void*)batch_round_kernel, gw, rargs))) return rc;
  }
  SB_BCUDA(bt, cudaGraphAddEventRecordNode(&ne1, g, &nloop, 1, bt->ev[1]));
  {
    void* args[] = {&bt->d_patches, &bt->d_band_patch, &nbands, &a, &bt->d_ctl,
                    &bt->d_band_partials, &bt->d_band_ipartials};
    if ((rc = badd_kernel(bt, g, &n3, &ne1, 1, (void*)batch_ledger_kernel, gb, args))) return rc;
  }
  {
    void* args[] = {&npatch, &bt->d_patches, &bt->d_ctl, &bt->d_band_partials,
                    &bt->d_band_ipartials, &mode1, &bt->d_g, &handle, &use0};
    if ((rc = badd_kernel(bt, g, &n4, &n3, 1, (void*)batch_ledger_finish_kernel, gw, args)))
      return rc;
  }
  SB_BCUDA(bt, cudaGraphInstantiate(&bt->exec, g, 0));
  return SB_OK;
}

int batch_check_params(sb_batch* bt, const sb_mobile_params* p) {
  const double vals[] = {p->gravity_m_s2, p->earth_pressure_coefficient, p->cfl,
                         p->dry_tolerance_m, p->basal_friction_coefficient};
  for (double v : vals)
    if (!std::isfinite(v) || v <= 0.0)
      return bfail(bt, SB_ERR_BAD_ARG, "MobileV2 configuration must be finite/positive");
  if (p->use_external)
    return bfail(bt, SB_ERR_BAD_ARG, "[soilb200] batched patches take no external acceleration");
  return SB_OK;
}

void* batch_field(sb_batch* bt, int patch, int field, int* kind) {
  // kind: 0 support quanta (datum), 1 height quanta, 2 float
  const long long base = bt->base[patch];
  const int par = bt->parity[patch];
  switch (field) {
    case SB_FIELD_Z_BASE: *kind = 0; return bt->z + base;
    case SB_FIELD_B_EFF: *kind = 0; return bt->b + base;
    case SB_FIELD_MOBILE: *kind = 1; return bt->h[par] + base;
    case SB_FIELD_MOMENTUM_X: *kind = 2; return bt->qx[par] + base;
    case SB_FIELD_MOMENTUM_Y: *kind = 2; return bt->qy[par] + base;
    default: return nullptr;
  }
}

}  // namespace

extern "C" {

int sb_batch_create(int device, int n_patches, const sb_patch_desc* patches, sb_batch** out) {
  if (!out) return SB_ERR_BAD_ARG;
  *out = nullptr;
  if (n_patches <= 0 || n_patches > (1 << 20) || !patches) return SB_ERR_BAD_ARG;
  for (int i = 0; i < n_patches; ++i) {
    const sb_patch_desc& d = patches[i];
    if (d.ny < 2 || d.nx < 2 || (long long)d.ny * d.nx > (1LL << 28) || !(d.dx_m > 0.0) ||
        !(d.dy_m > 0.0) || !std::isfinite(d.dx_m) || !std::isfinite(d.dy_m) ||
        d.height_exponent < 4 || d.height_exponent > 40 || !std::isfinite(d.datum_m))
      return SB_ERR_BAD_ARG;
  }
  sb_batch* bt = new sb_batch();
  *out = bt;
  bt->device = device;
  bt->npatch = n_patches;
  bt->desc.assign(patches, patches + n_patches);
  SB_BCUDA(bt, cudaSetDevice(device));
  SB_BCUDA(bt, cudaStreamCreateWithFlags(&bt->stream, cudaStreamNonBlocking));
  long long off = 0, max_cells = 0;
  for (int i = 0; i < n_patches; ++i) {
    const int pitch = (bt->desc[i].nx + 31) / 32 * 32;  // 128-byte aligned rows
    bt->pitch.push_back(pitch);
    bt->base.push_back(off);
    off += (long long)pitch * bt->desc[i].ny;
    max_cells = std::max(max_cells, (long long)bt->desc[i].ny * bt->desc[i].nx);
    bt->label_base.push_back(bt->label_base.empty()
                                 ? 0
                                 : bt->label_base.back() +
                                       (long long)bt->desc[i - 1].ny * bt->desc[i - 1].nx);
    bt->rows.push_back(16);
    bt->parity.push_back(0);
  }
  bt->elems = off;
  bt->max_cells = max_cells;
  const size_t bytes = (size_t)off * 4;
  void** fields[] = {(void**)&bt->b, (void**)&bt->z, (void**)&bt->h[0], (void**)&bt->h[1],
                     (void**)&bt->qx[0], (void**)&bt->qx[1], (void**)&bt->qy[0], (void**)&bt->qy[1]};
  for (void** f : fields) {
    SB_BCUDA(bt, cudaMalloc(f, bytes));
    SB_BCUDA(bt, cudaMemsetAsync(*f, 0, bytes, bt->stream));
  }
  SB_BCUDA(bt, cudaMalloc(&bt->staging, (size_t)max_cells * sizeof(double)));
  SB_BCUDA(bt, cudaMalloc(&bt->range_error, sizeof(int)));
  SB_BCUDA(bt, cudaMalloc(&bt->d_patches, (size_t)n_patches * sizeof(BatchPatch)));
  SB_BCUDA(bt, cudaMalloc(&bt->d_ctl, (size_t)n_patches * sizeof(BatchCtl)));
  SB_BCUDA(bt, cudaMemsetAsync(bt->d_ctl, 0, (size_t)n_patches * sizeof(BatchCtl), bt->stream));
  SB_BCUDA(bt, cudaMallocHost(&bt->h_ctl, (size_t)n_patches * sizeof(BatchCtl)));
  SB_BCUDA(bt, cudaMalloc(&bt->d_g, sizeof(BatchGlobal)));
  SB_BCUDA(bt, cudaMemsetAsync(bt->d_g, 0, sizeof(BatchGlobal), bt->stream));
  SB_BCUDA(bt, cudaMalloc(&bt->dt_dev, sizeof(double)));
  SB_BCUDA(bt, cudaMallocHost(&bt->dt_host, sizeof(double)));
  SB_BCUDA(bt, cudaEventCreate(&bt->ev[0]));
  SB_BCUDA(bt, cudaEventCreate(&bt->ev[1]));
  SB_BCUDA(bt, cudaStreamSynchronize(bt->stream));
  return SB_OK;
}

int sb_batch_destroy(sb_batch* bt) {
  if (!bt) return SB_OK;
  cudaSetDevice(bt->device);
  if (bt->stream) cudaStreamSynchronize(bt->stream);
  if (bt->exec) cudaGraphExecDestroy(bt->exec);
  if (bt->graph) cudaGraphDestroy(bt->graph);
  void* dev[] = {bt->b, bt->z, bt->h[0], bt->h[1], bt->qx[0], bt->qx[1], bt->qy[0], bt->qy[1],
                 bt->staging, bt->range_error, bt->d_patches, bt->d_item_patch, bt->d_band_patch,
                 bt->d_ctl, bt->d_g, bt->d_item_partials, bt->d_band_partials,
                 bt->d_band_ipartials, bt->dt_dev, bt->lab_parent, bt->lab_slope,
                 bt->lab_severity, bt->lab_zero_i, bt->lab_zero_d, bt->lab_roots.count,
                 bt->lab_roots.area6, bt->lab_roots.volume, bt->lab_roots.exc_start,
                 bt->lab_roots.exc_stop, bt->lab_roots.max_exc_start, bt->lab_roots.max_exc_stop,
                 bt->lab_roots.prev_overlap, bt->lab_root_list, bt->lab_out, bt->lab_arrive,
                 bt->labels};
  for (void* p : dev)
    if (p) cudaFree(p);
  if (bt->lab_out_host) cudaFreeHost(bt->lab_out_host);
  if (bt->h_ctl) cudaFreeHost(bt->h_ctl);
  if (bt->dt_host) cudaFreeHost(bt->dt_host);
  for (cudaEvent_t e : bt->ev)
    if (e) cudaEventDestroy(e);
  if (bt->stream) cudaStreamDestroy(bt->stream);
  delete bt;
  return SB_OK;
}

int sb_batch_upload(sb_batch* bt, int patch, int field, const double* host) {
  if (!bt || !host) return SB_ERR_BAD_ARG;
  if (patch < 0 || patch >= bt->npatch)
    return bfail(bt, SB_ERR_BAD_ARG, "[soilb200] patch %d out of range", patch);
  int kind = 0;
  void* dst = batch_field(bt, patch, field, &kind);
  if (!dst) return bfail(bt, SB_ERR_BAD_ARG, "[soilb200] field %d is not a patch field", field);
  SB_BCUDA(bt, cudaSetDevice(bt->device));
  const sb_patch_desc& d = bt->desc[patch];
  SB_BCUDA(bt, cudaMemcpyAsync(bt->staging, host, (size_t)d.ny * d.nx * 8, cudaMemcpyHostToDevice,
                               bt->stream));
  const int grid = grid_for((long long)d.ny * d.nx);
  if (kind == 2) {
    to_float_kernel<<<grid, kThreads, 0, bt->stream>>>(bt->staging, (float*)dst, d.ny, d.nx,
                                                        bt->pitch[patch]);
    bt->launches++;
    SB_BCUDA(bt, cudaGetLastError());
    SB_BCUDA(bt, cudaStreamSynchronize(bt->stream));
    return SB_OK;
  }
  SB_BCUDA(bt, cudaMemsetAsync(bt->range_error, 0, sizeof(int), bt->stream));
  to_fixed_kernel<<<grid, kThreads, 0, bt->stream>>>(bt->staging, (int32_t*)dst, d.ny, d.nx,
                                                      bt->pitch[patch], kind == 0 ? d.datum_m : 0.0,
                                                      std::ldexp(1.0, d.height_exponent),
                                                      bt->range_error);
  bt->launches++;
  SB_BCUDA(bt, cudaGetLastError());
  int herr = 0;
  SB_BCUDA(bt, cudaMemcpyAsync(&herr, bt->range_error, sizeof(int), cudaMemcpyDeviceToHost, bt->stream));
  SB_BCUDA(bt, cudaStreamSynchronize(bt->stream));
  if (herr)
    return bfail(bt, SB_ERR_RANGE,
                 "[soilb200] patch %d field %d exceeds the fixed-point range (2^31 quanta of 2^-%d m)",
                 patch, field, d.height_exponent);
  return SB_OK;
}

int sb_batch_download(sb_batch* bt, int patch, int field, double* host) {
  if (!bt || !host) return SB_ERR_BAD_ARG;
  if (patch < 0 || patch >= bt->npatch)
    return bfail(bt, SB_ERR_BAD_ARG, "[soilb200] patch %d out of range", patch);
  int kind = 0;
  void* src = batch_field(bt, patch, field, &kind);
  if (!src) return bfail(bt, SB_ERR_BAD_ARG, "[soilb200] field %d is not a patch field", field);
  SB_BCUDA(bt, cudaSetDevice(bt->device));
  const sb_patch_desc& d = bt->desc[patch];
  const int grid = grid_for((long long)d.ny * d.nx);
  if (kind == 2)
    from_float_kernel<<<grid, kThreads, 0, bt->stream>>>((const float*)src, bt->staging, d.ny, d.nx,
                                                          bt->pitch[patch]);
  else
    from_fixed_kernel<<<grid, kThreads, 0, bt->stream>>>((const int32_t*)src, bt->staging, d.ny,
                                                          d.nx, bt->pitch[patch],
                                                          kind == 0 ? d.datum_m : 0.0,
                                                          std::ldexp(1.0, -d.height_exponent));
  bt->launches++;
  SB_BCUDA(bt, cudaGetLastError());
  SB_BCUDA(bt, cudaMemcpyAsync(host, bt->staging, (size_t)d.ny * d.nx * 8, cudaMemcpyDeviceToHost,
                               bt->stream));
  SB_BCUDA(bt, cudaStreamSynchronize(bt->stream));
  return SB_OK;
}

int sb_batch_set_rows(sb_batch* bt, const int* rows_per_warp) {
  if (!bt || !rows_per_warp) return SB_ERR_BAD_ARG;
  for (int i = 0; i < bt->npatch; ++i)
    if (rows_per_warp[i] < kBatchMinRows || rows_per_warp[i] > kBatchMaxRows)
      return bfail(bt, SB_ERR_BAD_ARG, "[soilb200] rows per warp must be in [%d, %d]",
                   kBatchMinRows, kBatchMaxRows);
  bt->rows.assign(rows_per_warp, rows_per_warp + bt->npatch);
  bt->rows_version++;
  return SB_OK;
}

int sb_batch_get_rows(sb_batch* bt, int* rows_per_warp) {
  if (!bt || !rows_per_warp) return SB_ERR_BAD_ARG;
  std::copy(bt->rows.begin(), bt->rows.end(), rows_per_warp);
  return SB_OK;
}

int sb_batch_step(sb_batch* bt, double dt_s, const sb_mobile_params* params,
                  sb_mobile_stats* per_patch) {
  if (!bt || !params || !per_patch) return SB_ERR_BAD_ARG;
  if (!std::isfinite(dt_s) || dt_s <= 0.0) return bfail(bt, SB_ERR_BAD_ARG, "dt must be finite/positive");
  int rc = batch_check_params(bt, params);
  if (rc) return rc;
  SB_BCUDA(bt, cudaSetDevice(bt->device));
  if (!bt->exec || std::memcmp(&bt->key, params, sizeof(sb_mobile_params)) != 0 ||
      bt->graph_rows_version != bt->rows_version) {
    if ((rc = batch_tables(bt, params))) return rc;
    if ((rc = batch_build_graph(bt))) return rc;
    bt->key = *params;
    bt->graph_rows_version = bt->rows_version;
  }
  *bt->dt_host = dt_s;
  SB_BCUDA(bt, cudaMemcpyAsync(bt->dt_dev, bt->dt_host, sizeof(double), cudaMemcpyHostToDevice,
                               bt->stream));
  SB_BCUDA(bt, cudaGraphLaunch(bt->exec, bt->stream));
  SB_BCUDA(bt, cudaMemcpyAsync(bt->h_ctl, bt->d_ctl, (size_t)bt->npatch * sizeof(BatchCtl),
                               cudaMemcpyDeviceToHost, bt->stream));
  SB_BCUDA(bt, cudaStreamSynchronize(bt->stream));
  float loop_ms = 0.f;
  SB_BCUDA(bt, cudaEventElapsedTime(&loop_ms, bt->ev[0], bt->ev[1]));
  int rounds = 0, bad = -1;
  for (int i = 0; i < bt->npatch; ++i) {
    const BatchCtl& B = bt->h_ctl[i];
    const FvControl& k = B.k;
    const sb_patch_desc& d = bt->desc[i];
    sb_mobile_stats* out = per_patch + i;
    std::memset(out, 0, sizeof(*out));
    out->substep_loop_ms = loop_ms;
    out->substeps = k.substeps;
    out->static_skip = k.static_skip;
    out->cfl_limited = k.cfl_limited;
    out->status = k.status;
    out->maximum_cfl = k.max_cfl;
    const double area = d.dx_m * d.dy_m;
    for (int j = 0; j < 2; ++j) {
      out->conservative_impulse_m4_s[j] = k.diag[j] * area;
      out->external_impulse_m4_s[j] = k.diag[2 + j] * area;
      out->friction_impulse_m4_s[j] = k.diag[4 + j] * area;
    }
    out->friction_dissipation = k.diag[6] * area;
    out->external_work = k.diag[7] * area;
    const double q = std::ldexp(1.0, -d.height_exponent);
    fill_ledger_geom(true, d.dx_m, d.dy_m, q, B.before, params, &out->before);
    fill_ledger_geom(true, d.dx_m, d.dy_m, q, B.after, params, &out->after);
    bt->parity[i] = k.parity;
    rounds = std::max(rounds, k.substeps);
    if (k.status != 0 && bad < 0) bad = i;
  }
  bt->launches += 5 + 2LL * rounds;
  if (bad >= 0) {
    const int st = bt->h_ctl[bad].k.status;
    if (st == SB_ERR_SUBSTEP_CAP)
      return bfail(bt, SB_ERR_SUBSTEP_CAP, "MobileV2 maximum_substeps exceeded (patch %d)", bad);
    return bfail(bt, st, "[soilb200] device status %d (patch %d)", st, bad);
  }
  return SB_OK;
}

// Chooses rows per warp for each group of patches with the same row count:
// every candidate is timed on the live state, which is copied first and put
// back after each trial; groups are tuned one after another, keeping the best
// choice so far for the others.
int sb_batch_autotune(sb_batch* bt, double dt_s, const sb_mobile_params* params, int trials,
                      double* best_ms) {
  if (!bt || !params || trials <= 0) return SB_ERR_BAD_ARG;
  SB_BCUDA(bt, cudaSetDevice(bt->device));
  static const int cand[] = {4, 8, 16, 32, 64};
  const size_t bytes = (size_t)bt->elems * 4;
  void* save[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  void* live[6] = {bt->h[0], bt->h[1], bt->qx[0], bt->qx[1], bt->qy[0], bt->qy[1]};
  for (int i = 0; i < 6; ++i) {
    if (cudaMalloc(&save[i], bytes) != cudaSuccess) {
      for (int j = 0; j < i; ++j) cudaFree(save[j]);
      return bfail(bt, SB_ERR_CUDA, "[soilb200] autotune snapshot allocation failed");
    }
    SB_BCUDA(bt, cudaMemcpyAsync(save[i], live[i], bytes, cudaMemcpyDeviceToDevice, bt->stream));
  }
  std::vector<BatchCtl> ctl_save(bt->npatch);
  SB_BCUDA(bt, cudaMemcpyAsync(ctl_save.data(), bt->d_ctl, (size_t)bt->npatch * sizeof(BatchCtl),
                               cudaMemcpyDeviceToHost, bt->stream));
  SB_BCUDA(bt, cudaStreamSynchronize(bt->stream));
  const std::vector<int> parity_save = bt->parity;
  std::vector<sb_mobile_stats> stats(bt->npatch);
  std::vector<int> groups;
  for (const auto& d : bt->desc)
    if (std::find(groups.begin(), groups.end(), d.ny) == groups.end()) groups.push_back(d.ny);
  std::vector<int> best = bt->rows;
  double best_t = 0.0;
  int rc = SB_OK;
  auto restore = [&]() -> int {
    for (int i = 0; i < 6; ++i)
      SB_BCUDA(bt, cudaMemcpyAsync(live[i], save[i], bytes, cudaMemcpyDeviceToDevice, bt->stream));
    SB_BCUDA(bt, cudaMemcpyAsync(bt->d_ctl, ctl_save.data(), (size_t)bt->npatch * sizeof(BatchCtl),
                                 cudaMemcpyHostToDevice, bt->stream));
    SB_BCUDA(bt, cudaStreamSynchronize(bt->stream));
    bt->parity = parity_save;
    return SB_OK;
  };
  auto timed = [&](const std::vector<int>& rows, double* ms) -> int {
    int r = sb_batch_set_rows(bt, rows.data());
    if (r) return r;
    double t = 0.0;
    for (int k = 0; k < trials && !r; ++k) {
      r = sb_batch_step(bt, dt_s, params, stats.data());
      t += stats[0].substep_loop_ms;
    }
    const int r2 = restore();
    *ms = t;
    return r ? r : r2;
  };
  if ((rc = timed(best, &best_t)) == SB_OK) {
    for (int ny : groups) {
      for (int c : cand) {
        std::vector<int> trial = best;
        bool changed = false;
        for (int i = 0; i < bt->npatch; ++i)
          if (bt->desc[i].ny == ny && trial[i] != c) {
            trial[i] = c;
            changed = true;
          }
        if (!changed) continue;
        double t = 0.0;
        if ((rc = timed(trial, &t))) break;
        if (t < best_t) {
          best_t = t;
          best = trial;
        }
      }
      if (rc) break;
    }
  }
  for (void* p : save) cudaFree(p);
  if (rc) return rc;
  if (best_ms) *best_ms = best_t / trials;
  return sb_batch_set_rows(bt, best.data());
}

// Per-patch labelling: the single-grid yield + union-find kernels run patch by
// patch on the batch arena (each patch's current ping-pong buffer, its own
// quantum and datum), scratch reused, labels kept per patch.
static int batch_label_alloc(sb_batch* bt) {
  if (bt->lab_parent) return SB_OK;
  const size_t n = (size_t)bt->max_cells;
  long long total = 0;
  for (int i = 0; i < bt->npatch; ++i) total += (long long)bt->desc[i].ny * bt->desc[i].nx;
  SB_BCUDA(bt, cudaMalloc(&bt->lab_parent, n * 4));
  SB_BCUDA(bt, cudaMalloc(&bt->lab_slope, n * 4));
  SB_BCUDA(bt, cudaMalloc(&bt->lab_severity, n * 4));
  SB_BCUDA(bt, cudaMalloc(&bt->lab_zero_i, n * 4));
  SB_BCUDA(bt, cudaMemsetAsync(bt->lab_zero_i, 0, n * 4, bt->stream));
  SB_BCUDA(bt, cudaMalloc(&bt->lab_zero_d, n * 8));
  SB_BCUDA(bt, cudaMemsetAsync(bt->lab_zero_d, 0, n * 8, bt->stream));
  SB_BCUDA(bt, cudaMalloc(&bt->lab_roots.count, n * 4));
  SB_BCUDA(bt, cudaMalloc(&bt->lab_roots.area6, n * 8));
  SB_BCUDA(bt, cudaMalloc(&bt->lab_roots.volume, n * 8));
  SB_BCUDA(bt, cudaMalloc(&bt->lab_roots.exc_start, n * 8));
  SB_BCUDA(bt, cudaMalloc(&bt->lab_roots.exc_stop, n * 8));
  SB_BCUDA(bt, cudaMalloc(&bt->lab_roots.max_exc_start, n * 8));
  SB_BCUDA(bt, cudaMalloc(&bt->lab_roots.max_exc_stop, n * 8));
  SB_BCUDA(bt, cudaMalloc(&bt->lab_roots.prev_overlap, n * 4));
  SB_BCUDA(bt, cudaMalloc(&bt->lab_root_list, n * 4));
  SB_BCUDA(bt, cudaMalloc(&bt->lab_out, (size_t)bt->npatch * sizeof(LabelOut)));
  SB_BCUDA(bt, cudaMallocHost(&bt->lab_out_host, (size_t)bt->npatch * sizeof(LabelOut)));
  SB_BCUDA(bt, cudaMalloc(&bt->lab_arrive, sizeof(unsigned int)));
  SB_BCUDA(bt, cudaMemsetAsync(bt->lab_arrive, 0, sizeof(unsigned int), bt->stream));
  SB_BCUDA(bt, cudaMalloc(&bt->labels, (size_t)total * 4));
  return SB_OK;
}

int sb_batch_label(sb_batch* bt, const sb_label_params* p, sb_label_stats* out) {
  if (!bt || !p || !out) return SB_ERR_BAD_ARG;
  if (p->connectivity != 4 && p->connectivity != 8)
    return bfail(bt, SB_ERR_BAD_ARG, "[LargeAvalanche] connectivity must be 4 or 8");
  SB_BCUDA(bt, cudaSetDevice(bt->device));
  int rc = batch_label_alloc(bt);
  if (rc) return rc;
  SB_BCUDA(bt, cudaMemsetAsync(bt->lab_out, 0, (size_t)bt->npatch * sizeof(LabelOut), bt->stream));
  for (int i = 0; i < bt->npatch; ++i) {
    const sb_patch_desc& d = bt->desc[i];
    LabelConst c{};
    c.ny = d.ny;
    c.nx = d.nx;
    c.pitch = bt->pitch[i];
    c.tiles_x = (d.nx + kLabelTile - 1) / kLabelTile;
    c.connectivity = p->connectivity;
    c.dx = d.dx_m;
    c.dy = d.dy_m;
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
    c.Q = std::ldexp(1.0, -d.height_exponent);
    c.datum = d.datum_m;
    c.release_latches = 0;  // no latches in a batch
    const long long base = bt->base[i];
    const int tiles = c.tiles_x * ((d.ny + kLabelTile - 1) / kLabelTile);
    LabelOut* lo = bt->lab_out + i;
    label_init_local_kernel<true><<<tiles, kLabelInitThreads, 0, bt->stream>>>(
        c, bt->b + base, bt->z + base, bt->h[0] + base, bt->h[1] + base, bt->qx[0] + base,
        bt->qx[1] + base, bt->qy[0] + base, bt->qy[1] + base, &bt->d_ctl[i].k, bt->lab_parent,
        bt->lab_slope, bt->lab_severity, bt->lab_zero_i, bt->lab_zero_d, bt->lab_zero_d,
        bt->lab_roots);
    label_merge_kernel<<<tiles, kThreads, 0, bt->stream>>>(c, bt->lab_parent, lo);
    label_compress_kernel<true><<<grid_for((long long)d.ny * d.nx), kThreads, 0, bt->stream>>>(
        c, bt->lab_parent, bt->b + base, bt->z + base, bt->lab_slope, bt->lab_severity,
        bt->lab_zero_i, bt->lab_zero_i, bt->lab_roots, bt->lab_root_list, lo, 0);
    label_reduce_kernel<<<32, kThreads, 0, bt->stream>>>(bt->lab_roots, bt->lab_root_list, lo,
                                                          bt->lab_arrive);
    SB_BCUDA(bt, cudaGetLastError());
    SB_BCUDA(bt, cudaMemcpyAsync(bt->labels + bt->label_base[i], bt->lab_parent,
                                 (size_t)d.ny * d.nx * 4, cudaMemcpyDeviceToDevice, bt->stream));
    bt->launches += 4;
  }
  SB_BCUDA(bt, cudaMemcpyAsync(bt->lab_out_host, bt->lab_out,
                               (size_t)bt->npatch * sizeof(LabelOut), cudaMemcpyDeviceToHost,
                               bt->stream));
  SB_BCUDA(bt, cudaStreamSynchronize(bt->stream));
  int status = SB_OK;
  for (int i = 0; i < bt->npatch; ++i) {
    const LabelOut& o = bt->lab_out_host[i];
    const sb_patch_desc& d = bt->desc[i];
    sb_label_stats& s = out[i];
    std::memset(&s, 0, sizeof(s));
    s.status = o.status;
    s.unstable_cell_count = o.total_unstable;
    s.connected_region_count = o.regions;
    s.largest_connected_cell_count = o.largest;
    s.winner_root = o.winner;
    s.union_passes = 2;
    const double f = d.dx_m * d.dy_m / 6.0;
    s.largest_connected_area_m2 = (double)o.area6 * f;
    s.largest_connected_mobilizable_volume_m3 =
        (double)o.volume * std::ldexp(1.0, -d.height_exponent) * f;
    s.excess_start_sum_rad = (double)o.exc_start / kExcessScale;
    s.excess_start_max_rad = (double)o.max_exc_start / kExcessScale;
    s.excess_stop_sum_rad = (double)o.exc_stop / kExcessScale;
    s.excess_stop_max_rad = (double)o.max_exc_stop / kExcessScale;
    if (o.status && status == SB_OK)
      status = bfail(bt, SB_ERR_NONCONVERGENCE,
                     "NUMERICAL_NONCONVERGENCE: device avalanche connected components (patch %d)",
                     i);
  }
  return status;
}

int sb_batch_download_labels(sb_batch* bt, int patch, int32_t* host) {
  if (!bt || !host || patch < 0 || patch >= bt->npatch) return SB_ERR_BAD_ARG;
  if (!bt->labels) return bfail(bt, SB_ERR_STATE, "[soilb200] sb_batch_label has not run");
  const sb_patch_desc& d = bt->desc[patch];
  SB_BCUDA(bt, cudaMemcpyAsync(host, bt->labels + bt->label_base[patch], (size_t)d.ny * d.nx * 4,
                               cudaMemcpyDeviceToHost, bt->stream));
  SB_BCUDA(bt, cudaStreamSynchronize(bt->stream));
  return SB_OK;
}

int sb_batch_last_error(sb_batch* bt, char* buf, size_t len) {
  if (!bt || !buf || len == 0) return SB_ERR_BAD_ARG;
  std::snprintf(buf, len, "%s", bt->err);
  return SB_OK;
}

int64_t sb_batch_kernel_launch_count(sb_batch* bt) { return bt ? bt->launches : 0; }

void* sb_batch_stream(sb_batch* bt) { return bt ? (void*)bt->stream : nullptr; }

}  // extern "C"
