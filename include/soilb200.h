/*
 * soilb200 -- C ABI of the B200 (sm_100a) Mobile V2 granular-terrain step.
 *
 * Plain C types only; every call returns an int status (SB_OK == 0).  One
 * context owns one terrain grid resident on one GPU: the fields that the
 * reference keeps in DeviceBulkState (z_base, b_eff, mobile, momentum_x,
 * momentum_y; runtime/bulk_state_authority.py:541-619) plus scratch.
 *
 * Two precisions share one API:
 *   SB_FP64  -- double fields; arithmetic mirrors the reference NumPy solver
 *               operation for operation (parity instantiation).
 *   SB_FX32  -- production: heights stored as int32 multiples of a quantum
 *               2^-height_exponent m (b_eff/z_base relative to datum_m),
 *               momentum float32.  Mass moves in whole quanta, so volume is
 *               conserved exactly and ledgers are exact integer sums.
 *
 * Reference interfaces replaced (paths inside the reference project):
 *   sb_ctx_create/destroy, sb_upload/download
 *       DeviceBulkState.__init__ / _upload_full / explicit_host_view
 *       (runtime/bulk_state_authority.py:510-600, :683-704)
 *   sb_mobile_step
 *       MobileV2ReferenceSolver.step (experimental/mobile_v2_reference.py:191-314),
 *       WarpMobileV2ReferenceSolver.step (experimental/mobile_v2_warp.py:251-344),
 *       WarpProductionMobileV2Solver.step_resident
 *       (bulk_interaction/warp_mobile_v2.py:148-245)
 *   sb_ledger
 *       DeviceBulkState.reservoir_reduction (runtime/bulk_state_authority.py:1036-1066)
 *   sb_entrain / sb_deposit
 *       DeviceBulkState.entrain_host_indices / deposit_host_indices
 *       (runtime/bulk_state_authority.py:920-1034)
 *   sb_label
 *       DeviceLargeAvalancheBridge.observe_and_maybe_mobilize, diagnosis part
 *       (runtime/gpu_large_avalanche.py:541-676)
 *   sb_relax_full
 *       slope_model.relax_critical_slope (slope_model.py:273-343)
 *   sb_relax_reached
 *       EventDrivenMinimumSlopeAdapter.solve (solvers/event_driven_slope.py:83-302)
 *   sb_frontier_seed / sb_frontier_run
 *       EarthmovingPhysicsCore._seed_gpu_residual_frontier and
 *       _advance_gpu_residual_frontier (runtime/v2_physics_core.py:1153-1254)
 *       over WarpCompactActiveEdgeOperator (solvers/warp_compact_frontier.py:144-392)
 *   sb_last_error
 *       the reference's exception messages (ValueError / RuntimeError text)
 */
#ifndef SOILB200_H
#define SOILB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum sb_status {
  SB_OK = 0,
  SB_ERR_BAD_ARG = 1,         /* ValueError in the reference */
  SB_ERR_SUBSTEP_CAP = 2,     /* "MobileV2 maximum_substeps exceeded" */
  SB_ERR_POSITIVITY = 3,      /* "MobileV2 positivity failure" */
  SB_ERR_NONCONVERGENCE = 4,  /* "NUMERICAL_NONCONVERGENCE: ..." */
  SB_ERR_CUDA = 5,            /* CUDA runtime/driver error */
  SB_ERR_WAIT_LIMIT = 6,      /* a bounded device-side wait gave up */
  SB_ERR_STATE = 7,           /* call order / missing data */
  SB_ERR_RANGE = 8,           /* value outside the fixed-point range */
  SB_ERR_CAPACITY = 9         /* request larger than a fixed, preallocated capacity */
};

enum sb_precision { SB_FP64 = 0, SB_FX32 = 1 };

/* Field identifiers; names follow DeviceBulkState. */
enum sb_field {
  SB_FIELD_Z_BASE = 0,
  SB_FIELD_B_EFF = 1,
  SB_FIELD_MOBILE = 2,
  SB_FIELD_MOMENTUM_X = 3,
  SB_FIELD_MOMENTUM_Y = 4,
  SB_FIELD_EXTERNAL_X = 5,    /* optional external acceleration, m/s^2 */
  SB_FIELD_EXTERNAL_Y = 6,
  SB_FIELD_FRONTIER_REACHED = 7,   /* int32 */
  SB_FIELD_LABELS = 8,             /* int32, read-only: canonical component labels */
  SB_FIELD_UNSTABLE = 9,           /* int32, read-only */
  SB_FIELD_SLOPE = 10,             /* read-only, radians */
  SB_FIELD_SEVERITY = 11,          /* read-only */
  SB_FIELD_LATCH = 12,             /* int32 */
  SB_FIELD_PREVIOUS_COMPONENT = 13, /* int32 */
  SB_FIELD_FORCING = 14,            /* int32 flat: nonzero = tool forcing (no deposition) */
  SB_FIELD_M2R_CUMULATIVE = 15,     /* float64 flat: settled volume per cell (deposition), m^3 */
  /* large-avalanche per-cell history (flat; float64 in both precisions) */
  SB_FIELD_R2M_CUMULATIVE = 16,         /* activated volume per cell, m^3 */
  SB_FIELD_FIRST_ACTIVATION_TIME = 17,  /* s */
  SB_FIELD_LAST_ACTIVATION_TIME = 18,   /* s */
  SB_FIELD_OWNED_SURFACE = 19,          /* free surface at activation, m */
  SB_FIELD_OWNED_EXPORT_BASELINE = 20,
  SB_FIELD_EXPORT_CUMULATIVE = 21,
  SB_FIELD_ACTIVATION_COUNT = 22        /* int32 flat */
};

typedef struct sb_ctx sb_ctx;

typedef struct sb_grid_desc {
  int device;
  int ny;                /* rows (TerrainGrid.shape[0]) */
  int nx;                /* columns */
  double dx_m;
  double dy_m;
  int tile_size;         /* frontier / dirty-tile size (reference default 64) */
  int precision;         /* enum sb_precision */
  int height_exponent;   /* SB_FX32: quantum = 2^-height_exponent m */
  double datum_m;        /* SB_FX32: b_eff/z_base are stored relative to this */
} sb_grid_desc;

/* MobileV2Config keys (experimental/mobile_v2_reference.py:16-27). */
typedef struct sb_mobile_params {
  double gravity_m_s2;
  double earth_pressure_coefficient;
  double cfl;
  double dry_tolerance_m;
  double start_angle_deg;
  double basal_friction_coefficient;
  int maximum_substeps;
  int use_external;            /* 1: apply SB_FIELD_EXTERNAL_X/Y */
  double density_kg_m3;        /* production ledger density (weighted sums) */
} sb_mobile_params;

/* Ledger of one state; uniform-area and Triangle-A-C-weighted reductions. */
typedef struct sb_mobile_ledger {
  double mass_m3;              /* sum(h) dx dy */
  double momentum_m4_s[2];     /* sum(q) dx dy */
  double kinetic;              /* per unit density, uniform area */
  double gravitational;
  double internal;
  double volume_w_m3;          /* sum(h w), w = Triangle-A-C vertex weights */
  double momentum_w[2];        /* density * sum(q w) */
  double kinetic_w_j;          /* 0.5 density sum(h |u|^2 w) */
  double potential_w_j;        /* density g sum(h b w) */
  double pressure_w_j;         /* density 0.5 K g sum(h^2 w) */
  double max_speed_m_s;
  double min_h_m;
  int64_t mass_quanta;         /* SB_FX32: exact sum of h quanta */
  int64_t volume_w_quanta;     /* SB_FX32: exact sum of h quanta * (6 w / dx dy) */
  double resting_volume_w_m3;  /* sum(max(b_eff - z_base, 0) w) (reservoir_reduction) */
  int64_t resting_w_quanta;    /* SB_FX32: exact form of resting_volume_w_m3 */
} sb_mobile_ledger;

typedef struct sb_mobile_stats {
  int substeps;
  int static_skip;             /* 1 when the static short-circuit returned */
  int cfl_limited;
  int status;
  double maximum_cfl;
  double conservative_impulse_m4_s[2];
  double friction_impulse_m4_s[2];
  double external_impulse_m4_s[2];
  double friction_dissipation;     /* per unit density */
  double external_work;            /* per unit density */
  sb_mobile_ledger before;
  sb_mobile_ledger after;
  double substep_loop_ms;      /* device time of the substep loop (CUDA events) */
} sb_mobile_stats;

int sb_ctx_create(const sb_grid_desc* desc, sb_ctx** out);
int sb_ctx_destroy(sb_ctx* ctx);
/* Row-major ny*nx host arrays.  Float fields take/give float64; int fields int32. */
int sb_upload(sb_ctx* ctx, int field, const double* host);
int sb_download(sb_ctx* ctx, int field, double* host);
int sb_upload_i32(sb_ctx* ctx, int field, const int32_t* host);
int sb_download_i32(sb_ctx* ctx, int field, int32_t* host);
int sb_synchronize(sb_ctx* ctx);

int sb_mobile_step(sb_ctx* ctx, double dt_s, const sb_mobile_params* params,
                   sb_mobile_stats* out);
int sb_mobile_ledger_of(sb_ctx* ctx, const sb_mobile_params* params,
                        sb_mobile_ledger* out);

/* ---- Large-avalanche (FailureZone) labelling ---------------------------- */
/* Material/config keys of DeviceLargeAvalancheBridge.initialize
 * (runtime/gpu_large_avalanche.py:541-566); angles are passed both as tangents
 * and radians so callers can compute them exactly as the reference does. */
typedef struct sb_label_params {
  double tan_start;
  double tan_stop;
  double start_rad;
  double stop_rad;
  double density_kg_m3;
  double gravity_m_s2;
  double cohesion_pa;
  double mobilization_depth_m;
  double dry_tolerance_m;
  double activity_speed_m_s;
  int connectivity;            /* 4 or 8 */
  int release_settled_latches;
} sb_label_params;

typedef struct sb_label_stats {
  int status;
  int unstable_cell_count;
  int connected_region_count;
  int largest_connected_cell_count;
  int winner_root;             /* canonical label (min flat index) of the winner */
  int union_passes;
  int previous_overlap;        /* winner cells that were in the previous component */
  int pad;
  double largest_connected_area_m2;
  double largest_connected_mobilizable_volume_m3;
  double excess_start_sum_rad; /* over winner cells */
  double excess_start_max_rad;
  double excess_stop_sum_rad;
  double excess_stop_max_rad;
} sb_label_stats;

/* Yield initialisation + connected components + component reductions. */
int sb_label(sb_ctx* ctx, const sb_label_params* params, sb_label_stats* out);
/* Components of a caller-provided int32 mask (nonzero = member); replaces the
 * CPU _largest_connected_region(mask, connectivity)
 * (bulk_interaction/large_avalanche.py:711-778).  Labels via SB_FIELD_LABELS. */
int sb_label_mask(sb_ctx* ctx, const int32_t* mask, int connectivity, sb_label_stats* out);
/* update_previous_and_tiles (gpu_large_avalanche.py:277-306): previous-component
 * mask and, when seed_frontier, frontier_reached + the frontier tile flags. */
int sb_label_commit(sb_ctx* ctx, int keep_candidate, int seed_frontier);

/* ---- Repose relaxation ---------------------------------------------------- */
typedef struct sb_relax_params {
  double spacing0_m;           /* spacing along axis 0 (rows) */
  double spacing1_m;           /* spacing along axis 1 (columns) */
  double critical_slope;       /* tan(critical angle) */
  double tolerance_m;
  int max_iterations;          /* full: iterations; frontier: rounds */
  int weighted;                /* frontier: Triangle-A-C vertex weights, else uniform */
} sb_relax_params;

typedef struct sb_relax_stats {
  int iterations;              /* full: iterations run; frontier: rounds */
  int converged;
  int status;
  int active_tiles;            /* frontier: active tiles at the last round start */
  int moved_edges;             /* frontier: transfers applied */
  int pad;
} sb_relax_stats;

/* relax_critical_slope on SB_FIELD_B_EFF (slope_model.py:273-343). */
int sb_relax_full(sb_ctx* ctx, const sb_relax_params* params, sb_relax_stats* out);
/* The same sweeps queued on the context's stream without waiting for them or
 * reading statistics back (at most max_iterations; for interleaving with other
 * device work, e.g. learned proposals). */
int sb_relax_sweeps(sb_ctx* ctx, const sb_relax_params* params);
/* Event-driven reached-bbox MiniSlope on SB_FIELD_B_EFF
 * (EventDrivenMinimumSlopeAdapter._relax_dynamic_frontier,
 * solvers/event_driven_slope.py:166-302): seeds = the current
 * SB_FIELD_FRONTIER_REACHED mask; every iteration runs the eight colour
 * sub-phases on pairs with a reached endpoint only, marks both endpoints of
 * every moved pair reached, and the solve ends after a confirming scan of the
 * reachable pairs shows max excess <= tolerance.  The grown reached mask is
 * left in SB_FIELD_FRONTIER_REACHED.  iterations > max_iterations ->
 * SB_ERR_NONCONVERGENCE (the reference's numerical safety limit). */
int sb_relax_reached(sb_ctx* ctx, const sb_relax_params* params, sb_relax_stats* out);
/* Frontier seeds: reached := 1 at the cells and their 3x3-stencil tiles become
 * active (_seed_gpu_residual_frontier, v2_physics_core.py:1153-1170). */
int sb_frontier_seed_cells(sb_ctx* ctx, const int32_t* flat_indices, int count);
/* Activate tiles directly (tile id = row_tile * tiles_x + col_tile). */
int sb_frontier_seed_tiles(sb_ctx* ctx, const int32_t* tile_ids, int count);
/* Residual frontier rounds on SB_FIELD_B_EFF until no tile is active. */
int sb_frontier_run(sb_ctx* ctx, const sb_relax_params* params, sb_relax_stats* out);
/* Copies the next-round active tile flags (int32 per tile) to the host. */
int sb_frontier_active_tiles(sb_ctx* ctx, int32_t* flags, int capacity);
int sb_frontier_tile_count(sb_ctx* ctx);
/* out4 = {sum of values, max 8-neighbour slope, min value, sum of quanta (SB_FX32)}
 * of SB_FIELD_B_EFF or SB_FIELD_Z_BASE (RelaxationStats volume / max_slope,
 * slope_model.py:261-270, :331-342). */
int sb_field_stats(sb_ctx* ctx, int field, double spacing0_m, double spacing1_m, double* out4);

/* ---- Resting <-> Mobile exchange (runtime/bulk_state_authority.py:103-149,
 *      entrain_host_indices / deposit_host_indices :920-1034) ------------ */
/* b_eff -= d, mobile += d with d = min(max(depth,0), max(b_eff - z_base, 0));
 * volume_m3 = sum(d * w) (exact in SB_FX32). */
int sb_entrain(sb_ctx* ctx, const int32_t* flat_indices, const double* requested_depth_m,
               int count, double* volume_m3);
/* Same, with the requested depth b_eff - target_surface (a cut to a surface). */
int sb_entrain_to_surface(sb_ctx* ctx, const int32_t* flat_indices,
                          const double* target_surface_m, int count, double* volume_m3);
/* mobile -= d, b_eff += d, momentum scaled by the retained fraction;
 * out3 = {deposited volume m3, removed momentum x, y (density * q * w)}. */
int sb_deposit(sb_ctx* ctx, const int32_t* flat_indices, const double* requested_depth_m,
               int count, double density_kg_m3, double* out3);

/* ---- Fused plain terrain step ----------------------------------------------
 * One call = one physics step of the production GPU core restricted to this
 * library's operators (runtime/v2_physics_core.py:708-1003): tool cut
 * entrainment to target surfaces -> Mobile V2 step (all CFL substeps) ->
 * large-avalanche labelling, classification and persistence
 * (gpu_large_avalanche.py:541-676) -> frontier seeding for local
 * instabilities -> residual MiniSlope frontier rounds, gated as the
 * reference gates them (quiet mobile layer, no mobilizable yield).  The whole
 * step is one CUDA graph launch with one host synchronisation.  The cut
 * command is copied on the host into the context's mapped pinned buffers
 * (read by the graph over the host link), so the caller's arrays may be
 * pageable and are not referenced after the call. */
typedef struct sb_path_params {
  sb_mobile_params mobile;
  sb_label_params label;
  sb_relax_params relax;       /* residual frontier: spacing, tan(stop angle), tolerance, rounds */
  int minimum_connected_cells; /* LargeAvalancheTransitionConfig thresholds */
  int residual_mode;           /* 0 never, 1 gated like the reference, 2 every step */
  double minimum_connected_area_m2;
  double minimum_mobilizable_volume_m3;
  double minimum_mean_excess_start_deg;
  double persistence_time_s;
  double settled_mobile_volume_m3;
  double settled_speed_m_s;
} sb_path_params;

typedef struct sb_path_stats {
  sb_mobile_stats mobile;
  sb_label_stats label;
  sb_relax_stats relax;
  double entrained_m3;
  double persistence_s;
  double mean_excess_start_deg;
  int classification;          /* 0 NO_LARGE_EVENT, 1 LOCAL_STATIC_INSTABILITY,
                                  2 PERSISTING_LARGE_UNSTABLE_REGION, 3 LARGE_AVALANCHE_MOBILE_PATH */
  int candidate;
  int transition_ready;
  int residual_ran;
  double device_ms;            /* device time of the step graph (first to last node) */
} sb_path_stats;

int sb_path_step(sb_ctx* ctx, double dt_s, const int32_t* cut_flat_indices,
                 const double* cut_target_surface_m, int cut_count, const sb_path_params* params,
                 sb_path_stats* out);
/* Clears the persistence state of the fused step (reset of the bridge). */
int sb_path_reset(sb_ctx* ctx);
/* Device-time breakdown of the last sb_path_step when the context was created
 * with SOILB200_STAGE_EVENTS=1 (event nodes between the stages of the step
 * graph: start + entrainment, before-ledger, substep loop + yield/union-find
 * tile pass, border merge, compression, reduction/classification, previous
 * mask + seeding, residual frontier).  No counterpart in the reference (a
 * profiling aid).  Returns the number of stage times written (ms), 0 when
 * disabled, a negative status on bad arguments. */
int sb_path_stage_times(sb_ctx* ctx, float* out_ms, int capacity);

/* ---- Allocation-free connected components --------------------------------
 * No counterpart in the reference.  For callers that must not allocate device
 * memory once running -- e.g. a simulator plugin whose frame callbacks forbid
 * cudaMalloc (it can block, synchronise the device and break real-time step
 * budgets), or a host that hands the plugin a fixed device-memory budget at
 * start-up and owns every allocation after that.  The caller passes device
 * pointers for the int32 mask (nonzero = member) and the int32 output labels
 * (canonical: -1 outside the mask, else the component's minimum flat index),
 * both ny*nx row-major, plus the stream to run on.  Scratch (per-root counters
 * and the root list) is a file-scope static device array reserved on every
 * GPU that loads the library until process exit; it is never allocated by
 * this call.  Limit: ny*nx <= 524288 cells (SB_ERR_CAPACITY beyond).  The
 * first call on a device looks up the scratch address with the device
 * current and keeps it for the process (after cudaDeviceReset the module is
 * reloaded at a new address, so do not call this across a device reset).
 * Every call shares the one scratch array (its contents persist; each call clears what
 * must start at zero), so calls that overlap on the GPU race: serialise them
 * (one stream, or wait between calls).  Blocks until the stats are read.
 * dx_m/dy_m only scale largest_connected_area_m2. */
int sb_label_mask_static(const int32_t* d_mask, int32_t* d_labels, int ny, int nx,
                         int connectivity, double dx_m, double dy_m, void* stream,
                         sb_label_stats* out);

/* ---- Large-avalanche activation and lifecycle (runtime/gpu_large_avalanche.py
 *      kernels mobilize :308-372, reduce_persistence :374-451; host
 *      observe_and_maybe_mobilize :541-676, _persistence_summary :785-840) ----
 * sb_avalanche_mobilize acts on the component selected by the last sb_label:
 * each unlatched cell moves min(max(b_eff - z_base, 0), depth * severity)
 * Resting -> Mobile at zero momentum (above the dry tolerance), latches, and
 * records its activation history.  sb_avalanche_persistence reduces the
 * lifecycle sums; net terrain change is against the b_eff snapshot taken by
 * sb_avalanche_set_initial_resting (zeros before the first snapshot). */
typedef struct sb_mobilize_stats {
  double transferred_volume_m3;      /* sum(transfer * w) */
  double newly_activated_volume_m3;
  double reactivated_volume_m3;
  double newly_activated_area_m2;
  double reactivated_area_step_m2;
  int64_t transferred_w6_quanta;     /* SB_FX32: exact */
  int cells;
  int pad;
} sb_mobilize_stats;

typedef struct sb_persistence_stats {
  int unique_cells_ever_activated;
  int cells_activated_more_than_once;
  int current_mobile_cell_count;
  int retired_candidate_cell_count;
  int active_tile_count;
  int pad;
  double cumulative_r2m_m3;
  double cumulative_m2r_m3;
  double unique_activated_area_m2;
  double reactivated_area_m2;
  double current_mobile_volume_m3;
  double maximum_mobile_speed_m_s;
  double net_terrain_volume_change_m3;
  double net_spatial_transfer_m3;
  double activated_slope_sum_rad;
  double activated_slope_max_rad;
  double slope_minus_stop_sum_rad;
  double start_minus_slope_sum_rad;
  double retired_candidate_area_m2;
  double moving_mobile_volume_m3;
} sb_persistence_stats;

int sb_avalanche_set_initial_resting(sb_ctx* ctx);
int sb_avalanche_mobilize(sb_ctx* ctx, double activation_time_s, double mobilization_depth_m,
                          double dry_tolerance_m, sb_mobilize_stats* out);
int sb_avalanche_persistence(sb_ctx* ctx, double start_angle_rad, double stop_angle_rad,
                             double dry_tolerance_m, double activity_speed_m_s,
                             sb_persistence_stats* out);

/* ---- Surface publication (runtime/bulk_state_authority.py: dirty tracking
 *      :733-781 with kernels :156-192, tile downloads :1280-1328, batched
 *      bilinear queries :1138-1183 with kernel :195-231) ---------------------
 * Free surface = b_eff + mobile.  sb_surface_capture snapshots it;
 * sb_surface_dirty_tiles flags every tile (tile_size of the context, row-major
 * tile ids) holding a cell whose surface moved by more than tolerance_m since
 * the snapshot (flags: ceil(ny/tile) * ceil(nx/tile) int32).
 * sb_surface_region downloads rows [r0, r1) x cols [c0, c1).
 * sb_surface_sample_bilinear samples at fractional (row, col), clamped. */
int sb_surface_capture(sb_ctx* ctx);
int sb_surface_dirty_tiles(sb_ctx* ctx, double tolerance_m, int32_t* flags, int ntiles);
int sb_surface_region(sb_ctx* ctx, int r0, int r1, int c0, int c1, double* out);
int sb_surface_sample_bilinear(sb_ctx* ctx, const double* rows, const double* cols, int count,
                               double* out);

/* ---- Mobile -> Resting deposition (bulk_interaction/warp_deposition.py:23-130,
 *      WarpDepositionOperator.step_resident :183-238) -------------------------
 * Every cell with mobile material, no tool forcing (SB_FIELD_FORCING) and
 * speed |q/h| <= speed_threshold whose free surface is below the cohesive
 * stop yield settles min(h, rate*dt) into b_eff (all of h when
 * settle_subcell_tail), momentum shrinking in proportion; b_eff + h is
 * unchanged.  All cells read the pre-step surface.  Sums as the reference's
 * weighted_sum: volume sum(settled * w), momentum density * sum(removed q * w). */
typedef struct sb_deposition_params {
  double settling_rate_m_s;    /* 0.30 */
  double speed_threshold_m_s;  /* 0.18 */
  double density_kg_m3;        /* MaterialScenario.assumed_bulk_density_kg_m3 */
  double gravity_m_s2;         /* 9.81 */
  double cohesion_pa;          /* MaterialScenario.cohesion_proxy_pa */
  double stop_angle_deg;       /* MaterialScenario.stop_angle_deg */
  int settle_subcell_tail;
  int pad;
} sb_deposition_params;

typedef struct sb_deposition_stats {
  double deposited_volume_m3;
  double removed_momentum_kg_m_s[2];
  int64_t deposited_w6_quanta;  /* SB_FX32: exact sum of settled quanta * (6 w / dx dy) */
  int cells;                    /* cells that settled material */
  int pad;
} sb_deposition_stats;

int sb_deposition_step(sb_ctx* ctx, double dt_s, const sb_deposition_params* params,
                       sb_deposition_stats* out);

/* ---- Batched terrain patches ----------------------------------------------
 * Many independent Mobile V2 grids ("patches": parallel dig environments of
 * uneven sizes) advanced by shared launches.  The reference steps one
 * DeviceBulkState per call (WarpProductionMobileV2Solver.step_resident,
 * bulk_interaction/warp_mobile_v2.py:188-245; MobileV2ReferenceSolver.step,
 * experimental/mobile_v2_reference.py:191-314); a batch runs that step for
 * every patch with the SB_FX32 arithmetic of sb_mobile_step, each patch with
 * its own quantum, CFL substeps and ledgers.  Patch fields are those of a
 * context: SB_FIELD_Z_BASE, SB_FIELD_B_EFF, SB_FIELD_MOBILE,
 * SB_FIELD_MOMENTUM_X/Y (row-major ny*nx float64 on the host).  No external
 * acceleration.  One stream per batch; calls are synchronous at return. */
typedef struct sb_batch sb_batch;

typedef struct sb_patch_desc {
  int ny, nx;
  double dx_m, dy_m;
  int height_exponent;         /* patch quantum 2^-k m, 4 <= k <= 40 */
  int pad;
  double datum_m;              /* datum of the patch's b_eff / z_base quanta */
} sb_patch_desc;

int sb_batch_create(int device, int n_patches, const sb_patch_desc* patches, sb_batch** out);
int sb_batch_destroy(sb_batch* batch);
int sb_batch_upload(sb_batch* batch, int patch, int field, const double* host);
int sb_batch_download(sb_batch* batch, int patch, int field, double* host);
/* Tile shape: rows per warp strip for every patch (4..256; default 16). */
int sb_batch_set_rows(sb_batch* batch, const int* rows_per_warp);
int sb_batch_get_rows(sb_batch* batch, int* rows_per_warp);
/* One physics step of dt_s for every patch; per_patch[n_patches] receives each
 * patch's record (as sb_mobile_step's).  The first failing patch's status is
 * returned, its index in the message. */
int sb_batch_step(sb_batch* batch, double dt_s, const sb_mobile_params* params,
                  sb_mobile_stats* per_patch);
/* Times every candidate rows-per-warp for each group of equal-height patches
 * (trials steps each, on the live state, which is copied first and put back)
 * and keeps the fastest; best_ms = substep-loop time of one step with it. */
int sb_batch_autotune(sb_batch* batch, double dt_s, const sb_mobile_params* params, int trials,
                      double* best_ms);
/* Large-avalanche labelling of every patch's current state: the single-grid
 * sb_label yield + canonical union-find (runtime/gpu_large_avalanche.py:
 * 58-275), patch by patch; out[n_patches] receives each patch's record.  A
 * batch models no latches or previous components (none set, none released). */
int sb_batch_label(sb_batch* batch, const sb_label_params* params, sb_label_stats* out);
/* Canonical labels of one patch after sb_batch_label (ny*nx int32, -1 = stable). */
int sb_batch_download_labels(sb_batch* batch, int patch, int32_t* host);
int sb_batch_last_error(sb_batch* batch, char* buffer, size_t length);
int64_t sb_batch_kernel_launch_count(sb_batch* batch);
void* sb_batch_stream(sb_batch* batch);

/* ---- Learned repose proposal ------------------------------------------------
 * No counterpart in the reference (its repose relaxation is the plain sweep,
 * slope_model.py:273-343, alone).  A 4-layer 3x3 convolution net proposes
 * per-edge outflows of b_eff; they are applied in flux form and the plain
 * sweeps (sb_relax_full / sb_frontier_run) finish to the tolerance.
 * Convolutions: BF16 NHWC activations (channels 16 or 32), FP32 accumulate on
 * the tensor cores; weights prepacked per row offset dy in the canonical
 * K-major layout (n = dx*cout + co rows, k = ci).  Device pointers, 16-byte
 * aligned; work is queued on `stream`; d_status (device int, may be null)
 * becomes 1 if a bounded device wait gave up.  out_f32 = 0 writes BF16 (all
 * cout channels); out_f32 = k (multiple of 4) writes FP32, first k channels. */
const char* sb_learned_last_error(void);
int sb_learned_conv(const void* in, void* out, const void* wpk, const void* mask, int batch, int h,
                    int w, int cin, int cout, int relu, int out_f32, int rows_per_cta,
                    int* d_status, void* stream);
/* dW[3][3][cin][cout] (f32) of a layer from its input and output gradient;
 * partial: ceil(w/128)*ceil(h/rows)*batch*3*128*cout floats of scratch. */
int sb_learned_wgrad(const void* in, const void* grad, float* partial, size_t partial_floats,
                     float* dw, int batch, int h, int w, int cin, int cout, int rows_per_cta,
                     int* d_status, void* stream);
/* Features (bf16 [batch][h][w][16]: channels 0..3 = height drop along the
 * east, north, north-east, north-west edges over L*tan_crit) of float64
 * heights; training loss of f32 fluxes [pixel][4] against target height
 * changes. */
int sb_learned_features_f64(const double* heights, void* feat, int batch, int h, int w, double dx,
                            double dy, double tan_crit, void* stream);
int sb_learned_loss(const float* flux, const float* target_dh, float* resid, void* dflux,
                    double* loss_part, int batch, int h, int w, double dx, double dy,
                    double tan_crit, float inv_scale2_n, void* stream);
int sb_learned_loss_blocks(int batch, int h, int w);
/* Inference of the whole 4-layer network in one launch: features bf16
 * [batch][h][w][16] -> f32 fluxes [batch][h][w][4] (the last layer's first
 * four channels), equal bit for bit to the four sb_learned_conv calls (ReLU
 * after the first three, BF16 activations).  w1..w4: packed weights of the
 * layers 16->32, 32->32, 32->32, 32->16.  rows_per_cta = 0 picks about one
 * wave of CTAs.  Activations stay in shared memory: one CTA per SM streams a
 * 122-pixel column strip down a band of rows. */
int sb_learned_forward(const void* feat, float* flux, const void* w1, const void* w2,
                       const void* w3, const void* w4, int batch, int h, int w, int rows_per_cta,
                       int* d_status, void* stream);
/* On a context's resident b_eff (SB_FX32): features, then the network's
 * fluxes (f32 [ny][nx][4]) applied in whole height quanta (tq: int32
 * [ny][nx][4] scratch). */
int sb_learned_features(sb_ctx* ctx, void* feat, double tan_crit);
int sb_learned_apply(sb_ctx* ctx, const float* flux, int32_t* tq, double tan_crit);

int sb_last_error(sb_ctx* ctx, char* buffer, size_t length);
/* Number of kernels this context has launched (cumulative). */
int64_t sb_kernel_launch_count(sb_ctx* ctx);
/* The cudaStream_t every operation of this context is issued on (for timing
 * with events or ordering caller work; do not destroy it). */
void* sb_stream(sb_ctx* ctx);
const char* sb_version(void);
/* sizeof() of an ABI struct by name ("sb_grid_desc", "sb_mobile_params",
 * "sb_mobile_ledger", "sb_mobile_stats", ...); 0 if unknown.  Lets bindings
 * verify their struct layouts against the compiled library. */
size_t sb_sizeof(const char* type_name);

#ifdef __cplusplus
}
#endif

#endif /* SOILB200_H */
