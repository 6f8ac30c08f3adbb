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
  SB_ERR_RANGE = 8            /* value outside the fixed-point range */
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
  SB_FIELD_PREVIOUS_COMPONENT = 13 /* int32 */
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

int sb_last_error(sb_ctx* ctx, char* buffer, size_t length);
/* Number of kernels this context has launched (cumulative). */
int64_t sb_kernel_launch_count(sb_ctx* ctx);
const char* sb_version(void);
/* sizeof() of an ABI struct by name ("sb_grid_desc", "sb_mobile_params",
 * "sb_mobile_ledger", "sb_mobile_stats", ...); 0 if unknown.  Lets bindings
 * verify their struct layouts against the compiled library. */
size_t sb_sizeof(const char* type_name);

#ifdef __cplusplus
}
#endif

#endif /* SOILB200_H */
