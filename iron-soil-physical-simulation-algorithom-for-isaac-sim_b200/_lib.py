"""ctypes binding of ``libsoilb200.so`` (declarations mirror include/soilb200.h).

The library is the only compute path: if it is missing or no CUDA device is
usable, every entry point raises :class:`B200BackendUnavailable` -- there is
no CPU fallback (the reference likewise refuses to relabel a missing Warp
backend as a GPU pass, ``performance/warp_backend.py`` / ``probe_warp``).
"""

from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libsoilb200.so"

SB_OK = 0
SB_ERR_BAD_ARG = 1
SB_ERR_SUBSTEP_CAP = 2
SB_ERR_POSITIVITY = 3
SB_ERR_NONCONVERGENCE = 4
SB_ERR_CUDA = 5
SB_ERR_WAIT_LIMIT = 6
SB_ERR_STATE = 7
SB_ERR_RANGE = 8
SB_ERR_CAPACITY = 9

SB_FP64 = 0
SB_FX32 = 1

FIELD = {
    "z_base": 0,
    "b_eff": 1,
    "mobile": 2,
    "momentum_x": 3,
    "momentum_y": 4,
    "external_x": 5,
    "external_y": 6,
    "frontier_reached": 7,
    "labels": 8,
    "unstable": 9,
    "slope": 10,
    "severity": 11,
    "latch": 12,
    "previous_component": 13,
    "forcing": 14,
    "m2r_cumulative": 15,
    "r2m_cumulative": 16,
    "first_activation_time": 17,
    "last_activation_time": 18,
    "owned_surface": 19,
    "owned_export_baseline": 20,
    "export_cumulative": 21,
    "activation_count": 22,
}
INT_FIELDS = {"frontier_reached", "labels", "unstable", "latch", "previous_component", "forcing",
              "activation_count"}


class B200BackendUnavailable(RuntimeError):
    """The CUDA library or a usable B200 device is not available."""


class B200DeviceError(RuntimeError):
    """A CUDA error raised while running an operation on an existing context."""


class NumericalNonconvergenceError(RuntimeError):
    """Device loop exceeded its bound (reference: solvers/event_driven_slope.py:510-533)."""


class GridDesc(C.Structure):
    _fields_ = [
        ("device", C.c_int), ("ny", C.c_int), ("nx", C.c_int),
        ("dx_m", C.c_double), ("dy_m", C.c_double), ("tile_size", C.c_int),
        ("precision", C.c_int), ("height_exponent", C.c_int), ("datum_m", C.c_double),
    ]


class MobileParams(C.Structure):
    _fields_ = [
        ("gravity_m_s2", C.c_double), ("earth_pressure_coefficient", C.c_double),
        ("cfl", C.c_double), ("dry_tolerance_m", C.c_double),
        ("start_angle_deg", C.c_double), ("basal_friction_coefficient", C.c_double),
        ("maximum_substeps", C.c_int), ("use_external", C.c_int),
        ("density_kg_m3", C.c_double),
    ]


class MobileLedger(C.Structure):
    _fields_ = [
        ("mass_m3", C.c_double), ("momentum_m4_s", C.c_double * 2),
        ("kinetic", C.c_double), ("gravitational", C.c_double), ("internal", C.c_double),
        ("volume_w_m3", C.c_double), ("momentum_w", C.c_double * 2),
        ("kinetic_w_j", C.c_double), ("potential_w_j", C.c_double),
        ("pressure_w_j", C.c_double), ("max_speed_m_s", C.c_double),
        ("min_h_m", C.c_double), ("mass_quanta", C.c_int64),
        ("volume_w_quanta", C.c_int64), ("resting_volume_w_m3", C.c_double),
        ("resting_w_quanta", C.c_int64),
    ]


class MobileStats(C.Structure):
    _fields_ = [
        ("substeps", C.c_int), ("static_skip", C.c_int), ("cfl_limited", C.c_int),
        ("status", C.c_int), ("maximum_cfl", C.c_double),
        ("conservative_impulse_m4_s", C.c_double * 2),
        ("friction_impulse_m4_s", C.c_double * 2),
        ("external_impulse_m4_s", C.c_double * 2),
        ("friction_dissipation", C.c_double), ("external_work", C.c_double),
        ("before", MobileLedger), ("after", MobileLedger),
        ("substep_loop_ms", C.c_double),
    ]


class LabelParams(C.Structure):
    _fields_ = [
        ("tan_start", C.c_double), ("tan_stop", C.c_double), ("start_rad", C.c_double),
        ("stop_rad", C.c_double), ("density_kg_m3", C.c_double), ("gravity_m_s2", C.c_double),
        ("cohesion_pa", C.c_double), ("mobilization_depth_m", C.c_double),
        ("dry_tolerance_m", C.c_double), ("activity_speed_m_s", C.c_double),
        ("connectivity", C.c_int), ("release_settled_latches", C.c_int),
    ]


class LabelStats(C.Structure):
    _fields_ = [
        ("status", C.c_int), ("unstable_cell_count", C.c_int),
        ("connected_region_count", C.c_int), ("largest_connected_cell_count", C.c_int),
        ("winner_root", C.c_int), ("union_passes", C.c_int), ("previous_overlap", C.c_int),
        ("pad", C.c_int), ("largest_connected_area_m2", C.c_double),
        ("largest_connected_mobilizable_volume_m3", C.c_double),
        ("excess_start_sum_rad", C.c_double), ("excess_start_max_rad", C.c_double),
        ("excess_stop_sum_rad", C.c_double), ("excess_stop_max_rad", C.c_double),
    ]


class RelaxParams(C.Structure):
    _fields_ = [
        ("spacing0_m", C.c_double), ("spacing1_m", C.c_double), ("critical_slope", C.c_double),
        ("tolerance_m", C.c_double), ("max_iterations", C.c_int), ("weighted", C.c_int),
    ]


class RelaxStats(C.Structure):
    _fields_ = [
        ("iterations", C.c_int), ("converged", C.c_int), ("status", C.c_int),
        ("active_tiles", C.c_int), ("moved_edges", C.c_int), ("pad", C.c_int),
    ]


class PathParams(C.Structure):
    _fields_ = [
        ("mobile", MobileParams), ("label", LabelParams), ("relax", RelaxParams),
        ("minimum_connected_cells", C.c_int), ("residual_mode", C.c_int),
        ("minimum_connected_area_m2", C.c_double), ("minimum_mobilizable_volume_m3", C.c_double),
        ("minimum_mean_excess_start_deg", C.c_double), ("persistence_time_s", C.c_double),
        ("settled_mobile_volume_m3", C.c_double), ("settled_speed_m_s", C.c_double),
    ]


class PathStats(C.Structure):
    _fields_ = [
        ("mobile", MobileStats), ("label", LabelStats), ("relax", RelaxStats),
        ("entrained_m3", C.c_double), ("persistence_s", C.c_double),
        ("mean_excess_start_deg", C.c_double), ("classification", C.c_int),
        ("candidate", C.c_int), ("transition_ready", C.c_int), ("residual_ran", C.c_int),
        ("device_ms", C.c_double),
    ]


_LIB = None
class DepositionParams(C.Structure):
    _fields_ = [
        ("settling_rate_m_s", C.c_double), ("speed_threshold_m_s", C.c_double),
        ("density_kg_m3", C.c_double), ("gravity_m_s2", C.c_double), ("cohesion_pa", C.c_double),
        ("stop_angle_deg", C.c_double), ("settle_subcell_tail", C.c_int), ("pad", C.c_int),
    ]


class DepositionStats(C.Structure):
    _fields_ = [
        ("deposited_volume_m3", C.c_double), ("removed_momentum_kg_m_s", C.c_double * 2),
        ("deposited_w6_quanta", C.c_int64), ("cells", C.c_int), ("pad", C.c_int),
    ]


class MobilizeStats(C.Structure):
    _fields_ = [
        ("transferred_volume_m3", C.c_double), ("newly_activated_volume_m3", C.c_double),
        ("reactivated_volume_m3", C.c_double), ("newly_activated_area_m2", C.c_double),
        ("reactivated_area_step_m2", C.c_double), ("transferred_w6_quanta", C.c_int64),
        ("cells", C.c_int), ("pad", C.c_int),
    ]


class PersistenceStats(C.Structure):
    _fields_ = [
        ("unique_cells_ever_activated", C.c_int), ("cells_activated_more_than_once", C.c_int),
        ("current_mobile_cell_count", C.c_int), ("retired_candidate_cell_count", C.c_int),
        ("active_tile_count", C.c_int), ("pad", C.c_int),
        ("cumulative_r2m_m3", C.c_double), ("cumulative_m2r_m3", C.c_double),
        ("unique_activated_area_m2", C.c_double), ("reactivated_area_m2", C.c_double),
        ("current_mobile_volume_m3", C.c_double), ("maximum_mobile_speed_m_s", C.c_double),
        ("net_terrain_volume_change_m3", C.c_double), ("net_spatial_transfer_m3", C.c_double),
        ("activated_slope_sum_rad", C.c_double), ("activated_slope_max_rad", C.c_double),
        ("slope_minus_stop_sum_rad", C.c_double), ("start_minus_slope_sum_rad", C.c_double),
        ("retired_candidate_area_m2", C.c_double), ("moving_mobile_volume_m3", C.c_double),
    ]


class PatchDesc(C.Structure):
    _fields_ = [
        ("ny", C.c_int), ("nx", C.c_int), ("dx_m", C.c_double), ("dy_m", C.c_double),
        ("height_exponent", C.c_int), ("pad", C.c_int), ("datum_m", C.c_double),
    ]


_PROTOTYPES = {
    "sb_ctx_create": (C.c_int, [C.POINTER(GridDesc), C.POINTER(C.c_void_p)]),
    "sb_ctx_destroy": (C.c_int, [C.c_void_p]),
    "sb_upload": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "sb_download": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "sb_upload_i32": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "sb_download_i32": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "sb_synchronize": (C.c_int, [C.c_void_p]),
    "sb_mobile_step": (C.c_int, [C.c_void_p, C.c_double, C.POINTER(MobileParams),
                                 C.POINTER(MobileStats)]),
    "sb_mobile_ledger_of": (C.c_int, [C.c_void_p, C.POINTER(MobileParams),
                                      C.POINTER(MobileLedger)]),
    "sb_last_error": (C.c_int, [C.c_void_p, C.c_char_p, C.c_size_t]),
    "sb_kernel_launch_count": (C.c_int64, [C.c_void_p]),
    "sb_stream": (C.c_void_p, [C.c_void_p]),
    "sb_version": (C.c_char_p, []),
    "sb_sizeof": (C.c_size_t, [C.c_char_p]),
    "sb_label": (C.c_int, [C.c_void_p, C.POINTER(LabelParams), C.POINTER(LabelStats)]),
    "sb_label_commit": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "sb_label_mask": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.POINTER(LabelStats)]),
    "sb_label_mask_static": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int,
                                       C.c_double, C.c_double, C.c_void_p,
                                       C.POINTER(LabelStats)]),
    "sb_relax_full": (C.c_int, [C.c_void_p, C.POINTER(RelaxParams), C.POINTER(RelaxStats)]),
    "sb_relax_sweeps": (C.c_int, [C.c_void_p, C.POINTER(RelaxParams)]),
    "sb_relax_reached": (C.c_int, [C.c_void_p, C.POINTER(RelaxParams), C.POINTER(RelaxStats)]),
    "sb_frontier_seed_cells": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    "sb_frontier_seed_tiles": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    "sb_frontier_run": (C.c_int, [C.c_void_p, C.POINTER(RelaxParams), C.POINTER(RelaxStats)]),
    "sb_frontier_active_tiles": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    "sb_frontier_tile_count": (C.c_int, [C.c_void_p]),
    "sb_field_stats": (C.c_int, [C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_void_p]),
    "sb_path_step": (C.c_int, [C.c_void_p, C.c_double, C.c_void_p, C.c_void_p, C.c_int,
                               C.POINTER(PathParams), C.POINTER(PathStats)]),
    "sb_path_reset": (C.c_int, [C.c_void_p]),
    "sb_path_stage_times": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    "sb_entrain": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                             C.POINTER(C.c_double)]),
    "sb_entrain_to_surface": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                        C.POINTER(C.c_double)]),
    "sb_deposit": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_double,
                             C.c_void_p]),
    "sb_deposition_step": (C.c_int, [C.c_void_p, C.c_double, C.POINTER(DepositionParams),
                                     C.POINTER(DepositionStats)]),
    "sb_avalanche_set_initial_resting": (C.c_int, [C.c_void_p]),
    "sb_avalanche_mobilize": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_double,
                                        C.POINTER(MobilizeStats)]),
    "sb_avalanche_persistence": (C.c_int, [C.c_void_p, C.c_double, C.c_double, C.c_double,
                                           C.c_double, C.POINTER(PersistenceStats)]),
    "sb_surface_capture": (C.c_int, [C.c_void_p]),
    "sb_surface_dirty_tiles": (C.c_int, [C.c_void_p, C.c_double, C.c_void_p, C.c_int]),
    "sb_surface_region": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p]),
    "sb_surface_sample_bilinear": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                             C.c_void_p]),
    "sb_batch_create": (C.c_int, [C.c_int, C.c_int, C.POINTER(PatchDesc),
                                  C.POINTER(C.c_void_p)]),
    "sb_batch_destroy": (C.c_int, [C.c_void_p]),
    "sb_batch_upload": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p]),
    "sb_batch_download": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_void_p]),
    "sb_batch_set_rows": (C.c_int, [C.c_void_p, C.c_void_p]),
    "sb_batch_get_rows": (C.c_int, [C.c_void_p, C.c_void_p]),
    "sb_batch_step": (C.c_int, [C.c_void_p, C.c_double, C.POINTER(MobileParams), C.c_void_p]),
    "sb_batch_autotune": (C.c_int, [C.c_void_p, C.c_double, C.POINTER(MobileParams), C.c_int,
                                    C.POINTER(C.c_double)]),
    "sb_batch_last_error": (C.c_int, [C.c_void_p, C.c_char_p, C.c_size_t]),
    "sb_batch_label": (C.c_int, [C.c_void_p, C.POINTER(LabelParams), C.c_void_p]),
    "sb_batch_download_labels": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "sb_batch_kernel_launch_count": (C.c_int64, [C.c_void_p]),
    "sb_batch_stream": (C.c_void_p, [C.c_void_p]),
    "sb_learned_last_error": (C.c_char_p, []),
    "sb_learned_conv": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                           C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                           C.c_int, C.c_void_p, C.c_void_p]),
    "sb_learned_wgrad": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t,
                                            C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                            C.c_int, C.c_void_p, C.c_void_p]),
    "sb_learned_features_f64": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                                                   C.c_int, C.c_double, C.c_double, C.c_double,
                                                   C.c_void_p]),
    "sb_learned_loss": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                           C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_double,
                                           C.c_double, C.c_double, C.c_float, C.c_void_p]),
    "sb_learned_loss_blocks": (C.c_int, [C.c_int, C.c_int, C.c_int]),
    "sb_learned_forward": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int,
                                     C.c_void_p, C.c_void_p]),
    "sb_learned_features": (C.c_int, [C.c_void_p, C.c_void_p, C.c_double]),
    "sb_learned_apply": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_double]),
}

# ctypes mirror of each ABI struct, checked against sb_sizeof() in the tests.
ABI_STRUCTS = {
    "sb_grid_desc": GridDesc,
    "sb_mobile_params": MobileParams,
    "sb_mobile_ledger": MobileLedger,
    "sb_mobile_stats": MobileStats,
    "sb_label_params": LabelParams,
    "sb_label_stats": LabelStats,
    "sb_relax_params": RelaxParams,
    "sb_relax_stats": RelaxStats,
    "sb_path_params": PathParams,
    "sb_path_stats": PathStats,
    "sb_patch_desc": PatchDesc,
    "sb_deposition_params": DepositionParams,
    "sb_deposition_stats": DepositionStats,
    "sb_mobilize_stats": MobilizeStats,
    "sb_persistence_stats": PersistenceStats,
}


def exported_symbols() -> list[str]:
    return sorted(_PROTOTYPES)


def load():
    """Load the library (once).  Raises B200BackendUnavailable when absent."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = Path(os.environ.get("SOILB200_LIB", LIB_PATH))
    if not path.exists():
        raise B200BackendUnavailable(
            f"[soilb200] {path.name} is not built; run __graft_entry__.build() "
            "(there is no CPU fallback)")
    lib = C.CDLL(str(path))
    for name, (res, args) in _PROTOTYPES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib


def register(name: str, restype, argtypes) -> None:
    """Add a prototype (used by modules that bind further entry points)."""
    _PROTOTYPES[name] = (restype, argtypes)
    if _LIB is not None:
        fn = getattr(_LIB, name)
        fn.restype = restype
        fn.argtypes = argtypes


def last_error(ctx) -> str:
    buf = C.create_string_buffer(1024)
    load().sb_last_error(ctx, buf, 1024)
    return buf.value.decode(errors="replace")


def batch_last_error(batch) -> str:
    buf = C.create_string_buffer(1024)
    load().sb_batch_last_error(batch, buf, 1024)
    return buf.value.decode(errors="replace")


def check(ctx, status: int, what: str = "", *, batch=None) -> None:
    """Map a status code to the reference's exception types and messages."""
    if status == SB_OK:
        return
    msg = (batch_last_error(batch) if batch is not None else last_error(ctx)) or \
        f"{what} failed with status {status}"
    if status in (SB_ERR_BAD_ARG, SB_ERR_RANGE):
        raise ValueError(msg)
    if status == SB_ERR_NONCONVERGENCE:
        raise NumericalNonconvergenceError(msg)
    if status == SB_ERR_CUDA:
        raise B200DeviceError(msg)
    raise RuntimeError(msg)
