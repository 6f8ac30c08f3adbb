"""Large-avalanche (FailureZone) labelling on the GPU.

Mirrors the diagnosis part of the reference's ``DeviceLargeAvalancheBridge``
(``runtime/gpu_large_avalanche.py:469-676``): cohesive start/stop yield on the
free surface, 8- (or 4-) connected components of the unstable mask with
canonical min-index labels, the largest component (ties -> smallest label),
its area / mobilizable volume / slope excess, persistence in physical time
and the classification ``NO_LARGE_EVENT`` / ``LOCAL_STATIC_INSTABILITY`` /
``PERSISTING_LARGE_UNSTABLE_REGION`` / ``LARGE_AVALANCHE_MOBILE_PATH``
(:645-676), then ``update_previous_and_tiles`` which seeds the residual
frontier for local instabilities (:277-306).  ``MaterialScenario`` and
``LargeAvalancheTransitionConfig`` are restated with the reference's fields
(``bulk_state/models.py:51-62``; ``bulk_interaction/large_avalanche.py:38-144``).
"""

from __future__ import annotations

from dataclasses import dataclass, fields

import numpy as np

from . import _lib
from .grid import DeviceGrid

LITERATURE_REDUCED_ORDER_UNCALIBRATED = "LITERATURE_BASED_REDUCED_ORDER_UNCALIBRATED"


@dataclass(frozen=True)
class MaterialScenario:
    name: str
    assumed_bulk_density_kg_m3: float
    internal_friction_angle_deg: float
    cohesion_proxy_pa: float
    tool_friction_coefficient: float
    start_angle_deg: float
    stop_angle_deg: float
    mobile_friction_coefficient: float

    def __post_init__(self) -> None:
        if not isinstance(self.name, str) or not self.name.strip():
            raise ValueError("[MaterialScenario] name must be non-empty")
        if not self.assumed_bulk_density_kg_m3 > 0.0:
            raise ValueError("[MaterialScenario] assumed density must be > 0")
        if self.cohesion_proxy_pa < 0.0:
            raise ValueError("[MaterialScenario] cohesion must be non-negative")


@dataclass(frozen=True)
class LargeAvalancheTransitionConfig:
    minimum_connected_cells: int = 32
    minimum_connected_area_m2: float = 0.08
    minimum_mobilizable_volume_m3: float = 0.004
    minimum_mean_excess_start_deg: float = 0.0
    persistence_time_s: float = 0.12
    mobilization_depth_m: float = 0.08
    gravity_velocity_length_m: float = 0.25
    velocity_efficiency: float = 0.45
    mobile_activity_speed_m_s: float = 0.05
    mobile_activity_volume_m3: float = 1.0e-5
    dry_tolerance_m: float = 1.0e-8
    settled_mobile_volume_m3: float = 1.0e-5
    settled_speed_m_s: float = 0.05
    connectivity: int = 8
    parameter_basis: str = LITERATURE_REDUCED_ORDER_UNCALIBRATED
    sensitivity_case: str = "nominal_uncalibrated"

    def __post_init__(self) -> None:
        if not isinstance(self.minimum_connected_cells, int) or self.minimum_connected_cells < 1:
            raise ValueError("[LargeAvalanche] minimum_connected_cells must be >= 1")
        if self.connectivity not in (4, 8):
            raise ValueError("[LargeAvalanche] connectivity must be 4 or 8")
        numeric = np.asarray([
            self.minimum_connected_area_m2, self.minimum_mobilizable_volume_m3,
            self.minimum_mean_excess_start_deg, self.persistence_time_s,
            self.mobilization_depth_m, self.gravity_velocity_length_m, self.velocity_efficiency,
            self.mobile_activity_speed_m_s, self.mobile_activity_volume_m3, self.dry_tolerance_m,
            self.settled_mobile_volume_m3, self.settled_speed_m_s], dtype=np.float64)
        if not np.all(np.isfinite(numeric)) or np.any(numeric < 0.0):
            raise ValueError("[LargeAvalanche] numeric configuration must be finite/non-negative")
        if self.persistence_time_s <= 0.0:
            raise ValueError("[LargeAvalanche] persistence_time_s must be positive")
        if self.mobilization_depth_m <= 0.0 or self.gravity_velocity_length_m <= 0.0:
            raise ValueError("[LargeAvalanche] failure depth/velocity length must be positive")
        if not 0.0 < self.velocity_efficiency <= 1.0:
            raise ValueError("[LargeAvalanche] velocity_efficiency must lie in (0, 1]")
        if self.parameter_basis != LITERATURE_REDUCED_ORDER_UNCALIBRATED:
            raise ValueError("[LargeAvalanche] transition parameters must remain explicitly "
                             "literature-based reduced-order / uncalibrated")
        if not self.sensitivity_case:
            raise ValueError("[LargeAvalanche] sensitivity_case must be non-empty")

    @classmethod
    def from_mapping(cls, value: dict) -> "LargeAvalancheTransitionConfig":
        if not isinstance(value, dict):
            raise TypeError("[LargeAvalanche] configuration must be a mapping")
        names = {f.name for f in fields(cls)}
        unknown = sorted(set(value) - names)
        if unknown:
            raise ValueError(f"[LargeAvalanche] unknown configuration fields: {unknown}")
        return cls(**value)


@dataclass(frozen=True)
class LabelDiagnosis:
    """Diagnosis subset of the reference ``DeviceLargeAvalancheResult`` (:469-507)."""

    classification: str
    unstable_cell_count: int
    connected_region_count: int
    largest_connected_cell_count: int
    largest_connected_area_m2: float
    largest_connected_mobilizable_volume_m3: float
    mean_excess_start_deg: float
    maximum_excess_start_deg: float
    mean_excess_stop_deg: float
    maximum_excess_stop_deg: float
    persistence_s: float
    candidate: bool
    transition_ready: bool
    winner_label: int
    union_iterations: int


@dataclass(frozen=True)
class DeviceLargeAvalancheResult:
    """Field set of the reference's DeviceLargeAvalancheResult
    (runtime/gpu_large_avalanche.py:469-507)."""

    classification: str
    transitioned: bool
    unstable_cell_count: int
    connected_region_count: int
    largest_connected_cell_count: int
    largest_connected_area_m2: float
    largest_connected_mobilizable_volume_m3: float
    mean_excess_start_deg: float
    maximum_excess_start_deg: float
    persistence_s: float
    transferred_volume_m3: float
    gravity_initiation_impulse_kg_m_s: np.ndarray
    residual_seed_tile_ids: np.ndarray
    union_iterations: int
    parameter_basis: str
    sensitivity_case: str
    newly_activated_volume_m3: float
    reactivated_volume_m3: float
    newly_activated_area_m2: float
    reactivated_area_step_m2: float
    cumulative_resting_to_mobile_m3: float
    cumulative_mobile_to_resting_m3: float
    unique_cells_ever_activated: int
    cells_activated_more_than_once: int
    unique_activated_area_m2: float
    reactivated_area_m2: float
    retired_candidate_area_m2: float
    current_mobile_volume_m3: float
    moving_mobile_volume_m3: float
    maximum_mobile_speed_m_s: float
    active_tile_count: int
    net_terrain_volume_change_m3: float
    net_spatial_transfer_m3: float
    mean_activated_slope_deg: float
    maximum_activated_slope_deg: float
    mean_slope_minus_theta_stop_deg: float
    mean_theta_start_minus_slope_deg: float


class B200LargeAvalancheBridge:
    NO_LARGE_EVENT = "NO_LARGE_EVENT"
    LOCAL_STATIC_INSTABILITY = "LOCAL_STATIC_INSTABILITY"
    PERSISTING_LARGE_UNSTABLE_REGION = "PERSISTING_LARGE_UNSTABLE_REGION"
    LARGE_AVALANCHE_MOBILE_PATH = "LARGE_AVALANCHE_MOBILE_PATH"

    def __init__(self, grid: DeviceGrid, material: MaterialScenario,
                 config: LargeAvalancheTransitionConfig | None = None, *,
                 gravity_m_s2: float = 9.81, state=None) -> None:
        self.state = state
        self._clock_s = 0.0
        self.grid = grid
        self.material = material
        self.config = config or LargeAvalancheTransitionConfig()
        self.gravity = float(gravity_m_s2)
        self._persistence_s = 0.0
        self._has_previous = False

    def reset(self) -> None:
        self._persistence_s = 0.0
        self._has_previous = False

    @staticmethod
    def label_params(material: MaterialScenario, config: LargeAvalancheTransitionConfig, *,
                     release: bool, gravity: float = 9.81) -> _lib.LabelParams:
        """The C-ABI labelling parameters of a material and transition config."""
        start = float(np.deg2rad(material.start_angle_deg))
        stop = float(np.deg2rad(material.stop_angle_deg))
        return _lib.LabelParams(
            float(np.tan(start)), float(np.tan(stop)), start, stop,
            float(material.assumed_bulk_density_kg_m3), float(gravity),
            float(material.cohesion_proxy_pa), float(config.mobilization_depth_m),
            float(config.dry_tolerance_m), float(config.mobile_activity_speed_m_s),
            int(config.connectivity), 1 if release else 0)

    def _params(self, release: bool) -> _lib.LabelParams:
        return self.label_params(self.material, self.config, release=release,
                                 gravity=self.gravity)

    def label(self, *, release_settled_latches: bool = True) -> _lib.LabelStats:
        """Yield + components + component reductions (no classification)."""
        st = _lib.LabelStats()
        _lib.check(self.grid.ctx, _lib.load().sb_label(
            self.grid.ctx, self._params(release_settled_latches), st), "label")
        return st

    def labels(self) -> np.ndarray:
        """Canonical labels: -1 for stable cells, else the component's min flat index."""
        return self.grid.download("labels")

    def observe(self, dt_s: float, *, release_settled_latches: bool = True) -> LabelDiagnosis:
        dt = float(dt_s)
        if not np.isfinite(dt) or dt <= 0.0:
            raise ValueError("[GpuLargeAvalanche] dt_s must be finite/positive")
        st = self.label(release_settled_latches=release_settled_latches)
        cfg = self.config
        largest = int(st.largest_connected_cell_count)
        area = float(st.largest_connected_area_m2)
        volume = float(st.largest_connected_mobilizable_volume_m3)
        mean_start = float(np.rad2deg(st.excess_start_sum_rad / largest)) if largest else 0.0
        mean_stop = float(np.rad2deg(st.excess_stop_sum_rad / largest)) if largest else 0.0
        extent_pass = largest >= cfg.minimum_connected_cells and area >= cfg.minimum_connected_area_m2
        volume_pass = volume >= cfg.minimum_mobilizable_volume_m3
        excess_pass = mean_start >= cfg.minimum_mean_excess_start_deg
        candidate = extent_pass and volume_pass and excess_pass
        overlap = int(st.previous_overlap) > 0
        if candidate:
            self._persistence_s = (self._persistence_s + dt if overlap or not self._has_previous
                                   else dt)
        else:
            self._persistence_s = 0.0
        ready = candidate and self._persistence_s >= cfg.persistence_time_s
        if ready:
            cls = self.LARGE_AVALANCHE_MOBILE_PATH
        elif candidate:
            cls = self.PERSISTING_LARGE_UNSTABLE_REGION
        elif int(st.unstable_cell_count) > 0:
            cls = self.LOCAL_STATIC_INSTABILITY
        else:
            cls = self.NO_LARGE_EVENT
        _lib.check(self.grid.ctx, _lib.load().sb_label_commit(
            self.grid.ctx, 1 if candidate else 0,
            1 if cls == self.LOCAL_STATIC_INSTABILITY else 0), "label commit")
        self._has_previous = candidate
        return LabelDiagnosis(
            cls, int(st.unstable_cell_count), int(st.connected_region_count), largest, area,
            volume, mean_start, float(np.rad2deg(st.excess_start_max_rad)), mean_stop,
            float(np.rad2deg(st.excess_stop_max_rad)), self._persistence_s, candidate, ready,
            int(st.winner_root), int(st.union_passes))


def _observe_and_maybe_mobilize(self, dt_s: float, *, release_settled_latches: bool = True
                                ) -> DeviceLargeAvalancheResult:
    """Diagnosis, then (when the transition is ready) activation of the selected
    component, and the lifecycle summary (reference
    runtime/gpu_large_avalanche.py:541-676, :785-840)."""
    diag = self.observe(dt_s, release_settled_latches=release_settled_latches)
    lib = _lib.load()
    cfg = self.config
    self._clock_s += float(dt_s)
    now = float(getattr(self.state, "timestamp_device_s", self._clock_s)) if self.state else self._clock_s
    mob = _lib.MobilizeStats()
    if diag.transition_ready:
        _lib.check(self.grid.ctx, lib.sb_avalanche_mobilize(
            self.grid.ctx, now, float(cfg.mobilization_depth_m), float(cfg.dry_tolerance_m), mob),
            "mobilize")
    start = float(np.deg2rad(self.material.start_angle_deg))
    stop = float(np.deg2rad(self.material.stop_angle_deg))
    per = _lib.PersistenceStats()
    _lib.check(self.grid.ctx, lib.sb_avalanche_persistence(
        self.grid.ctx, start, stop, float(cfg.dry_tolerance_m),
        float(cfg.mobile_activity_speed_m_s), per), "persistence")
    ntiles = int(lib.sb_frontier_tile_count(self.grid.ctx))
    flags = np.zeros(max(ntiles, 1), dtype=np.int32)
    _lib.check(self.grid.ctx, lib.sb_frontier_active_tiles(self.grid.ctx, flags.ctypes.data,
                                                           int(ntiles)), "seed tiles")
    seeds = np.flatnonzero(flags[:ntiles])
    unique = int(per.unique_cells_ever_activated)

    def mean_deg(x):
        return float(np.rad2deg(x / unique)) if unique else 0.0

    return DeviceLargeAvalancheResult(
        classification=diag.classification, transitioned=float(mob.transferred_volume_m3) > 0.0,
        unstable_cell_count=diag.unstable_cell_count,
        connected_region_count=diag.connected_region_count,
        largest_connected_cell_count=diag.largest_connected_cell_count,
        largest_connected_area_m2=diag.largest_connected_area_m2,
        largest_connected_mobilizable_volume_m3=diag.largest_connected_mobilizable_volume_m3,
        mean_excess_start_deg=diag.mean_excess_start_deg,
        maximum_excess_start_deg=diag.maximum_excess_start_deg,
        persistence_s=diag.persistence_s, transferred_volume_m3=float(mob.transferred_volume_m3),
        gravity_initiation_impulse_kg_m_s=np.zeros(2),
        residual_seed_tile_ids=np.asarray(seeds, dtype=np.int32),
        union_iterations=diag.union_iterations,
        parameter_basis=getattr(cfg, "parameter_basis", ""),
        sensitivity_case=getattr(cfg, "sensitivity_case", ""),
        newly_activated_volume_m3=float(mob.newly_activated_volume_m3),
        reactivated_volume_m3=float(mob.reactivated_volume_m3),
        newly_activated_area_m2=float(mob.newly_activated_area_m2),
        reactivated_area_step_m2=float(mob.reactivated_area_step_m2),
        cumulative_resting_to_mobile_m3=float(per.cumulative_r2m_m3),
        cumulative_mobile_to_resting_m3=float(per.cumulative_m2r_m3),
        unique_cells_ever_activated=unique,
        cells_activated_more_than_once=int(per.cells_activated_more_than_once),
        unique_activated_area_m2=float(per.unique_activated_area_m2),
        reactivated_area_m2=float(per.reactivated_area_m2),
        retired_candidate_area_m2=float(per.retired_candidate_area_m2),
        current_mobile_volume_m3=float(per.current_mobile_volume_m3),
        moving_mobile_volume_m3=float(per.moving_mobile_volume_m3),
        maximum_mobile_speed_m_s=float(per.maximum_mobile_speed_m_s),
        active_tile_count=int(per.active_tile_count),
        net_terrain_volume_change_m3=float(per.net_terrain_volume_change_m3),
        net_spatial_transfer_m3=float(per.net_spatial_transfer_m3),
        mean_activated_slope_deg=mean_deg(per.activated_slope_sum_rad),
        maximum_activated_slope_deg=float(np.rad2deg(per.activated_slope_max_rad)),
        mean_slope_minus_theta_stop_deg=mean_deg(per.slope_minus_stop_sum_rad),
        mean_theta_start_minus_slope_deg=mean_deg(per.start_minus_slope_sum_rad),
    )


B200LargeAvalancheBridge.observe_and_maybe_mobilize = _observe_and_maybe_mobilize


def label_mask(grid: DeviceGrid, mask: np.ndarray, connectivity: int = 8):
    """Connected components of ``mask`` on the GPU -> (canonical labels, LabelStats)."""
    m = np.ascontiguousarray(np.asarray(mask, dtype=bool).astype(np.int32))
    if m.shape != grid.shape:
        raise ValueError("[LargeAvalanche] connected mask must match the grid shape")
    st = _lib.LabelStats()
    _lib.check(grid.ctx, _lib.load().sb_label_mask(grid.ctx, m.ctypes.data, int(connectivity), st),
               "label mask")
    return grid.download("labels"), st


def largest_connected_region(mask: np.ndarray, connectivity: int, *, device: int = 0):
    """GPU drop-in for ``_largest_connected_region`` (large_avalanche.py:711-778).

    Returns (largest component mask, region count, largest size).  Ties resolve
    to the component with the smallest flat index, which is also the first
    maximum in the reference's run-order dictionary.
    """
    source = np.asarray(mask, dtype=bool)
    if source.ndim != 2:
        raise ValueError("[LargeAvalanche] connected mask must be 2-D")
    if not np.any(source):
        return np.zeros_like(source), 0, 0
    if min(source.shape) < 2:
        raise ValueError("[soilb200] masks need at least 2 rows and 2 columns")
    grid = DeviceGrid(source.shape, 1.0, 1.0, precision="fx32", device=device)
    try:
        labels, st = label_mask(grid, source, connectivity)
    finally:
        grid.close()
    return labels == int(st.winner_root), int(st.connected_region_count), \
        int(st.largest_connected_cell_count)


def label_mask_preallocated(mask_ptr: int, labels_ptr: int, shape, connectivity: int = 8, *,
                            dx_m: float = 1.0, dy_m: float = 1.0, stream: int = 0):
    """Connected components with no device allocation by this library.

    For callers that cannot allocate device memory while they run (a plugin
    frame callback with a fixed memory budget handed over at start-up, where
    cudaMalloc may block or synchronise the device).  ``mask_ptr`` / ``labels_ptr`` are
    device addresses of int32 row-major ``shape`` arrays (e.g. from
    ``tensor.data_ptr()``); the scratch is a fixed static device array, so
    ``shape`` may hold at most 524288 cells and concurrent calls must not
    overlap on the GPU.  Returns the ``LabelStats`` record.
    """
    ny, nx = int(shape[0]), int(shape[1])
    st = _lib.LabelStats()
    rc = _lib.load().sb_label_mask_static(mask_ptr, labels_ptr, ny, nx, int(connectivity),
                                          float(dx_m), float(dy_m), stream, st)
    if rc == _lib.SB_ERR_CAPACITY:
        raise ValueError(f"[soilb200] {ny}x{nx} = {ny * nx} cells exceeds the static "
                         "scratch capacity of 524288 cells")
    if rc == _lib.SB_ERR_BAD_ARG:
        raise ValueError("[soilb200] invalid pointers, shape or connectivity")
    if rc == _lib.SB_ERR_NONCONVERGENCE:
        raise _lib.NumericalNonconvergenceError(
            "NUMERICAL_NONCONVERGENCE: device avalanche connected components")
    if rc != _lib.SB_OK:
        raise _lib.B200DeviceError(f"[soilb200] sb_label_mask_static failed with status {rc}")
    return st
