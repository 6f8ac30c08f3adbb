"""Device-authoritative bulk state and the production Mobile V2 operator.

``B200BulkState`` plays the role of the reference's ``DeviceBulkState``
(``runtime/bulk_state_authority.py:493-1406``): one resident field set per
terrain (``z_base`` zero, ``b_eff`` = initial resting heightmap, ``mobile``,
``momentum_x/y``, ``frontier_reached``), Triangle-A-C vertex weights (computed
in closed form on the device), the reservoir reduction, and the donor-limited
entrain/deposit exchange.  ``B200ProductionMobileV2Solver`` mirrors
``WarpProductionMobileV2Solver`` (``bulk_interaction/warp_mobile_v2.py:91-253``)
and returns the same ``WarpMobileStep`` record fields
(``bulk_interaction/warp_mobile_layer.py:349-371``).
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from .grid import DeviceGrid, choose_quantization
from .mobile_v2 import MobileV2Config, mobile_params


class BulkStateAuthorityError(RuntimeError):
    """Forbidden host/device transfer (reference BulkStateAuthorityError)."""


class B200BulkState:
    def __init__(self, shape, dx_m: float, dy_m: float, initial_resting_m: np.ndarray, *,
                 z_base_m: np.ndarray | None = None, device: int = 0, tile_size: int = 64,
                 precision: str = "fx32", height_exponent: int | None = None,
                 datum_m: float | None = None, mobile_headroom_m: float = 0.0) -> None:
        if int(tile_size) < 4:
            raise ValueError("[DeviceBulkState] tile_size must be >= 4")
        initial = np.asarray(initial_resting_m, dtype=np.float64)
        if initial.shape != tuple(shape):
            raise ValueError("[DeviceBulkState] initial heightmap shape mismatch")
        if not np.all(np.isfinite(initial)):
            raise ValueError("[DeviceBulkState] initial heightmap must be finite")
        z = np.zeros(initial.shape) if z_base_m is None else np.asarray(z_base_m, np.float64)
        if precision == "fx32" and (height_exponent is None or datum_m is None):
            k, d = choose_quantization(initial, z, mobile=np.asarray([mobile_headroom_m]))
            height_exponent = k if height_exponent is None else height_exponent
            datum_m = d if datum_m is None else datum_m
        self.grid = DeviceGrid(initial.shape, dx_m, dy_m, precision=precision, device=device,
                               tile_size=tile_size, height_exponent=height_exponent or 28,
                               datum_m=datum_m or 0.0)
        self.shape = self.grid.shape
        self.size = self.grid.size
        self.tile_size = int(tile_size)
        self.precision = precision
        self._timestamp_device_s = 0.0
        self._dirty_tile_ids: set[int] = set()
        self.grid.upload("z_base", z)
        self.grid.upload("b_eff", initial)
        self.grid.upload("mobile", np.zeros(initial.shape))
        self.grid.upload("momentum_x", np.zeros(initial.shape))
        self.grid.upload("momentum_y", np.zeros(initial.shape))
        # reference for the large-avalanche net terrain change (initial_resting)
        _lib.check(self.grid.ctx, _lib.load().sb_avalanche_set_initial_resting(self.grid.ctx),
                   "initial resting")

    # ------------------------------------------------------------------ time
    @property
    def timestamp_device_s(self) -> float:
        return self._timestamp_device_s

    def advance_time(self, dt_s: float) -> None:
        dt = float(dt_s)
        if not np.isfinite(dt) or dt < 0.0:
            raise ValueError("[DeviceBulkState] dt_s must be finite/non-negative")
        self._timestamp_device_s += dt

    @property
    def tile_shape(self) -> tuple[int, int]:
        return ((self.shape[0] + self.tile_size - 1) // self.tile_size,
                (self.shape[1] + self.tile_size - 1) // self.tile_size)

    @property
    def tile_count(self) -> int:
        t = self.tile_shape
        return t[0] * t[1]

    def close(self) -> None:
        self.grid.close()

    # ------------------------------------------------------ surface publication
    def mark_dirty_tiles(self, tile_ids) -> None:
        for tile_id in np.asarray(tuple(tile_ids), dtype=np.int64).ravel():
            if tile_id < 0 or tile_id >= self.tile_count:
                raise ValueError("[DeviceBulkState] dirty tile ID outside grid")
            self._dirty_tile_ids.add(int(tile_id))

    def mark_dirty_bbox(self, bbox_yx) -> None:
        row0, row1, col0, col1 = (int(v) for v in bbox_yx)
        if row1 <= row0 or col1 <= col0:
            return
        tiles_y, tiles_x = self.tile_shape
        fy, ly = max(0, row0 // self.tile_size), min(tiles_y - 1, (row1 - 1) // self.tile_size)
        fx, lx = max(0, col0 // self.tile_size), min(tiles_x - 1, (col1 - 1) // self.tile_size)
        self.mark_dirty_tiles(r * tiles_x + c for r in range(fy, ly + 1) for c in range(fx, lx + 1))

    def capture_surface_for_dirty_tracking(self) -> None:
        """Snapshot the resident free surface before a mutating device operator."""
        _lib.check(self.grid.ctx, _lib.load().sb_surface_capture(self.grid.ctx), "capture")

    def collect_surface_dirty_tiles(self, *, tolerance_m: float = 1.0e-10) -> np.ndarray:
        """Tiles whose surface moved since the snapshot (compact flags only)."""
        tol = float(tolerance_m)
        if not np.isfinite(tol) or tol < 0.0:
            raise ValueError("[DeviceBulkState] dirty tolerance must be finite/non-negative")
        flags = np.zeros(self.tile_count, dtype=np.int32)
        _lib.check(self.grid.ctx, _lib.load().sb_surface_dirty_tiles(
            self.grid.ctx, tol, flags.ctypes.data, int(flags.size)), "dirty tiles")
        ids = np.flatnonzero(flags).astype(np.int32)
        self.mark_dirty_tiles(ids)
        return ids

    def consume_dirty_tile_ids(self) -> np.ndarray:
        out = np.asarray(sorted(self._dirty_tile_ids), dtype=np.int32)
        self._dirty_tile_ids.clear()
        return out

    def download_dirty_tiles(self, tile_ids=None) -> dict:
        """Current free surface of the selected (default: all dirty) tiles, each
        with its one-cell overlap to the next tile, as the reference publishes."""
        selected = (np.asarray(tuple(tile_ids), dtype=np.int32) if tile_ids is not None
                    else self.consume_dirty_tile_ids())
        tiles_y, tiles_x = self.tile_shape
        out = {}
        for tile in selected:
            t = int(tile)
            if t < 0 or t >= tiles_y * tiles_x:
                raise ValueError("[DeviceBulkState] dirty tile ID outside grid")
            row, col = divmod(t, tiles_x)
            r0, c0 = row * self.tile_size, col * self.tile_size
            r1 = min(r0 + self.tile_size + 1, self.shape[0])
            c1 = min(c0 + self.tile_size + 1, self.shape[1])
            buf = np.empty((r1 - r0, c1 - c0), dtype=np.float64)
            _lib.check(self.grid.ctx, _lib.load().sb_surface_region(
                self.grid.ctx, r0, r1, c0, c1, buf.ctypes.data), "tile download")
            out[t] = buf
        return out

    def sample_surface_bilinear(self, row_col, *, source: str) -> np.ndarray:
        """Batched bilinear free-surface heights at fractional (row, col)."""
        if not source:
            raise ValueError("[DeviceBulkState] terrain query source must be non-empty")
        q = np.asarray(row_col, dtype=np.float64)
        if q.ndim != 2 or q.shape[1] != 2 or not np.all(np.isfinite(q)):
            raise ValueError("[DeviceBulkState] terrain queries must be finite [N,2]")
        if q.shape[0] == 0:
            return np.empty(0, dtype=np.float64)
        rows = np.ascontiguousarray(q[:, 0])
        cols = np.ascontiguousarray(q[:, 1])
        out = np.empty(q.shape[0], dtype=np.float64)
        _lib.check(self.grid.ctx, _lib.load().sb_surface_sample_bilinear(
            self.grid.ctx, rows.ctypes.data, cols.ctypes.data, int(q.shape[0]), out.ctypes.data),
            "surface query")
        return out

    # ---------------------------------------------------------------- ledger
    def reservoir_reduction(self, density_kg_m3: float) -> dict:
        density = float(density_kg_m3)
        if not np.isfinite(density) or density <= 0.0:
            raise ValueError("[DeviceBulkState] density must be finite/positive")
        L = _lib.MobileLedger()
        params = mobile_params(MobileV2Config(dx_m=self.grid.dx, dy_m=self.grid.dy),
                               density_kg_m3=density)
        _lib.check(self.grid.ctx, _lib.load().sb_mobile_ledger_of(self.grid.ctx, params, L),
                   "ledger")
        return {
            "resting_volume_m3": float(L.resting_volume_w_m3),
            "mobile_volume_m3": float(L.volume_w_m3),
            "mobile_momentum_kg_m_s": np.asarray([L.momentum_w[0], L.momentum_w[1], 0.0]),
            "resting_quanta_w6": int(L.resting_w_quanta),
            "mobile_quanta_w6": int(L.volume_w_quanta),
        }

    # -------------------------------------------------------------- exchange
    @staticmethod
    def _indices(flat_indices, size: int) -> np.ndarray:
        idx = np.ascontiguousarray(np.asarray(flat_indices, dtype=np.int32).reshape(-1))
        if np.any(idx < 0) or np.any(idx >= size):
            raise ValueError("[DeviceBulkState] entrainment index outside state")
        return idx

    def entrain_host_indices(self, flat_indices, requested_depth_m, *, reason: str) -> float:
        if not reason:
            raise ValueError("[DeviceBulkState] entrainment reason must be non-empty")
        idx = self._indices(flat_indices, self.size)
        depth = np.ascontiguousarray(np.asarray(requested_depth_m, dtype=np.float64).reshape(-1))
        if depth.shape != idx.shape or not np.all(np.isfinite(depth)):
            raise ValueError("[DeviceBulkState] invalid entrainment request")
        out = C.c_double(0.0)
        _lib.check(self.grid.ctx, _lib.load().sb_entrain(
            self.grid.ctx, idx.ctypes.data, depth.ctypes.data, int(idx.size), C.byref(out)),
            "entrain")
        return float(out.value)

    def entrain_to_surface(self, flat_indices, target_surface_m, *, reason: str) -> float:
        """Entrain resting material above ``target_surface_m`` (a tool cut)."""
        if not reason:
            raise ValueError("[DeviceBulkState] entrainment reason must be non-empty")
        idx = self._indices(flat_indices, self.size)
        target = np.ascontiguousarray(np.asarray(target_surface_m, dtype=np.float64).reshape(-1))
        if target.shape != idx.shape or not np.all(np.isfinite(target)):
            raise ValueError("[DeviceBulkState] invalid entrainment request")
        out = C.c_double(0.0)
        _lib.check(self.grid.ctx, _lib.load().sb_entrain_to_surface(
            self.grid.ctx, idx.ctypes.data, target.ctypes.data, int(idx.size), C.byref(out)),
            "entrain")
        return float(out.value)

    def deposit_host_indices(self, flat_indices, requested_depth_m, *, density_kg_m3: float,
                             reason: str) -> dict:
        if not reason:
            raise ValueError("[DeviceBulkState] deposition reason must be non-empty")
        idx = self._indices(flat_indices, self.size)
        depth = np.ascontiguousarray(np.asarray(requested_depth_m, dtype=np.float64).reshape(-1))
        if depth.shape != idx.shape or not np.all(np.isfinite(depth)):
            raise ValueError("[DeviceBulkState] invalid deposition request")
        out = np.zeros(3)
        _lib.check(self.grid.ctx, _lib.load().sb_deposit(
            self.grid.ctx, idx.ctypes.data, depth.ctypes.data, int(idx.size),
            float(density_kg_m3), out.ctypes.data), "deposit")
        return {"deposited_volume_m3": float(out[0]),
                "removed_mobile_momentum_kg_m_s": np.asarray([out[1], out[2], 0.0])}

    def set_tool_forcing_mask(self, mask) -> None:
        """Cells under active tool forcing (the reference's ``material_mask``):
        deposition leaves them alone."""
        self.grid.upload("forcing", np.asarray(mask, dtype=bool).astype(np.int32))

    # ------------------------------------------------------------ host view
    def explicit_host_view(self, *, source: str = "acceptance") -> dict:
        """Full-field download at an explicit boundary (never in the step path)."""
        if source not in {"acceptance", "checkpoint", "debug"}:
            raise BulkStateAuthorityError("[DeviceBulkState] invalid host view source")
        g = self.grid
        return {
            "z_base": g.download("z_base"),
            "b_eff": g.download("b_eff"),
            "mobile": g.download("mobile"),
            "momentum": np.stack((g.download("momentum_x"), g.download("momentum_y")), axis=-1),
            "frontier_reached": g.download("frontier_reached"),
        }


@dataclass(frozen=True)
class WarpMobileStep:
    """Field set of the reference production record (warp_mobile_layer.py:349-371)."""

    volume_before_m3: float
    volume_after_m3: float
    momentum_before_terrain_kg_m_s: np.ndarray
    momentum_after_terrain_kg_m_s: np.ndarray
    gravity_pressure_impulse_terrain_ns: np.ndarray
    basal_friction_impulse_terrain_ns: np.ndarray
    tool_impulse_on_mobile_terrain_ns: np.ndarray
    numerical_dissipative_impulse_terrain_ns: np.ndarray
    maximum_speed_m_s: float
    substeps: int
    cfl_limited: bool
    kinetic_energy_before_j: float
    kinetic_energy_after_j: float
    gravity_pressure_work_j: float
    basal_friction_work_j: float
    tool_work_j: float
    transport_numerical_energy_residual_j: float
    donor_export_m3: float
    receiver_import_m3: float
    transport_mass_residual_m3: float
    advected_momentum_crossings_kg_m_s: np.ndarray


class B200ProductionMobileV2Solver:
    """Mobile V2 on persistent device fields (reference warp_mobile_v2.py:91-253)."""

    backend_name = "GPU_B200_MOBILE_V2_PRODUCTION_SHARED_STATE"

    def __init__(self, *, state: B200BulkState | None = None,
                 config: MobileV2Config | None = None) -> None:
        self.config = config or MobileV2Config()
        self.state: B200BulkState | None = None
        self.material = None
        self.last_stats: _lib.MobileStats | None = None
        if state is not None:
            self.state = state

    def bind_device_state(self, state: B200BulkState, material, grid=None, integrator=None) -> None:
        del grid, integrator
        if not isinstance(state, B200BulkState):
            raise ValueError("[MobileV2Production] state must be a B200BulkState")
        self.state = state
        self.material = material

    def step_resident(self, dt_s: float, **_) -> WarpMobileStep:
        if self.state is None:
            raise RuntimeError("[MobileV2Production] bind state first")
        density = float(getattr(self.material, "assumed_bulk_density_kg_m3", 1.0))
        stats = _lib.MobileStats()
        params = mobile_params(self.config, density_kg_m3=density)
        g = self.state.grid
        _lib.check(g.ctx, _lib.load().sb_mobile_step(g.ctx, float(dt_s), params, stats),
                   "sb_mobile_step")
        self.last_stats = stats
        return production_record(stats, density, g.dx * g.dy)

    def diagnostics(self) -> dict:
        return {
            "backend_name": self.backend_name,
            "state": ["z_base", "b_eff", "mobile", "momentum_x", "momentum_y"],
            "pressure_flux": "0.5*K*g*h^2_CONSERVATIVE_FACE_FLUX",
            "K_classification": "ENGINEERING_CLOSURE_UNCALIBRATED",
        }


@dataclass(frozen=True)
class WarpDepositionStep:
    """Record of one deposition step (reference warp_deposition.py:136-140)."""

    deposited_volume_m3: float
    parameter_status: str
    removed_mobile_momentum_terrain_kg_m_s: np.ndarray


class B200DepositionOperator:
    """Incremental Mobile -> Resting deposition on the resident state
    (reference bulk_interaction/warp_deposition.py:143-255)."""

    backend_name = "GPU_B200_INCREMENTAL_DEPOSITION"

    def __init__(self, *, settling_rate_m_s: float = 0.30, speed_threshold_m_s: float = 0.18,
                 device=0, runtime=None) -> None:
        del device, runtime
        if settling_rate_m_s <= 0.0 or speed_threshold_m_s < 0.0:
            raise ValueError("[WarpDeposition] invalid configuration")
        self.settling_rate_m_s = float(settling_rate_m_s)
        self.speed_threshold_m_s = float(speed_threshold_m_s)
        self._state: B200BulkState | None = None

    def bind_device_state(self, state: B200BulkState) -> None:
        if not isinstance(state, B200BulkState):
            raise ValueError("[WarpDeposition] state/runtime ownership mismatch")
        self._state = state

    def step_resident(self, material, dt_s: float, *,
                      settle_subcell_tail: bool = False) -> WarpDepositionStep:
        if self._state is None:
            raise RuntimeError("[WarpDeposition] bind DeviceBulkState first")
        dt = float(dt_s)
        if not np.isfinite(dt) or dt <= 0.0:
            raise ValueError("[WarpDeposition] dt_s must be finite/positive")
        p = _lib.DepositionParams(self.settling_rate_m_s, self.speed_threshold_m_s,
                                  float(material.assumed_bulk_density_kg_m3), 9.81,
                                  float(material.cohesion_proxy_pa),
                                  float(material.stop_angle_deg), int(bool(settle_subcell_tail)), 0)
        out = _lib.DepositionStats()
        g = self._state.grid
        _lib.check(g.ctx, _lib.load().sb_deposition_step(g.ctx, dt, p, out), "deposition")
        return WarpDepositionStep(
            deposited_volume_m3=float(out.deposited_volume_m3),
            parameter_status="LITERATURE_BASED_REDUCED_ORDER_UNCALIBRATED",
            removed_mobile_momentum_terrain_kg_m_s=np.asarray(
                [out.removed_momentum_kg_m_s[0], out.removed_momentum_kg_m_s[1], 0.0]))

    def diagnostics(self) -> dict:
        return {
            "backend_name": self.backend_name,
            "resident_state": ["b_eff", "mobile", "momentum_x", "momentum_y"],
            "semantics": "incremental_mobile_to_resting_below_cohesive_stop_yield",
            "momentum_removal": "EXPLICITLY_REPORTED",
        }


def production_record(stats: _lib.MobileStats, density: float, area: float) -> WarpMobileStep:
    """WarpMobileStep from device ledgers (reference warp_mobile_v2.py:217-245)."""
    b, a = stats.before, stats.after
    before_p = np.asarray([b.momentum_w[0], b.momentum_w[1], 0.0])
    after_p = np.asarray([a.momentum_w[0], a.momentum_w[1], 0.0])
    if stats.static_skip:
        return WarpMobileStep(
            b.volume_w_m3, b.volume_w_m3, before_p, before_p.copy(), np.zeros(3), np.zeros(3),
            np.zeros(3), np.zeros(3), float(b.max_speed_m_s), 0, False, float(b.kinetic_w_j),
            float(b.kinetic_w_j), 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, np.zeros(3))
    gravity = np.asarray([stats.conservative_impulse_m4_s[0],
                          stats.conservative_impulse_m4_s[1], 0.0]) * density
    friction = np.asarray([stats.friction_impulse_m4_s[0], stats.friction_impulse_m4_s[1],
                           0.0]) * density
    fwork = float(stats.friction_dissipation) * density
    # fixed point: both volumes are exact quanta sums, so equal sums give 0.0
    residual_mass = float(a.volume_w_m3 - b.volume_w_m3)
    return WarpMobileStep(
        volume_before_m3=float(b.volume_w_m3), volume_after_m3=float(a.volume_w_m3),
        momentum_before_terrain_kg_m_s=before_p, momentum_after_terrain_kg_m_s=after_p,
        gravity_pressure_impulse_terrain_ns=gravity, basal_friction_impulse_terrain_ns=friction,
        tool_impulse_on_mobile_terrain_ns=np.zeros(3),
        numerical_dissipative_impulse_terrain_ns=after_p - before_p - gravity - friction,
        maximum_speed_m_s=float(a.max_speed_m_s), substeps=int(stats.substeps),
        cfl_limited=bool(stats.cfl_limited), kinetic_energy_before_j=float(b.kinetic_w_j),
        kinetic_energy_after_j=float(a.kinetic_w_j),
        gravity_pressure_work_j=float((a.potential_w_j + a.pressure_w_j)
                                      - (b.potential_w_j + b.pressure_w_j)),
        basal_friction_work_j=fwork, tool_work_j=0.0,
        transport_numerical_energy_residual_j=float(
            (a.kinetic_w_j + a.potential_w_j + a.pressure_w_j)
            - (b.kinetic_w_j + b.potential_w_j + b.pressure_w_j) + fwork),
        donor_export_m3=0.0, receiver_import_m3=0.0,
        transport_mass_residual_m3=residual_mass,
        advected_momentum_crossings_kg_m_s=np.zeros(3))
