"""Repose (MiniSlope) relaxation on the GPU.

* :func:`relax_critical_slope` -- drop-in for ``slope_model.relax_critical_slope``
  (reference ``slope_model.py:273-343``): same signature, validation messages
  and ``RelaxationStats`` record; the 8-phase colored iteration runs one launch
  per iteration inside a CUDA graph loop, convergence decided on the device.
* :class:`EventDrivenMinimumSlopeAdapter` -- the reference's reached-bbox
  backend (``solvers/event_driven_slope.py:16-302``): a sweep gated by a
  growing reached mask, confirmed before it stops.
* :class:`FrontierRelaxation` -- the production residual compact-frontier
  schedule (``runtime/v2_physics_core.py:1153-1254`` driving
  ``solvers/warp_compact_frontier.py``): seeds by cell (3x3 tile stencil) or
  tile, then rounds until no tile is active, all on the device.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _lib
from .grid import DeviceGrid, choose_quantization


@dataclass(frozen=True)
class RelaxationStats:
    """Same fields as the reference ``RelaxationStats`` (slope_model.py:17-23)."""

    iterations: int
    converged: bool
    max_slope: float
    volume_before: float
    volume_after: float


def _field_stats(grid: DeviceGrid, spacing) -> np.ndarray:
    out = np.zeros(4, dtype=np.float64)
    _lib.check(grid.ctx, _lib.load().sb_field_stats(grid.ctx, _lib.FIELD["b_eff"],
                                                     float(spacing[0]), float(spacing[1]),
                                                     out.ctypes.data), "field stats")
    return out


def relax_critical_slope(height: np.ndarray, grid_spacing, critical_angle_deg: float = 34.0,
                         max_iterations: int = 20_000, tolerance: float = 1e-8, *,
                         precision: str = "fp64", device: int = 0):
    """Relax all 8-neighbour slopes to ``tan(critical_angle_deg)`` on the GPU.

    Returns ``(relaxed_height, RelaxationStats)`` like the reference.  ``fp64``
    reproduces the reference bit for bit; ``fx32`` runs on int32 height quanta
    (transfers rounded up to whole quanta, exact volume conservation).
    """
    if height.ndim != 2 or min(height.shape) < 2:
        raise ValueError("height must be a 2-D array with both dimensions >= 2")
    if np.any(height < 0):
        raise ValueError("soil heights must be non-negative")
    if not 0.0 < critical_angle_deg < 90.0:
        raise ValueError("critical_angle_deg must be between 0 and 90")
    h = np.asarray(height, dtype=float)
    s0, s1 = grid_spacing
    if s0 <= 0 or s1 <= 0:
        raise ValueError("grid spacing must be positive")
    k, datum = choose_quantization(h) if precision == "fx32" else (28, 0.0)
    grid = DeviceGrid(h.shape, float(s1), float(s0), precision=precision, device=device,
                      height_exponent=k, datum_m=datum)
    try:
        grid.upload("b_eff", h)
        before = _field_stats(grid, (s0, s1))
        crit = float(np.tan(np.deg2rad(critical_angle_deg)))
        params = _lib.RelaxParams(float(s0), float(s1), crit, float(tolerance),
                                  int(max_iterations), 0)
        st = _lib.RelaxStats()
        _lib.check(grid.ctx, _lib.load().sb_relax_full(grid.ctx, params, st), "relax")
        after = _field_stats(grid, (s0, s1))
        out = grid.download("b_eff")
    finally:
        grid.close()
    area = s0 * s1
    stats = RelaxationStats(
        iterations=int(st.iterations), converged=bool(st.converged), max_slope=float(after[1]),
        volume_before=float(before[0] * area), volume_after=float(after[0] * area))
    return out, stats


@dataclass(frozen=True)
class FrontierStats:
    rounds: int
    converged: bool
    active_tiles_last_round: int
    moved_edges: int


class FrontierRelaxation:
    """Residual compact-frontier relaxation of ``b_eff`` on a :class:`DeviceGrid`.

    ``spacing`` is (axis-0 spacing, axis-1 spacing).  The reference production
    loop passes ``_neighbor_pairs(grid.dx, grid.dy)`` on its ``[row, col]``
    state, i.e. ``spacing=(dx, dy)``; that is the default here.
    """

    def __init__(self, grid: DeviceGrid, *, spacing=None, weighted: bool = True) -> None:
        self.grid = grid
        self.spacing = tuple(spacing) if spacing is not None else (grid.dx, grid.dy)
        self.weighted = bool(weighted)

    @property
    def tile_count(self) -> int:
        return int(_lib.load().sb_frontier_tile_count(self.grid.ctx))

    def seed_cells(self, flat_indices) -> None:
        idx = np.ascontiguousarray(np.unique(np.asarray(flat_indices, dtype=np.int32)))
        _lib.check(self.grid.ctx, _lib.load().sb_frontier_seed_cells(
            self.grid.ctx, idx.ctypes.data, int(idx.size)), "seed cells")

    def seed_mask(self, mask: np.ndarray) -> None:
        self.seed_cells(np.flatnonzero(np.asarray(mask, dtype=bool)))

    def seed_tiles(self, tile_ids) -> None:
        ids = np.ascontiguousarray(np.asarray(tile_ids, dtype=np.int32))
        _lib.check(self.grid.ctx, _lib.load().sb_frontier_seed_tiles(
            self.grid.ctx, ids.ctypes.data, int(ids.size)), "seed tiles")

    def active_tiles(self) -> np.ndarray:
        flags = np.zeros(self.tile_count, dtype=np.int32)
        _lib.check(self.grid.ctx, _lib.load().sb_frontier_active_tiles(
            self.grid.ctx, flags.ctypes.data, int(flags.size)), "active tiles")
        return np.flatnonzero(flags).astype(np.int32)

    def run(self, critical_slope: float, tolerance_m: float = 1e-8,
            max_rounds: int = 4096) -> FrontierStats:
        params = _lib.RelaxParams(float(self.spacing[0]), float(self.spacing[1]),
                                  float(critical_slope), float(tolerance_m), int(max_rounds),
                                  1 if self.weighted else 0)
        st = _lib.RelaxStats()
        _lib.check(self.grid.ctx, _lib.load().sb_frontier_run(self.grid.ctx, params, st),
                   "frontier")
        return FrontierStats(int(st.iterations), bool(st.converged), int(st.active_tiles),
                             int(st.moved_edges))


@dataclass(frozen=True)
class MiniSlopeConfig:
    """The relaxation keys of the reference ``SolverConfig``
    (config/loader.py:137-156) that the event-driven backend reads."""

    critical_angle_deg: float = 34.0
    tolerance: float = 1e-8
    large_avalanche_iteration_threshold: int = 1000
    numerical_safety_max_iterations: int = 1_000_000
    boundary_condition: str = "closed"


@dataclass(frozen=True)
class EventRelaxationResult:
    """Fields of the reference's ``RelaxationResult`` that this backend fills."""

    heightmap_initial: np.ndarray
    heightmap_stable: np.ndarray
    iteration_count: int
    converged: bool
    volume_before_m3: float
    volume_after_m3: float
    diagnostics: dict


def _window(mask: np.ndarray) -> list:
    rows, cols = np.nonzero(mask)
    if rows.size == 0:
        return [0, 0, 0, 0]
    return [int(rows.min()), int(cols.min()), int(rows.max()) + 1, int(cols.max()) + 1]


class EventDrivenMinimumSlopeAdapter:
    """GPU drop-in for the reference's reached-bbox MiniSlope backend
    (``solvers/event_driven_slope.py:16-302``).

    Changed cells (against the reference height, or marked with
    :meth:`mark_changed`) seed a reached mask; :meth:`solve` then runs the
    reference's direction/parity schedule on pairs with a reached endpoint
    only, growing the mask with every transfer, until a confirming scan finds
    no reachable excess above the tolerance (``sb_relax_reached``; FP64 is
    bit-identical to the reference, iteration counts equal).  Heights are
    ``H[y, x]`` like the reference's API; the device works on the transposed
    ``H[x, y]`` array, the reference's internal layout, so that its
    direction order and parities are the reference's.  ``grid`` is any object
    with ``nx, ny, dx, dy`` (the reference's ``TerrainGrid``).
    """

    backend_name = "B200_REACHED_BBOX_SWEEP"
    LOCALIZED_AVALANCHE = "LOCALIZED_AVALANCHE"
    LARGE_SUSTAINED_AVALANCHE = "LARGE_SUSTAINED_AVALANCHE"
    NO_EVENT = "NO_EVENT"

    def __init__(self, grid, config=None, *, tile_size: int = 32, precision: str = "fp64",
                 device: int = 0) -> None:
        self.tile_size = int(tile_size)
        if self.tile_size < 4:
            raise ValueError("[EventDrivenMiniSlope] tile_size must be >= 4")
        self.config = config if config is not None else MiniSlopeConfig()
        if self.config.large_avalanche_iteration_threshold < 1:
            raise ValueError("[EventDrivenMiniSlope] large avalanche threshold must be >= 1")
        if (self.config.numerical_safety_max_iterations
                < self.config.large_avalanche_iteration_threshold):
            raise ValueError("[EventDrivenMiniSlope] numerical safety limit must be >= "
                             "large avalanche threshold")
        if getattr(self.config, "boundary_condition", "closed") != "closed":
            raise ValueError("[EventDrivenMiniSlope] only the closed boundary is supported")
        self.nx, self.ny = int(grid.nx), int(grid.ny)
        self.dx, self.dy = float(grid.dx), float(grid.dy)
        self.shape = (self.ny, self.nx)
        self.precision = precision
        self.device = device
        self._grid: DeviceGrid | None = None
        self._quant = None
        self._reference_height: np.ndarray | None = None
        self._pending_changed: np.ndarray | None = None
        self.last_classification = self.NO_EVENT
        self.last_diagnostics: dict = {}

    def _device_grid(self, h_xy: np.ndarray) -> DeviceGrid:
        # H[x, y]: axis 0 = x (spacing dx), axis 1 = y (spacing dy)
        quant = choose_quantization(h_xy) if self.precision == "fx32" else (28, 0.0)
        if self._grid is None or quant != self._quant:
            if self._grid is not None:
                self._grid.close()
            self._grid = DeviceGrid((self.nx, self.ny), self.dy, self.dx,
                                    precision=self.precision, device=self.device,
                                    height_exponent=quant[0], datum_m=quant[1])
            self._quant = quant
        return self._grid

    def _validated(self, heightmap) -> np.ndarray:
        h = np.array(heightmap, dtype=np.float64, copy=True)
        if h.shape != self.shape:
            raise ValueError("[EventDrivenMiniSlope] heightmap shape mismatch")
        if not np.all(np.isfinite(h)):
            raise ValueError("[EventDrivenMiniSlope] heightmap must be finite")
        return h

    def set_reference_height(self, heightmap) -> None:
        self._reference_height = self._validated(heightmap)
        self._pending_changed = np.zeros(self.shape, dtype=bool)

    def mark_changed(self, changed_mask) -> None:
        changed = np.asarray(changed_mask, dtype=bool)
        if changed.shape != self.shape:
            raise ValueError("[EventDrivenMiniSlope] changed mask shape mismatch")
        if self._pending_changed is None:
            self._pending_changed = changed.copy()
        else:
            self._pending_changed |= changed

    def reset(self) -> None:
        self._reference_height = None
        self._pending_changed = None
        self.last_classification = self.NO_EVENT
        self.last_diagnostics = {}

    def close(self) -> None:
        if self._grid is not None:
            self._grid.close()
            self._grid = None

    def solve(self, heightmap) -> EventRelaxationResult:
        initial = self._validated(heightmap)
        if self._reference_height is None:
            self.set_reference_height(initial)
        changed = np.abs(initial - self._reference_height) > max(self.config.tolerance, 1e-12)
        if self._pending_changed is not None:
            changed |= self._pending_changed
        area = self.dx * self.dy
        volume = float(initial.sum() * area)
        if not np.any(changed):
            diag = self._diagnostics(changed, changed, 0, self.NO_EVENT)
            self._complete(initial, diag)
            return EventRelaxationResult(initial, initial.copy(), 0, True, volume, volume, diag)
        grid = self._device_grid(initial.T)
        grid.upload("b_eff", np.ascontiguousarray(initial.T))
        grid.upload("frontier_reached", np.ascontiguousarray(changed.T).astype(np.int32))
        crit = float(np.tan(np.deg2rad(self.config.critical_angle_deg)))
        params = _lib.RelaxParams(self.dx, self.dy, crit, float(self.config.tolerance),
                                  int(self.config.numerical_safety_max_iterations), 0)
        st = _lib.RelaxStats()
        _lib.check(grid.ctx, _lib.load().sb_relax_reached(grid.ctx, params, st), "relax")
        stable = np.ascontiguousarray(grid.download("b_eff").T)
        reached = np.ascontiguousarray(grid.download("frontier_reached").T != 0)
        iterations = int(st.iterations)
        ratio = float(np.count_nonzero(reached)) / reached.size
        cls = (self.LARGE_SUSTAINED_AVALANCHE
               if ratio >= 0.5 or iterations > self.config.large_avalanche_iteration_threshold
               else self.LOCALIZED_AVALANCHE)
        diag = self._diagnostics(changed, reached, iterations, cls)
        self._complete(stable, diag)
        return EventRelaxationResult(initial, stable, iterations, bool(st.converged), volume,
                                     float(stable.sum() * area), diag)

    def _diagnostics(self, seeds, reached, iterations: int, cls: str) -> dict:
        thr = int(self.config.large_avalanche_iteration_threshold)
        seed_w, reach_w = _window(seeds), _window(reached)
        count = int(np.count_nonzero(reached))
        return {
            "adapter": self.__class__.__name__, "backend": self.backend_name,
            "seed_cell_count": int(np.count_nonzero(seeds)), "reached_cell_count": count,
            "reached_cell_ratio": count / float(reached.size), "tile_size": self.tile_size,
            "seed_bbox_yx": seed_w, "propagation_bbox_yx": reach_w,
            "propagation_crossed_seed_bbox": reach_w != seed_w,
            "avalanche_classification": cls,
            "large_avalanche_iteration_threshold": thr,
            "numerical_safety_max_iterations": int(self.config.numerical_safety_max_iterations),
            "actual_iterations_to_convergence": iterations,
            "continued_beyond_large_avalanche_threshold": iterations > thr,
            "future_resting_to_mobile_transfer_required": cls == self.LARGE_SUSTAINED_AVALANCHE,
            "propagation_truncated": False,
        }

    def _complete(self, stable, diag) -> None:
        self._reference_height = np.array(stable, copy=True)
        self._pending_changed = np.zeros(self.shape, dtype=bool)
        self.last_classification = str(diag["avalanche_classification"])
        self.last_diagnostics = dict(diag)
