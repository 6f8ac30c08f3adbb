"""Repose (MiniSlope) relaxation on the GPU.

* :func:`relax_critical_slope` -- drop-in for ``slope_model.relax_critical_slope``
  (reference ``slope_model.py:273-343``): same signature, validation messages
  and ``RelaxationStats`` record; the 8-phase colored iteration runs one launch
  per iteration inside a CUDA graph loop, convergence decided on the device.
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
