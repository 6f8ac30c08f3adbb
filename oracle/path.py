"""CPU restatement of the plain terrain step -- TEST INFRASTRUCTURE ONLY.

One physics step of the production GPU core restricted to the operators the
CUDA library replaces, in the reference's order
(``runtime/v2_physics_core.py:708-1003``):

1. tool entrainment to target surfaces, donor-limited by ``b_eff - z_base``
   (``runtime/bulk_state_authority.py:103-149`` ``entrain``);
2. the Mobile V2 step (``oracle.mobile_v2.step``, the FP64 restatement of
   ``experimental/mobile_v2_reference.py:191-314``);
3. large-avalanche diagnosis: cohesive start/stop yield, 8-connected
   canonical labels, the winner (largest component, ties -> smallest root)
   and its area / mobilizable volume / slope excess
   (``runtime/gpu_large_avalanche.py:58-275``), persistence and
   classification (``:620-676``), previous-candidate mask and residual seeds
   (``update_previous_and_tiles`` ``:277-306``);
4. the residual gate (``v2_physics_core.py:955-1003``): the pending frontier
   tiles run only while the mobile layer is quiet (mobile volume and speed at
   or below the settled thresholds) and no physically mobilizable yield
   exists; then the compact-frontier rounds of ``_advance_gpu_residual_frontier``
   (``:1172-1254``, ``oracle.relax.frontier_relax``, Triangle-A-C weighted).

Statistics that the GPU keeps as exact integers are kept the same way here
(area in units of dx*dy/6, mobilizable volume and slope excess in 2^-32
fixed point), so the winner record compares exactly except where a
transcendental function (``arctan``) of the C library and of CUDA differ in
the last bit.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import labels as L
from . import mobile_v2 as M
from . import relax as R

CLASSIFICATIONS = ("NO_LARGE_EVENT", "LOCAL_STATIC_INSTABILITY",
                   "PERSISTING_LARGE_UNSTABLE_REGION", "LARGE_AVALANCHE_MOBILE_PATH")
SCALE = 4294967296.0  # 2^32 fixed-point unit of the volume and excess sums


@dataclass
class PathOracleConfig:
    """Material and transition parameters of the step (defaults: the
    reference's ``LargeAvalancheTransitionConfig``, large_avalanche.py:38-66)."""

    dx: float = 0.05
    density: float = 1600.0
    cohesion: float = 0.0
    start_angle_deg: float = 38.0
    stop_angle_deg: float = 30.0
    mobile_friction: float = 0.55
    gravity: float = 9.81
    minimum_connected_cells: int = 32
    minimum_connected_area_m2: float = 0.08
    minimum_mobilizable_volume_m3: float = 0.004
    minimum_mean_excess_start_deg: float = 0.0
    persistence_time_s: float = 0.12
    mobilization_depth_m: float = 0.08
    mobile_activity_speed_m_s: float = 0.05
    dry_tolerance_m: float = 1.0e-8
    settled_mobile_volume_m3: float = 1.0e-5
    settled_speed_m_s: float = 0.05
    connectivity: int = 8
    tile: int = 64
    tolerance_m: float = 1.0e-8
    max_rounds: int = 4096
    residual: str = "gated"   # "never" | "gated" | "always"


@dataclass
class PathOracleStep:
    substeps: int
    entrained_m3: float
    classification: str
    unstable_cells: int
    regions: int
    largest: int
    winner: int
    area6: int
    volume_fx: int
    exc_start_fx: int
    residual_ran: bool
    residual_rounds: int
    mobile_volume_m3: float
    max_speed_m_s: float
    labels: np.ndarray


def entrain(b, z, h, idx, target, w):
    """In-place donor-limited entrainment; returns the moved volume sum(d*w)."""
    if idx is None or len(idx) == 0:
        return 0.0
    idx = np.asarray(idx, dtype=np.int64)
    fb, fh, fz = b.reshape(-1), h.reshape(-1), z.reshape(-1)
    avail = np.maximum(fb[idx] - fz[idx], 0.0)
    d = np.minimum(np.maximum(fb[idx] - np.asarray(target, np.float64), 0.0), avail)
    fb[idx] = fb[idx] - d
    fh[idx] = fh[idx] + d
    return float(np.sum(d * w.reshape(-1)[idx]))


class PathOracle:
    """State + one ``step`` of the FP64 plain path on (ny, nx) cells."""

    def __init__(self, b_eff, z_base, cfg: PathOracleConfig | None = None):
        self.cfg = cfg or PathOracleConfig()
        c = self.cfg
        self.b = np.array(b_eff, dtype=np.float64)
        self.z = np.array(z_base, dtype=np.float64)
        self.h = np.zeros_like(self.b)
        self.q = np.zeros(self.b.shape + (2,))
        self.shape = self.b.shape
        self.w = R.vertex_weights(self.shape, c.dx, c.dx)
        self.w6 = R.vertex_weights6(self.shape)
        self.previous = np.zeros(self.shape, dtype=bool)
        self.reached = np.zeros(self.shape, dtype=bool)
        self.tiles_x = (self.shape[1] + c.tile - 1) // c.tile
        self.pending = np.empty(0, dtype=np.int32)
        self.persistence_s = 0.0
        self.has_previous = False
        self.mobile_cfg = M.OracleConfig(dx_m=c.dx, dy_m=c.dx, start_angle_deg=c.start_angle_deg,
                                         stop_angle_deg=c.stop_angle_deg,
                                         basal_friction_coefficient=c.mobile_friction)

    # -- mobile layer summaries of the after-step ledger (warp_mobile_v2.py:28-54)
    def _mobile_volume(self) -> float:
        return float(np.sum(self.h * self.w))

    def _max_speed(self) -> float:
        h = self.h
        wet = h > self.mobile_cfg.dry_tolerance_m
        if not np.any(wet):
            return 0.0
        qx, qy = self.q[..., 0][wet], self.q[..., 1][wet]
        hw = h[wet]
        return float(np.max(np.sqrt((qx * qx + qy * qy) / (hw * hw))))

    def _winner_record(self, y, labels):
        """Component summary + the winner's integer sums (gpu_large_avalanche.py:200-275)."""
        c = self.cfg
        regions, largest, winner, total = L.component_summary(labels)
        if winner < 0:
            return regions, 0, -1, total, 0, 0, 0, 0
        sel = labels == winner
        area6 = int(self.w6[sel].sum())
        t = np.minimum(np.maximum(self.b - self.z, 0.0), c.mobilization_depth_m * y["severity"])
        vol = int(np.sum(np.rint(t[sel] * self.w6[sel].astype(np.float64) * SCALE).astype(np.int64)))
        start_rad = np.deg2rad(c.start_angle_deg)
        exc = int(np.sum(np.rint(np.maximum(y["slope"][sel] - start_rad, 0.0) * SCALE)
                         .astype(np.int64)))
        overlap = int(np.count_nonzero(self.previous & sel))
        return regions, largest, winner, total, area6, vol, exc, overlap

    def step(self, dt: float, idx=None, target=None) -> PathOracleStep:
        c = self.cfg
        entrained = entrain(self.b, self.z, self.h, idx, target, self.w)
        s = M.step(self.mobile_cfg, self.b, self.h, self.q, dt)
        self.h, self.q = s.h, s.q
        tan_start = float(np.tan(np.deg2rad(c.start_angle_deg)))
        tan_stop = float(np.tan(np.deg2rad(c.stop_angle_deg)))
        y = L.yield_init(self.b, self.z, self.h, self.q[..., 0], self.q[..., 1], dx=c.dx,
                         dy=c.dx, tan_start=tan_start, tan_stop=tan_stop, density=c.density,
                         gravity=c.gravity, cohesion=c.cohesion,
                         mobilization_depth=c.mobilization_depth_m, dry=c.dry_tolerance_m)
        labels = L.canonical_labels(y["unstable"], c.connectivity)
        regions, largest, winner, total, area6, vol, exc, overlap = self._winner_record(y, labels)
        # classification and persistence (gpu_large_avalanche.py:645-676)
        f = c.dx * c.dx / 6.0
        area = area6 * f
        volume = vol / SCALE * f
        mean_start = (exc / SCALE / largest) * (180.0 / np.pi) if largest else 0.0
        candidate = (largest >= c.minimum_connected_cells and area >= c.minimum_connected_area_m2
                     and volume >= c.minimum_mobilizable_volume_m3
                     and mean_start >= c.minimum_mean_excess_start_deg)
        if candidate:
            self.persistence_s = (self.persistence_s + dt if (overlap > 0 or not self.has_previous)
                                  else dt)
        else:
            self.persistence_s = 0.0
        ready = candidate and self.persistence_s >= c.persistence_time_s
        cls = 3 if ready else 2 if candidate else 1 if total > 0 else 0
        self.has_previous = candidate
        sel = labels == winner if winner >= 0 else np.zeros(self.shape, dtype=bool)
        self.previous = sel & candidate
        if cls == 1 and winner >= 0:
            rows, cols = np.nonzero(sel)
            self.reached |= sel
            seeds = (rows // c.tile) * self.tiles_x + cols // c.tile
            self.pending = np.union1d(self.pending, seeds).astype(np.int32)
        # residual gate (v2_physics_core.py:955-1003)
        mobile_volume = self._mobile_volume()
        max_speed = self._max_speed()
        quiet = (mobile_volume <= c.settled_mobile_volume_m3
                 and max_speed <= c.settled_speed_m_s)
        yield_present = total > 0 and volume > c.dry_tolerance_m * c.dx * c.dx
        run = c.residual == "always" or (c.residual == "gated" and quiet and not yield_present)
        rounds = 0
        if run and self.pending.size:
            crit = float(np.tan(np.deg2rad(c.stop_angle_deg)))
            self.b, self.reached, rounds, _ = R.frontier_relax(
                self.b, self.reached, self.pending, tile=c.tile, spacing=(c.dx, c.dx),
                crit_tan=crit, tolerance=c.tolerance_m, weights=self.w,
                max_rounds=c.max_rounds)
            self.pending = np.empty(0, dtype=np.int32)
        return PathOracleStep(s.substeps, entrained, CLASSIFICATIONS[cls], total, regions,
                              largest, winner, area6, vol, exc, bool(run), rounds,
                              mobile_volume, max_speed, labels)
