"""The plain terrain-step path of the production GPU core, on one device.

Order of ``EarthmovingPhysicsCore._step_gpu`` (reference
``runtime/v2_physics_core.py:708-1003``) restricted to the operators of this
library: tool entrainment (the dig phase's resting->mobile activation) ->
``step_mobile`` (Mobile V2, :815) -> ``advance_large_avalanche`` (labelling,
:962) -> residual MiniSlope frontier (:989-1003, :1172-1254), which the
reference runs only while the mobile layer is quiet (mobile volume and speed
below the settled thresholds) and no physically mobilizable yield exists.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _lib

from .avalanche import B200LargeAvalancheBridge, LargeAvalancheTransitionConfig, MaterialScenario
from .bulk_state import B200BulkState, B200ProductionMobileV2Solver
from .mobile_v2 import MobileV2Config, mobile_params
from .relax import FrontierRelaxation

CLASSIFICATIONS = ("NO_LARGE_EVENT", "LOCAL_STATIC_INSTABILITY",
                   "PERSISTING_LARGE_UNSTABLE_REGION", "LARGE_AVALANCHE_MOBILE_PATH")
RESIDUAL_MODES = {"never": 0, "gated": 1, "always": 2}


@dataclass
class PathStepStats:
    substeps: int
    entrained_m3: float
    classification: str
    unstable_cells: int
    regions: int
    largest: int
    residual_rounds: int
    mobile_volume_m3: float
    max_speed_m_s: float


class PlainPath:
    """The plain step on one device.  ``fused=True`` (default) runs the whole
    step as one CUDA graph (``sb_path_step``, one host synchronisation);
    ``fused=False`` calls the operators one by one (same kernels, same results)."""

    def __init__(self, b_eff: np.ndarray, z_base: np.ndarray, *, dx: float,
                 material: MaterialScenario, mobile_config: MobileV2Config | None = None,
                 avalanche_config: LargeAvalancheTransitionConfig | None = None,
                 tile_size: int = 64, precision: str = "fx32", device: int = 0,
                 residual: str = "gated", mobile_headroom_m: float = 1.0,
                 fused: bool = True, tolerance_m: float = 1e-8,
                 max_rounds: int = 4096) -> None:
        self.state = B200BulkState(b_eff.shape, dx, dx, b_eff, z_base_m=z_base, device=device,
                                   tile_size=tile_size, precision=precision,
                                   mobile_headroom_m=mobile_headroom_m)
        self.material = material
        self.mobile = B200ProductionMobileV2Solver(config=mobile_config or MobileV2Config(
            dx_m=dx, dy_m=dx, start_angle_deg=material.start_angle_deg,
            stop_angle_deg=material.stop_angle_deg,
            basal_friction_coefficient=material.mobile_friction_coefficient))
        self.mobile.bind_device_state(self.state, material)
        self.avalanche = B200LargeAvalancheBridge(self.state.grid, material, avalanche_config)
        self.frontier = FrontierRelaxation(self.state.grid, weighted=True)
        if residual not in RESIDUAL_MODES:
            raise ValueError(f"[soilb200] residual must be one of {sorted(RESIDUAL_MODES)}")
        self.residual = residual
        self.critical_slope = float(np.tan(np.deg2rad(material.stop_angle_deg)))
        self.fused = bool(fused)
        self.tolerance_m = float(tolerance_m)
        self.max_rounds = int(max_rounds)
        self.last_stats: _lib.PathStats | None = None
        self._params = self._path_params()
        self._sb_path_step = _lib.load().sb_path_step

    def _path_params(self) -> _lib.PathParams:
        cfg = self.avalanche.config
        relax = _lib.RelaxParams(float(self.frontier.spacing[0]), float(self.frontier.spacing[1]),
                                 self.critical_slope, self.tolerance_m, self.max_rounds, 1)
        return _lib.PathParams(
            mobile_params(self.mobile.config,
                          density_kg_m3=float(self.material.assumed_bulk_density_kg_m3)),
            self.avalanche._params(True), relax, int(cfg.minimum_connected_cells),
            RESIDUAL_MODES[self.residual], float(cfg.minimum_connected_area_m2),
            float(cfg.minimum_mobilizable_volume_m3), float(cfg.minimum_mean_excess_start_deg),
            float(cfg.persistence_time_s), float(cfg.settled_mobile_volume_m3),
            float(cfg.settled_speed_m_s))

    @property
    def grid(self):
        return self.state.grid

    def step(self, dt_s: float, cut_cells=None, cut_targets=None) -> PathStepStats:
        if self.fused:
            return self._step_fused(dt_s, cut_cells, cut_targets)
        return self._step_operators(dt_s, cut_cells, cut_targets)

    def _step_fused(self, dt_s, cut_cells, cut_targets) -> PathStepStats:
        n = 0 if cut_cells is None else int(len(cut_cells))
        idx = tgt = None
        if n:
            idx = np.ascontiguousarray(cut_cells, dtype=np.int32)
            tgt = np.ascontiguousarray(cut_targets, dtype=np.float64)
            if tgt.shape != idx.shape:  # finiteness is checked by sb_path_step
                raise ValueError("[DeviceBulkState] invalid entrainment request")
        st = _lib.PathStats()
        g = self.grid
        _lib.check(g.ctx, self._sb_path_step(
            g.ctx, float(dt_s), idx.ctypes.data if n else None, tgt.ctypes.data if n else None,
            n, self._params, st), "sb_path_step")
        self.last_stats = st
        mob, lab = st.mobile, st.label
        self.mobile.last_stats = mob
        self.state.advance_time(dt_s)
        after = mob.after
        return PathStepStats(int(mob.substeps), float(st.entrained_m3),
                             CLASSIFICATIONS[st.classification], int(lab.unstable_cell_count),
                             int(lab.connected_region_count),
                             int(lab.largest_connected_cell_count),
                             int(st.relax.iterations) if st.residual_ran else 0,
                             float(after.volume_w_m3), float(after.max_speed_m_s))

    def _step_operators(self, dt_s, cut_cells, cut_targets) -> PathStepStats:
        entrained = 0.0
        if cut_cells is not None and len(cut_cells):
            entrained = self.state.entrain_to_surface(cut_cells, cut_targets, reason="bucket_cut")
        mob = self.mobile.step_resident(dt_s)
        self.state.advance_time(dt_s)
        diag = self.avalanche.observe(dt_s)
        cfg = self.avalanche.config
        rounds = 0
        quiet = (mob.volume_after_m3 <= cfg.settled_mobile_volume_m3
                 and mob.maximum_speed_m_s <= cfg.settled_speed_m_s)
        yield_present = (diag.unstable_cell_count > 0
                         and diag.largest_connected_mobilizable_volume_m3
                         > cfg.dry_tolerance_m * self.grid.dx * self.grid.dy)
        run = self.residual == "always" or (self.residual == "gated" and quiet and not yield_present)
        if run:
            rounds = self.frontier.run(self.critical_slope, self.tolerance_m, self.max_rounds).rounds
        return PathStepStats(int(mob.substeps), entrained, diag.classification,
                             diag.unstable_cell_count, diag.connected_region_count,
                             diag.largest_connected_cell_count, rounds,
                             float(mob.volume_after_m3), float(mob.maximum_speed_m_s))

    def settle(self, relaxation, tolerance_m: float, schedule=None,
               max_iterations: int = 400000):
        """Relaxes this path's resting surface (the resident b_eff) to repose
        in place, after the cuts: ``relaxation`` is a
        ``learned.LearnedRelaxation`` bound to this path's grid; ``schedule``
        its proposal schedule (``learned.SCHEDULE`` by default,
        ``learned.PLAIN`` for the plain relax_critical_slope sweep alone,
        reference ``slope_model.py:273-343``).  Either way the plain sweep
        finishes until every face slope is at most tan(angle) + tolerance, and
        the volume ledger stays exact (whole quanta).  Returns the RelaxStats
        of the finishing sweeps, ``iterations`` counting every sweep."""
        if relaxation.grid is not self.grid:
            raise ValueError("[soilb200] settle needs a relaxation bound to this path's grid")
        return relaxation.relax_scheduled(tolerance_m, schedule, max_iterations=max_iterations)

    STAGES = ("start", "entrainment", "before_ledger", "substeps_and_yield_tiles", "border_merge",
              "compression", "reduction_classification", "previous_and_seeds", "residual_frontier")

    def stage_times(self) -> dict:
        """Device ms per stage of the last fused step (needs the context created
        with SOILB200_STAGE_EVENTS=1; empty otherwise).  While the cut command
        buffer holds at most 4096 cells, one kernel starts the step and
        entrains the cut: "start" then holds both and "entrainment" only the
        stage marker."""
        import numpy as _np
        out = _np.zeros(16, dtype=_np.float32)
        n = int(_lib.load().sb_path_stage_times(self.grid.ctx, out.ctypes.data, out.size))
        return {name: float(out[k]) for k, name in enumerate(self.STAGES[:max(n, 0)])}

    def close(self) -> None:
        self.state.close()
