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

from .avalanche import B200LargeAvalancheBridge, LargeAvalancheTransitionConfig, MaterialScenario
from .bulk_state import B200BulkState, B200ProductionMobileV2Solver
from .mobile_v2 import MobileV2Config
from .relax import FrontierRelaxation


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
    def __init__(self, b_eff: np.ndarray, z_base: np.ndarray, *, dx: float,
                 material: MaterialScenario, mobile_config: MobileV2Config | None = None,
                 avalanche_config: LargeAvalancheTransitionConfig | None = None,
                 tile_size: int = 64, precision: str = "fx32", device: int = 0,
                 residual: str = "gated", mobile_headroom_m: float = 1.0) -> None:
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
        self.residual = residual
        self.critical_slope = float(np.tan(np.deg2rad(material.stop_angle_deg)))

    @property
    def grid(self):
        return self.state.grid

    def step(self, dt_s: float, cut_cells=None, cut_targets=None) -> PathStepStats:
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
            rounds = self.frontier.run(self.critical_slope, 1e-8).rounds
        return PathStepStats(int(mob.substeps), entrained, diag.classification,
                             diag.unstable_cell_count, diag.connected_region_count,
                             diag.largest_connected_cell_count, rounds,
                             float(mob.volume_after_m3), float(mob.maximum_speed_m_s))

    def close(self) -> None:
        self.state.close()
