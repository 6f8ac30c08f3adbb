#!/usr/bin/env python3
"""Generate golden fixtures by running the reference project's own Python code.

Run in a container that has the reference checked out (read-only is fine)::

    REFERENCE_ROOT=/root/reference python tests/golden/make_golden.py

The fixtures (small compressed ``.npz`` files next to this script) hold the
inputs and the reference's outputs, so the GPU tests and the oracle pins never
need the reference at run time.  Cases:

* ``fv_contracts.npz``  -- the ten Mobile V2 contract states of the reference
  tool ``tools/run_mobile_v2_reference_contracts.py`` (:77-177) plus the
  device-equivalence states of ``tools/run_mobile_v2_device_equivalence.py``
  (:36-61) and two rougher seeded states, stepped by
  ``MobileV2ReferenceSolver.step``.
* ``fv_gate.npz``       -- a 64x64 config-0-style terrain stepped 6 x 1/60 s at
  CFL 0.4 (guard bypassed as the reference allows via ``object.__setattr__``).
* ``relax.npz``         -- ``slope_model.relax_critical_slope`` on seeded piles
  and the sparse compact-frontier adapter on the 33x33 disturbance event of
  ``tests/test_warp_gpu_backends.py:166-259``.
* ``labels.npz``        -- ``_largest_connected_region`` and
  ``evaluate_cohesive_yield`` on seeded slope fields.
"""

from __future__ import annotations

import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF = Path(os.environ.get("REFERENCE_ROOT", "/root/reference"))
sys.path[:0] = [str(REF / "src"), str(REF)]
sys.dont_write_bytecode = True

from isaac_bulk_pipeline.experimental import (  # noqa: E402
    MobileV2Config,
    MobileV2ReferenceSolver,
    MobileV2State,
)


def _state(b, h, velocity=None):
    v = (np.zeros(h.shape + (2,)) if velocity is None
         else np.broadcast_to(velocity, h.shape + (2,)).copy())
    return MobileV2State(b, h, h[..., None] * v)


def fv_cases():
    """Input states (name -> (state, dt)) restated from the reference tools."""
    cfg = MobileV2Config()
    shape = (41, 41)
    y, x = np.indices(shape)
    cases = {}
    cases["STATIC_FLAT"] = (_state(np.ones(shape), np.full(shape, 0.1)), 0.05)
    free = 2.0 - np.tan(np.deg2rad(10.0)) * x * cfg.dx_m
    cases["STATIC_SLOPE"] = (_state(free - 0.08, np.full(shape, 0.08)), 0.05)
    H = np.full(shape, 0.8266754619)
    H[:, 19] = 1.82
    H[:, 20] = 0.5144415194
    H[:, 21] = 0.8266754619
    b = np.full(shape, 0.12)
    h = np.maximum(H - b, 0.0)
    v = np.zeros(shape + (2,))
    v[:, 20, 0] = 0.8
    cases["VALLEY"] = (MobileV2State(b, h, h[..., None] * v), 1.0 / 240.0)
    mound = 0.03 + 0.30 * np.exp(-((x - 20) ** 2 + (y - 20) ** 2) / 18.0)
    cases["MOUND"] = (_state(np.full(shape, 0.12), mound), 0.02)
    packet = 0.20 * np.exp(-((x - 13) ** 2 + (y - 20) ** 2) / 30.0)
    pv = np.zeros(shape + (2,))
    pv[..., 0] = 0.8
    cases["SMOOTH_PACKET"] = (_state(1.5 - 0.08 * x * cfg.dx_m, packet, pv), 0.04)
    opp = 0.12 * (np.exp(-((x - 12) ** 2 + (y - 20) ** 2) / 20.0)
                  + np.exp(-((x - 28) ** 2 + (y - 20) ** 2) / 20.0))
    ov = np.zeros(shape + (2,))
    ov[..., 0] = np.where(x < 20, 0.8, -0.8)
    cases["OPPOSING_PACKETS"] = (_state(np.full(shape, 0.12), opp, ov), 0.04)
    wet = np.zeros(shape)
    wet[12:29, 12:29] = 0.12
    wv = np.zeros(shape + (2,))
    wv[..., 0] = 0.5
    cases["WET_DRY"] = (_state(np.full(shape, 0.12), wet, wv), 0.04)
    # Seeded rough states: non-square, sloped support, random momentum.
    rng = np.random.default_rng(20260)
    ys, xs = np.indices((37, 53))
    bb = 0.3 + 0.15 * np.sin(xs / 5.0) * np.cos(ys / 7.0) + 0.02 * rng.random((37, 53))
    hh = np.maximum(0.0, 0.12 * np.exp(-((xs - 30) ** 2 + (ys - 15) ** 2) / 40.0)
                    + 0.01 * rng.random((37, 53)) - 0.004)
    qq = hh[..., None] * rng.normal(0.0, 0.3, (37, 53, 2))
    cases["ROUGH_37x53"] = (MobileV2State(bb, hh, qq), 0.03)
    ys, xs = np.indices((29, 29))
    bb = np.tan(np.deg2rad(25.0)) * xs * 0.05 + 0.05 * rng.random((29, 29))
    hh = np.where((xs > 8) & (xs < 20) & (ys > 8) & (ys < 20), 0.2, 0.0)
    cases["STEEP_BLOCK_29"] = (_state(bb, hh), 1.0 / 60.0)
    return cases


def make_fv_contracts():
    solver = MobileV2ReferenceSolver(MobileV2Config())
    arrays = {}
    names = []
    for name, (state, dt) in fv_cases().items():
        step = solver.step(state, dt)
        names.append(name)
        arrays[f"{name}/b"] = np.asarray(state.b_eff_m)
        arrays[f"{name}/h"] = np.asarray(state.h_m)
        arrays[f"{name}/q"] = np.asarray(state.q_m2_s)
        arrays[f"{name}/dt"] = np.float64(dt)
        arrays[f"{name}/h_out"] = step.state.h_m
        arrays[f"{name}/q_out"] = step.state.q_m2_s
        arrays[f"{name}/substeps"] = np.int64(step.substeps)
        arrays[f"{name}/scalars"] = np.asarray([
            step.maximum_cfl, step.mass_before_m3, step.mass_after_m3,
            step.kinetic_after_j_per_density, step.gravitational_after_j_per_density,
            step.internal_after_j_per_density, step.energy_after_j_per_density,
            step.friction_dissipation_j_per_density, step.minimum_h_m,
        ])
        arrays[f"{name}/impulses"] = np.stack([
            step.momentum_before_m4_s, step.momentum_after_m4_s,
            step.conservative_topography_wall_impulse_m4_s,
            step.friction_impulse_m4_s,
        ])
    arrays["names"] = np.asarray(names)
    np.savez_compressed(HERE / "fv_contracts.npz", **arrays)


def config0_terrain(n: int, seed: int, dx: float = 0.05):
    """Config-0-style inputs: 10 deg x-tilted plane, 8 Gaussian bumps, centre mound."""
    rng = np.random.default_rng(seed)
    ys, xs = np.indices((n, n), dtype=np.float64)
    x = xs * dx
    y = ys * dx
    z = np.tan(np.deg2rad(10.0)) * x
    for _ in range(8):
        amp = rng.uniform(0.05, 0.3)
        sig = rng.uniform(0.2, 1.0)
        cx, cy = rng.uniform(0.0, n * dx, size=2)
        z = z + amp * np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2.0 * sig * sig))
    c = (n - 1) * dx / 2.0
    h = 0.4 * np.exp(-((x - c) ** 2 + (y - c) ** 2) / (2.0 * 1.5 ** 2))
    return z, h


def make_fv_gate():
    cfg = MobileV2Config(basal_friction_coefficient=float(np.tan(np.deg2rad(35.0))))
    object.__setattr__(cfg, "cfl", 0.4)
    solver = MobileV2ReferenceSolver(cfg)
    b, h = config0_terrain(64, seed=0)
    state = MobileV2State(b, h, np.zeros(h.shape + (2,)))
    arrays = {"b": b, "h": h}
    subs = []
    for k in range(6):
        step = solver.step(state, 1.0 / 60.0)
        state = step.state
        subs.append(step.substeps)
        arrays[f"h_{k}"] = state.h_m
        arrays[f"q_{k}"] = state.q_m2_s
    arrays["substeps"] = np.asarray(subs)
    np.savez_compressed(HERE / "fv_gate.npz", **arrays)


def make_report_values():
    """Copy the numbers the reference ships in its own JSON reports."""
    import json
    out = {}
    rep = json.loads((REF / "outputs/mobile_v2_reference/mobile_v2_cpu_contracts.json").read_text())
    for name, case in rep["cases"].items():
        if "substeps" not in case:
            continue
        out[name] = {
            "substeps": case["substeps"],
            "maximum_CFL": case["maximum_CFL"],
            "mass_residual_m3": case["mass_residual_m3"],
            "energy_before": case["energy"]["before_j_per_density"],
            "energy_after": case["energy"]["after_j_per_density"],
            "kinetic_after": case["energy"]["kinetic_after_j_per_density"],
            "friction_dissipation": case["energy"]["friction_dissipation_j_per_density"],
        }
    eq = json.loads((REF / "outputs/mobile_v2_reference/mobile_v2_cpu_device_equivalence.json").read_text())
    device = {k: {"CPU_substeps": v["CPU_substeps"], "DEVICE_substeps": v["DEVICE_substeps"]}
              for k, v in eq["cases"].items()}
    (HERE / "reference_reports.json").write_text(json.dumps(
        {"cpu_contracts": out, "device_equivalence": device}, indent=1, sort_keys=True) + "\n")


if __name__ == "__main__":
    make_report_values()
    make_fv_contracts()
    make_fv_gate()
    if "--fv-only" in sys.argv:
        sys.exit(0)
    make_relax()
    make_labels()
