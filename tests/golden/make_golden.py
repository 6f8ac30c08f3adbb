#!/usr/bin/env python3
"""Generate golden fixtures by running the reference project's own Python code.

Run in a container that has the reference checked out (read-only is fine)::

    REFERENCE_ROOT=<path of the reference checkout> python tests/golden/make_golden.py

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
* ``deposition.npz``    -- the CPU ``DepositionOperator.apply``
  (bulk_interaction/deposition.py:67-160) on the three scenarios of the
  reference's device-deposition tests (tests/test_device_bulk_state.py:150-230)
  and a seeded static blanket below the stop angle.
* ``reference_checkpoint.npz`` -- an archive written by the reference's
  ``write_device_checkpoint`` from a stub core (``--checkpoint``).
* ``avalanche.npz``     -- ``LargeAvalancheTransitionController.observe_and_maybe_mobilize``
  (the CPU resting->mobile activation) called repeatedly on a pile and on a
  45 deg plane (``--avalanche``).
* ``event.npz``         -- ``EventDrivenMinimumSlopeAdapter.solve`` (the
  reached-bbox MiniSlope backend) on the reference's three acceptance
  scenarios and two seeded events (``--event``).
* ``fractal.npz``       -- ``slope_model.fractal_perlin_noise`` (the
  generator of the config-3 training patches) on four seeds/parameter sets
  (``--fractal``).
* ``surface.npz``       -- ``AirborneParcelModel._bilinear``
  (bulk_exchange/airborne.py:587-600), the reference's CPU bilinear sample of
  the free surface (resting + mobile), on seeded fields at in-range queries
  (grid points, cell interiors, the last row and column) (``--surface``); the
  Warp query kernel (runtime/bulk_state_authority.py:201-228) is the same
  formula with the queries clamped to the grid first.
* ``gate0.npz``         -- the 5 s config-0 gate: 256x256, seed 0, 300 steps of
  1/60 s at CFL 0.4 and mu = tan 35 deg, each followed by
  ``relax_critical_slope`` of ``b_eff`` at 35 deg (row-major array, spacing
  (dy, dx), tolerance 1e-8 m); final fields stored as float32 (the comparison
  bound is 1e-5 m), per-step substeps and relaxation iterations as integers.
"""

from __future__ import annotations

import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
if not os.environ.get("REFERENCE_ROOT"):
    raise SystemExit("set REFERENCE_ROOT to the reference project's checkout")
REF = Path(os.environ["REFERENCE_ROOT"])
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


def make_relax():
    """relax_critical_slope cases and compact-frontier events (CPU adapter)."""
    import slope_model as sm
    from isaac_bulk_pipeline.config import SolverConfig
    from isaac_bulk_pipeline.solvers import SparseTileFrontierMinimumSlopeAdapter
    from isaac_bulk_pipeline.terrain import TerrainGrid

    arrays = {}
    full = []
    # full-domain relax_critical_slope (H[axis0, axis1], spacing per axis)
    pile = sm.random_pile(40, 48, 0.05, 0.05, seed=5, peak_height=0.6)
    full.append(("PILE_40x48", pile, (0.05, 0.05), 34.0))
    ys, xs = np.indices((30, 25))
    cone = np.maximum(0.0, 0.9 - 0.09 * np.hypot(xs - 12.0, ys - 15.0))
    full.append(("CONE_30x25_ANISO", cone, (0.05, 0.08), 30.0))
    noise = 0.25 * (sm.fractal_perlin_noise(32, 32, seed=11) + 1.0)
    full.append(("NOISE_32", noise, (0.05, 0.05), 35.0))
    for name, h, spacing, angle in full:
        out, stats = sm.relax_critical_slope(h, spacing, critical_angle_deg=angle,
                                             max_iterations=20000, tolerance=1e-8)
        arrays[f"full/{name}/h"] = h
        arrays[f"full/{name}/spacing"] = np.asarray(spacing)
        arrays[f"full/{name}/angle"] = np.float64(angle)
        arrays[f"full/{name}/out"] = out
        arrays[f"full/{name}/iterations"] = np.int64(stats.iterations)
    arrays["full_names"] = np.asarray([n for n, *_ in full])

    events = []
    base = np.ones((33, 33))
    dist = base.copy()
    dist[16, 16] += 0.30
    seeds = np.zeros((33, 33), dtype=bool)
    seeds[16, 16] = True
    events.append(("DISTURB_33", base, dist, seeds, 8, 30.0))
    rng = np.random.default_rng(77)
    ys, xs = np.indices((40, 56))
    base2 = 0.5 + 0.2 * np.tan(np.deg2rad(20.0)) * xs * 0.05 + 0.002 * rng.random((40, 56))
    dist2 = base2.copy()
    seeds2 = np.zeros((40, 56), dtype=bool)
    for (r, c, a) in ((10, 12, 0.25), (30, 40, 0.35), (22, 27, -0.2)):
        dist2[r - 1:r + 2, c - 1:c + 2] += a
        seeds2[r - 1:r + 2, c - 1:c + 2] = True
    events.append(("MULTI_40x56", base2, dist2, seeds2, 8, 32.0))
    for name, b0, d, sd, tile, angle in events:
        ny, nx = d.shape
        grid = TerrainGrid(nx, ny, 0.05, 0.05, 0.0, 0.0, "/World/Terrain")
        cfg = SolverConfig(critical_angle_deg=angle, max_iterations=2000,
                           large_avalanche_iteration_threshold=1000,
                           numerical_safety_max_iterations=2000, tolerance=1.0e-8,
                           boundary_condition="closed", conservation_tolerance_m3=1.0e-7)
        cpu = SparseTileFrontierMinimumSlopeAdapter(grid, cfg, tile_size=tile)
        cpu.set_reference_height(b0)
        cpu.mark_changed(sd)
        res = cpu.solve(d)
        arrays[f"event/{name}/h"] = d
        arrays[f"event/{name}/seeds"] = sd
        arrays[f"event/{name}/tile"] = np.int64(tile)
        arrays[f"event/{name}/angle"] = np.float64(angle)
        arrays[f"event/{name}/out"] = res.heightmap_stable
        arrays[f"event/{name}/iterations"] = np.int64(res.iteration_count)
    arrays["event_names"] = np.asarray([n for n, *_ in events])
    np.savez_compressed(HERE / "relax.npz", **arrays)


def make_labels():
    """Connected-component and yield fixtures from the CPU avalanche detector."""
    from isaac_bulk_pipeline.bulk_interaction.large_avalanche import _largest_connected_region
    from isaac_bulk_pipeline.bulk_interaction.yield_criterion import evaluate_cohesive_yield
    from isaac_bulk_pipeline.bulk_state import MaterialScenario, TerrainVolumeIntegrator
    from isaac_bulk_pipeline.terrain import TerrainGrid

    arrays = {}
    names = []
    rng = np.random.default_rng(2024)
    masks = {
        "RANDOM_60x70_p045": rng.random((60, 70)) < 0.45,
        "RANDOM_64x64_p060": rng.random((64, 64)) < 0.60,
        "STRIPES_50x33": (np.indices((50, 33))[1] % 3) == 0,
        "CHECKER_31x31": (np.indices((31, 31)).sum(axis=0) % 2) == 0,
        "EMPTY_8x9": np.zeros((8, 9), dtype=bool),
        "FULL_9x8": np.ones((9, 8), dtype=bool),
    }
    for name, mask in masks.items():
        for conn in (4, 8):
            largest, count, size = _largest_connected_region(mask, conn)
            key = f"{name}/c{conn}"
            names.append(key)
            arrays[f"{key}/mask"] = mask
            arrays[f"{key}/largest"] = largest
            arrays[f"{key}/regions"] = np.int64(count)
            arrays[f"{key}/largest_size"] = np.int64(size)
    arrays["mask_names"] = np.asarray(names)
    # cohesive yield on a seeded noise pile (start 38, stop 30, cohesion 0)
    import slope_model as sm
    ny, nx = 48, 52
    grid = TerrainGrid(nx, ny, 0.05, 0.05, 0.0, 0.0, "/World/Terrain")
    integ = TerrainVolumeIntegrator.from_grid(grid)
    resting = 0.2 + 0.3 * (sm.fractal_perlin_noise(ny, nx, seed=3) + 1.0)
    mobile = np.zeros((ny, nx))
    material = MaterialScenario("golden", 1370.0, 29.8, 0.0, 0.5, 38.0, 30.0, 0.35)
    depth = np.minimum(resting, 0.08)
    ys = evaluate_cohesive_yield(resting, mobile, material, grid, integ, layer_depth_m=depth)
    arrays["yield/resting"] = resting
    arrays["yield/start_mask"] = ys.start_mask
    arrays["yield/slope_rad"] = ys.slope_rad
    arrays["yield/stop_margin"] = ys.yield_stop_margin_pa
    largest, count, size = _largest_connected_region(ys.start_mask, 8)
    arrays["yield/largest"] = largest
    arrays["yield/regions"] = np.int64(count)
    arrays["yield/largest_size"] = np.int64(size)
    np.savez_compressed(HERE / "labels.npz", **arrays)


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


def make_deposition():
    from isaac_bulk_pipeline.bulk_interaction import DepositionOperator
    from isaac_bulk_pipeline.bulk_state import MaterialScenario, TerrainVolumeIntegrator
    from isaac_bulk_pipeline.terrain import TerrainGrid

    material = MaterialScenario("device_state", 1370.0, 29.8, 800.0, 0.5, 38.0, 30.0, 0.35)
    arrays = {}
    cases = []
    grid16 = TerrainGrid(16, 16, 0.05, 0.05, 0.0, 0.0, "/World/Terrain")
    resting = np.ones(grid16.shape)
    mobile = np.zeros(grid16.shape)
    mobile[6:10, 6:10] = 0.03
    cases.append(("PATCH", grid16, resting, mobile, np.zeros(grid16.shape + (2,))))
    cols = np.arange(grid16.nx, dtype=np.float64)[None, :]
    resting = np.repeat(0.08 * cols, grid16.ny, axis=0)
    cases.append(("BLANKET", grid16, resting, np.max(resting) - resting + 0.02,
                  np.zeros(grid16.shape + (2,))))
    resting = np.zeros(grid16.shape)
    resting[8, 8] = 0.20
    mobile = np.zeros(grid16.shape)
    mobile[8, 9] = 0.01
    mom = np.zeros(grid16.shape + (2,))
    mom[8, 9, 0] = 0.02
    cases.append(("TAIL", grid16, resting, mobile, mom))
    grid = TerrainGrid(40, 32, 0.05, 0.05, 0.0, 0.0, "/World/Terrain")
    rng = np.random.default_rng(21)
    ys, xs = np.indices(grid.shape)
    resting = 0.5 + 0.02 * np.sin(xs / 3.0) + 0.02 * np.cos(ys / 4.0)
    mobile = np.where(rng.random(grid.shape) < 0.6, 0.004 + 0.03 * rng.random(grid.shape), 0.0)
    cases.append(("STATIC_NOISE", grid, resting, mobile, np.zeros(grid.shape + (2,))))
    names = []
    for name, g, rest, mob, q in cases:
        integ = TerrainVolumeIntegrator.from_grid(g)
        res = DepositionOperator().apply(rest, mob, q, material, g, integ, 1.0 / 60.0)
        names.append(name)
        arrays[f"{name}/resting"] = rest
        arrays[f"{name}/mobile"] = mob
        arrays[f"{name}/momentum"] = q
        arrays[f"{name}/resting_out"] = res.H_resting_m
        arrays[f"{name}/mobile_out"] = res.mobile_height_m
        arrays[f"{name}/volume"] = np.float64(res.deposited_volume_m3)
        arrays[f"{name}/tail"] = np.int32(integ.integrate(mob) <= g.dx * g.dy * min(g.dx, g.dy))
    arrays["names"] = np.asarray(names)
    arrays["material"] = np.asarray([1370.0, 29.8, 800.0, 0.5, 38.0, 30.0, 0.35])
    np.savez_compressed(HERE / "deposition.npz", **arrays)


def make_gate0(n: int = 256, steps: int = 300):
    import time

    import slope_model as sm

    cfg = MobileV2Config(basal_friction_coefficient=float(np.tan(np.deg2rad(35.0))))
    object.__setattr__(cfg, "cfl", 0.4)
    solver = MobileV2ReferenceSolver(cfg)
    b, h = config0_terrain(n, seed=0)
    state = MobileV2State(b, h, np.zeros(h.shape + (2,)))
    subs, iters = [], []
    t0 = time.time()
    for k in range(steps):
        step = solver.step(state, 1.0 / 60.0)
        subs.append(step.substeps)
        relaxed, rs = sm.relax_critical_slope(step.state.b_eff_m, (cfg.dy_m, cfg.dx_m),
                                              critical_angle_deg=35.0, max_iterations=20000,
                                              tolerance=1e-8)
        iters.append(rs.iterations)
        state = MobileV2State(relaxed, step.state.h_m, step.state.q_m2_s)
        if k in (59, 299):
            print(f"gate0 step {k + 1}: {time.time() - t0:.1f} s", flush=True)
    np.savez_compressed(HERE / "gate0.npz", b0_sum=np.float64(b.sum()), h0_sum=np.float64(h.sum()),
                        b_final=state.b_eff_m.astype(np.float32),
                        h_final=state.h_m.astype(np.float32),
                        substeps=np.asarray(subs, np.int32), relax_iterations=np.asarray(iters, np.int32),
                        mass_final=np.float64(np.sum(state.h_m) * cfg.dx_m * cfg.dy_m),
                        resting_final=np.float64(np.sum(state.b_eff_m) * cfg.dx_m * cfg.dy_m))


def make_fractal():
    """slope_model.fractal_perlin_noise, the reference's training-patch noise
    (slope_model.py:77-129): default parameters at 128^2 for seeds 0 and
    19999, a non-square field and non-default parameters."""
    import slope_model as S
    cases = [((128, 128, 0), {}), ((128, 128, 19999), {}), ((64, 96, 5), {}),
             ((50, 70, 3), {"base_cells": 4, "octaves": 3, "persistence": 0.4,
                            "lacunarity": 2.5})]
    arrays = {"count": np.int64(len(cases))}
    for k, (args, kw) in enumerate(cases):
        arrays[f"{k}/args"] = np.asarray(args, np.int64)
        arrays[f"{k}/kw"] = np.asarray([kw.get("base_cells", 3), kw.get("octaves", 5)], np.int64)
        arrays[f"{k}/kwf"] = np.asarray([kw.get("persistence", 0.52), kw.get("lacunarity", 2.0)])
        arrays[f"{k}/noise"] = S.fractal_perlin_noise(*args, **kw)
    np.savez_compressed(HERE / "fractal.npz", **arrays)


def make_surface():
    """Bilinear surface samples from the reference's CPU sampler
    (bulk_exchange/airborne.py:587-600) on resting + mobile fields."""
    from isaac_bulk_pipeline.bulk_exchange.airborne import AirborneParcelModel
    rng = np.random.default_rng(11)
    ny, nx = 37, 53
    resting = 0.4 + 0.3 * rng.random((ny, nx))
    mobile = np.where(rng.random((ny, nx)) < 0.3, 0.05 * rng.random((ny, nx)), 0.0)
    field = resting + mobile
    q = np.concatenate([
        np.column_stack([rng.uniform(0.0, ny - 1.0, 400), rng.uniform(0.0, nx - 1.0, 400)]),
        np.column_stack([rng.integers(0, ny, 40), rng.integers(0, nx, 40)]).astype(np.float64),
        np.asarray([[ny - 1.0, nx - 1.0], [0.0, 0.0], [ny - 1.0, 0.5], [3.25, nx - 1.0]]),
    ])
    values = np.asarray([AirborneParcelModel._bilinear(field, r, c) for r, c in q])
    np.savez_compressed(HERE / "surface.npz", resting=resting, mobile=mobile, queries=q,
                        values=values)


def make_event():
    """solvers.EventDrivenMinimumSlopeAdapter (solvers/event_driven_slope.py:
    16-302), the reached-bbox MiniSlope backend: the three scenarios of the
    reference's tests/test_minislope_dynamic_frontier_acceptance.py (single
    bump, toe excavation of a near-critical plane, whole-pile stress with the
    avalanche threshold below the iteration count) plus two seeded events on
    non-square grids (one with dx != dy), closed boundary, tile size 8."""
    from isaac_bulk_pipeline.config import SolverConfig
    from isaac_bulk_pipeline.solvers import EventDrivenMinimumSlopeAdapter
    from isaac_bulk_pipeline.terrain import TerrainGrid

    def config(angle=30.0, max_iterations=5000):
        return SolverConfig(critical_angle_deg=angle, max_iterations=max_iterations,
                            large_avalanche_iteration_threshold=max_iterations,
                            numerical_safety_max_iterations=max(10_000, max_iterations),
                            tolerance=1.0e-8, boundary_condition="closed",
                            conservation_tolerance_m3=1.0e-7)

    def plane(shape, dx, fraction):
        drop = np.tan(np.deg2rad(30.0)) * dx
        prof = 1.0 + np.arange(shape[1], dtype=np.float64) * (fraction * drop)
        return np.repeat(prof[None, :], shape[0], axis=0)

    cases = []
    base = np.ones((96, 96))
    dist = base.copy()
    dist[47, 53] += 0.30
    cases.append(("bump96", (96, 96, 0.05, 0.05), base, dist, config()))
    base = plane((65, 65), 0.05, 0.99)
    dist = base.copy()
    dist[28:37, 0] -= 0.10
    cases.append(("toe65", (65, 65, 0.05, 0.05), base, dist, config()))
    base = plane((33, 33), 0.05, 1.0)
    dist = base.copy()
    dist[:, 0] -= 0.10
    cases.append(("stress33", (33, 33, 0.05, 0.05), base, dist, config(max_iterations=100)))
    for name, (ny, nx), (dx, dy), seed in (("seeded70x90", (70, 90), (0.05, 0.05), 4),
                                           ("seeded41x57_aniso", (41, 57), (0.05, 0.04), 9)):
        rng = np.random.default_rng(seed)
        base = 0.5 + 0.2 * rng.random((ny, nx)) * 0.01
        dist = base.copy()
        for _ in range(3):
            r, c = rng.integers(3, ny - 4), rng.integers(3, nx - 4)
            dist[r - 2:r + 3, c - 2:c + 3] += rng.uniform(0.15, 0.35)
        cases.append((name, (nx, ny, dx, dy), base, dist, config(angle=33.0)))
    arrays = {"names": np.asarray([c[0] for c in cases])}
    for name, (nx, ny, dx, dy), base, dist, cfg in cases:
        grid = TerrainGrid(nx, ny, dx, dy, 0.0, 0.0, "/World/Terrain")
        solver = EventDrivenMinimumSlopeAdapter(grid, cfg, tile_size=8)
        solver.set_reference_height(base)
        res = solver.solve(dist)
        arrays[f"{name}/grid"] = np.asarray([nx, ny, dx, dy], np.float64)
        arrays[f"{name}/angle"] = np.float64(cfg.critical_angle_deg)
        arrays[f"{name}/threshold"] = np.int64(cfg.large_avalanche_iteration_threshold)
        arrays[f"{name}/base"] = base
        arrays[f"{name}/initial"] = dist
        arrays[f"{name}/stable"] = np.asarray(res.heightmap_stable)
        arrays[f"{name}/iterations"] = np.int64(res.iteration_count)
        arrays[f"{name}/classification"] = np.asarray(
            res.diagnostics["avalanche_classification"])
        arrays[f"{name}/propagation_bbox"] = np.asarray(
            res.diagnostics["propagation_bbox_yx"], np.int64)
        print(name, res.iteration_count, res.diagnostics["avalanche_classification"],
              res.diagnostics["propagation_bbox_yx"], flush=True)
    np.savez_compressed(HERE / "event.npz", **arrays)


def make_avalanche():
    """LargeAvalancheTransitionController.observe_and_maybe_mobilize
    (bulk_interaction/large_avalanche.py:289-422), the reference's CPU
    resting->mobile activation, called repeatedly (no transport in between)
    on a cohesionless pile and on the 45 deg plane of the reference's
    tests/test_large_avalanche_transition.py; z_base = 0, so its resting
    thickness is b_eff.  Per call: transition flag, transferred volume,
    persistence, unstable / largest counts and the fields after the call."""
    from isaac_bulk_pipeline.bulk_interaction import (LargeAvalancheTransitionConfig,
                                                      LargeAvalancheTransitionController)
    from isaac_bulk_pipeline.bulk_state import MaterialScenario, TerrainVolumeIntegrator
    from isaac_bulk_pipeline.terrain import TerrainGrid

    mat = MaterialScenario(name="golden_pile", assumed_bulk_density_kg_m3=1600.0,
                           internal_friction_angle_deg=35.0, cohesion_proxy_pa=0.0,
                           tool_friction_coefficient=0.5, start_angle_deg=38.0,
                           stop_angle_deg=30.0, mobile_friction_coefficient=0.55)
    n = 64
    ys, xs = np.indices((n, n), dtype=np.float64)
    pile = np.maximum(0.0, 1.6 - 1.1 * np.hypot(xs - n / 2, ys - n / 2) * 0.05) \
        + 0.02 * (1.0 + np.sin(xs / 3.0))
    plane = np.repeat((2.0 - np.tan(np.deg2rad(45.0)) * np.arange(21) * 0.05)[None, :], 21, axis=0)
    cases = [("pile64", pile, 12), ("plane21", plane, 10)]
    arrays = {"names": np.asarray([c[0] for c in cases]), "dt": np.float64(1.0 / 60.0)}
    for name, resting, calls in cases:
        ny, nx = resting.shape
        grid = TerrainGrid(nx, ny, 0.05, 0.05, 0.0, 0.0, "/World/Terrain")
        integ = TerrainVolumeIntegrator.from_grid(grid)
        ctrl = LargeAvalancheTransitionController(LargeAvalancheTransitionConfig())
        mobile = np.zeros_like(resting)
        momentum = np.zeros(resting.shape + (2,))
        arrays[f"{name}/resting0"] = resting.copy()
        rec = []
        for k in range(calls):
            res = ctrl.observe_and_maybe_mobilize(resting, mobile, momentum, mat, grid, integ,
                                                  1.0 / 60.0)
            d = res.diagnostics
            resting = np.asarray(res.H_resting_m).copy()
            mobile = np.asarray(res.mobile_height_m).copy()
            momentum = np.asarray(res.mobile_momentum_m2_s).copy()
            rec.append([float(res.transitioned), res.transferred_volume_m3, ctrl.persistence_s,
                        float(d.unstable_cell_count), float(d.largest_connected_cell_count)])
            arrays[f"{name}/resting_{k}"] = resting
            arrays[f"{name}/mobile_{k}"] = mobile
        arrays[f"{name}/record"] = np.asarray(rec)
        print(name, [(int(r[0]), round(r[1], 6), round(r[2], 4), int(r[3]), int(r[4])) for r in rec])
    np.savez_compressed(HERE / "avalanche.npz", **arrays)


def make_checkpoint():
    """An archive written by the reference's own write_device_checkpoint
    (runtime/device_checkpoint.py:65-124).  The writer only reads named
    attributes of the physics core, so a stub core stands in for the GPU
    runtime: a 24 x 32 grid whose every field holds distinct seeded values,
    large-avalanche persistence, frontier tiles and dirty tiles."""
    from types import SimpleNamespace

    from isaac_bulk_pipeline.runtime import device_checkpoint as D

    ny, nx = 24, 32
    rng = np.random.default_rng(17)
    fields = {}
    for name in D.FLOAT_FIELDS:
        fields[name] = rng.random((ny, nx))
    fields["z_base"] = 0.1 * rng.random((ny, nx))
    fields["b_eff"] = fields["z_base"] + 0.5 + rng.random((ny, nx))
    fields["mobile"] = np.where(rng.random((ny, nx)) < 0.3, 0.05 * rng.random((ny, nx)), 0.0)
    for name in D.INT_FIELDS:
        fields[name] = rng.integers(0, 2, (ny, nx)).astype(np.int32)
    fields["avalanche_activation_count"] = rng.integers(0, 4, (ny, nx)).astype(np.int32)

    runtime = SimpleNamespace(download=lambda name: fields[name].ravel().copy())
    state = SimpleNamespace(runtime=runtime, shape=(ny, nx),
                            authority=SimpleNamespace(value="DEVICE"),
                            timestamp_device_s=12.25, _dirty_tile_ids={3, 1})
    chain = SimpleNamespace(large_avalanche=SimpleNamespace(_persistence_s=0.0833,
                                                            _has_previous=True))
    metadata = SimpleNamespace(checkpoint_record=lambda: {"source": "golden_stub"})
    core = SimpleNamespace(runtime_backend="GPU_RUNTIME", device_state=state, gpu_chain=chain,
                           gpu_metadata=metadata, grid=SimpleNamespace(dx=0.05, dy=0.05),
                           _gpu_frontier_active_tiles=np.asarray([0, 2], np.int32),
                           _gpu_frontier_iterations=7, _static_relaxation_pending=False)
    out = D.write_device_checkpoint(core, HERE / "reference_checkpoint.npz",
                                    provenance={"writer": "reference write_device_checkpoint"})
    print("checkpoint", out["terrain_hash_sha256"], out["checkpoint_hash_sha256"])


if __name__ == "__main__":
    if "--checkpoint" in sys.argv:
        make_checkpoint()
        sys.exit(0)
    if "--avalanche" in sys.argv:
        make_avalanche()
        sys.exit(0)
    if "--event" in sys.argv:
        make_event()
        sys.exit(0)
    if "--surface" in sys.argv:
        make_surface()
        sys.exit(0)
    if "--fractal" in sys.argv:
        make_fractal()
        sys.exit(0)
    if "--gate0" in sys.argv:
        make_gate0()
        sys.exit(0)
    if "--deposition" in sys.argv:
        make_deposition()
        sys.exit(0)
    make_report_values()
    make_fv_contracts()
    make_fv_gate()
    if "--fv-only" in sys.argv:
        sys.exit(0)
    make_relax()
    make_labels()
