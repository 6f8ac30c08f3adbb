"""Parity of the headline workload: the config-1 plain path at 701^2.

The bench's default line measures this exact step sequence (seeded value-noise
pile, seed 1; the straight bucket cut; 1/60 s physics steps; cut entrainment
-> Mobile V2 -> labelling -> gated residual frontier, one CUDA graph per step).
Here it runs for 60 steps through ``PlainPath`` and is compared with the CPU
oracle of the whole step (``oracle.path``, restating
runtime/v2_physics_core.py:708-1003 with the gate of :955-1003):

* FP64 (the reference's arithmetic): fields bit-identical after every checked
  step, substep counts equal every step, canonical labels bit-identical,
  region count / largest component / winner / classification / residual
  decision equal every step, the winner's integer area exact and its
  fixed-point slope excess within one 2^-32 rad unit per cell (``arctan`` of
  CUDA and of the C library may differ in the last bit).
* FX32 (production: int32 height quanta + float32 momentum): labels bit-exact
  against the oracle's fixed-point yield + labelling evaluated on the GPU's
  own FX32 fields; max |h_fx32 - h_fp64| <= 1e-5 m and max |b_fx32 - b_fp64|
  <= 1e-5 m over the run; total material volume (resting + mobile quanta,
  Triangle-A-C weights) exactly conserved.
"""

import numpy as np
import pytest

import soilb200
from oracle import fixed_point as fx
from oracle import labels as L
from oracle import relax as R
from oracle.path import PathOracle, PathOracleConfig
from soilb200 import workloads
from soilb200.pipeline import PlainPath

pytestmark = pytest.mark.gpu

N = 701
DX = 0.05
DT = 1.0 / 60.0
STEPS = 60
CHECK_EVERY = 10
FX32_BOUND_M = 1.0e-5


def _material():
    # the bench's material (density 1600, start 38 deg, stop 30 deg, mu 0.55)
    return soilb200.MaterialScenario("config1_soil", 1600.0, 35.0, 0.0, 0.5, 38.0, 30.0, 0.55)


def _oracle_cfg(mat, **kw):
    return PathOracleConfig(dx=DX, density=mat.assumed_bulk_density_kg_m3,
                            cohesion=mat.cohesion_proxy_pa, start_angle_deg=mat.start_angle_deg,
                            stop_angle_deg=mat.stop_angle_deg,
                            mobile_friction=mat.mobile_friction_coefficient, **kw)


def _fields(path):
    g = path.grid
    return {k: g.download(k) for k in ("b_eff", "mobile", "momentum_x", "momentum_y")}


def _steep_cells(b, angle_deg):
    """Cells with a neighbour slope above the angle (axis-aligned pairs)."""
    crit = np.tan(np.deg2rad(angle_deg)) * DX
    m = np.zeros(b.shape, dtype=bool)
    d0 = np.abs(np.diff(b, axis=0)) > crit
    d1 = np.abs(np.diff(b, axis=1)) > crit
    m[:-1] |= d0
    m[1:] |= d0
    m[:, :-1] |= d1
    m[:, 1:] |= d1
    return m


def _compare_step(k, g, o):
    assert g.substeps == o.substeps, k
    assert g.classification == o.classification, k
    assert (g.unstable_cells, g.regions, g.largest) == (o.unstable_cells, o.regions, o.largest), k
    assert g.residual_rounds == o.residual_rounds, k


@pytest.fixture(scope="module")
def headline_runs():
    """Both precisions over the same 60-step schedule, FP64 checked against
    the oracle step by step; returns what the FX32 checks need."""
    cfg = workloads.config1(N, seed=1, dx=DX)
    mat = _material()
    sched = [cfg["cut"].footprint((k + 1) * DT) for k in range(STEPS)]
    fp64 = PlainPath(cfg["b_eff"], cfg["z_base"], dx=DX, material=mat, precision="fp64",
                     residual="gated")
    oracle = PathOracle(cfg["b_eff"], cfg["z_base"], _oracle_cfg(mat))
    fp64_fields = []
    for k, (idx, tgt) in enumerate(sched):
        g = fp64.step(DT, idx, tgt)
        o = oracle.step(DT, idx, tgt)
        _compare_step(k, g, o)
        lo = fp64.last_stats.label
        assert lo.winner_root == o.winner, k
        assert g.entrained_m3 == pytest.approx(o.entrained_m3, rel=1e-12, abs=1e-18), k
        if k % CHECK_EVERY == CHECK_EVERY - 1:
            f = _fields(fp64)
            assert np.array_equal(f["b_eff"], oracle.b), k
            assert np.array_equal(f["mobile"], oracle.h), k
            assert np.array_equal(f["momentum_x"], oracle.q[..., 0]), k
            assert np.array_equal(f["momentum_y"], oracle.q[..., 1]), k
            assert np.array_equal(fp64.avalanche.labels(), o.labels), k
            fp64_fields.append(f)
    fp64.close()
    yield cfg, mat, sched, fp64_fields


def test_fp64_headline_path_matches_oracle(headline_runs):
    """The fixture asserts the FP64 parity step by step; this test reports it."""
    _, _, _, fp64_fields = headline_runs
    assert len(fp64_fields) == STEPS // CHECK_EVERY
    # the cut really moved material into the mobile layer
    assert fp64_fields[-1]["mobile"].max() > 0.01


def test_fx32_headline_path_labels_bound_and_volume(headline_runs):
    cfg, mat, sched, fp64_fields = headline_runs
    path = PlainPath(cfg["b_eff"], cfg["z_base"], dx=DX, material=mat, precision="fx32",
                     residual="gated")
    grid = path.grid
    k_exp, datum, q = grid.height_exponent, grid.datum, grid.quantum
    r0 = path.state.reservoir_reduction(mat.assumed_bulk_density_kg_m3)
    total0 = r0["resting_quanta_w6"] + r0["mobile_quanta_w6"]
    worst_h = worst_b = 0.0
    for k, (idx, tgt) in enumerate(sched):
        st = path.step(DT, idx, tgt)
        r = path.state.reservoir_reduction(mat.assumed_bulk_density_kg_m3)
        assert r["resting_quanta_w6"] + r["mobile_quanta_w6"] == total0, k
        if k % CHECK_EVERY != CHECK_EVERY - 1:
            continue
        f = _fields(path)
        ref = fp64_fields[k // CHECK_EVERY]
        worst_h = max(worst_h, float(np.abs(f["mobile"] - ref["mobile"]).max()))
        worst_b = max(worst_b, float(np.abs(f["b_eff"] - ref["b_eff"]).max()))
        assert st.residual_rounds == 0  # labels were taken on these same fields
        bq = fx.quantize(f["b_eff"], datum, k_exp)
        zq = fx.quantize(grid.download("z_base"), datum, k_exp)
        hq = fx.quantize(f["mobile"], 0.0, k_exp)
        y = L.yield_init(bq, zq, hq, None, None, dx=DX, dy=DX,
                         tan_start=np.tan(np.deg2rad(mat.start_angle_deg)),
                         tan_stop=np.tan(np.deg2rad(mat.stop_angle_deg)),
                         density=mat.assumed_bulk_density_kg_m3, gravity=9.81,
                         cohesion=mat.cohesion_proxy_pa, mobilization_depth=0.08, dry=1e-8,
                         fixed_point=True, quantum=q)
        want = L.canonical_labels(y["unstable"], 8)
        got = path.avalanche.labels()
        assert np.array_equal(got, want), k
        regions, largest, winner, total = L.component_summary(want)
        assert (st.regions, st.largest, st.unstable_cells) == (regions, largest, total), k
    path.close()
    assert worst_h <= FX32_BOUND_M, worst_h
    assert worst_b <= FX32_BOUND_M, worst_b


@pytest.mark.parametrize("residual,seed", [("always", 3), ("gated", 5)])
def test_fp64_small_path_with_residual_matches_oracle(residual, seed):
    """A 192^2 pile with the residual frontier on (``always``) and gated, with
    residual seeds queued at the start: the gate, seeding from local
    instabilities and the compact-frontier rounds against the oracle, fields
    bit-identical."""
    n = 192
    b = workloads.noise_pile(n, seed, DX)
    cut = workloads.BucketCut((n, n), DX, b, start=(0.25 * n * DX, 0.5 * n * DX))
    mat = _material()
    path = PlainPath(b, np.zeros_like(b), dx=DX, material=mat, precision="fp64", tile_size=32,
                     residual=residual)
    oracle = PathOracle(b, np.zeros_like(b), _oracle_cfg(mat, tile=32, residual=residual))
    # pending residual seeds at the start (the steepest cells of the pile, as
    # the reference's _seed_gpu_residual_frontier queues changed cells): the
    # reached mask and the 3x3-stencil tiles, on both sides
    seeds = _steep_cells(b, mat.stop_angle_deg)
    path.frontier.seed_mask(seeds)
    oracle.reached |= seeds
    oracle.pending = R.seed_tiles(seeds, 32)
    ran = 0
    for k in range(40):
        idx, tgt = cut.footprint((k + 1) * DT)
        g = path.step(DT, idx, tgt)
        o = oracle.step(DT, idx, tgt)
        _compare_step(k, g, o)
        ran += int(o.residual_rounds > 0)
        if k % 8 == 7:
            f = _fields(path)
            assert np.array_equal(f["b_eff"], oracle.b), k
            assert np.array_equal(f["mobile"], oracle.h), k
            assert np.array_equal(path.avalanche.labels(), o.labels), k
    path.close()
    if residual == "always":
        assert ran > 0
