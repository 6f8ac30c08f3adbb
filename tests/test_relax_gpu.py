"""GPU parity of the repose relaxation kernels (through the C ABI).

* relax_critical_slope, FP64: bit-identical heights and identical iteration
  counts vs the reference (golden fixtures); FX32: bit-identical to the
  fixed-point CPU mirror, exact volume, within 1e-6 m of FP64.
* compact frontier, FP64 uniform weights on the transposed (x, y) storage the
  reference's CPU adapter uses: bit-identical heights and equal round counts
  vs the reference's ``SparseTileFrontierMinimumSlopeAdapter``; weighted
  (Triangle-A-C) production semantics and FX32 vs the oracle schedule,
  including exact conservation of sum(w * h).
* event-driven reached-bbox backend (``EventDrivenMinimumSlopeAdapter``,
  FP64): bit-identical heights, equal iteration counts, classification and
  propagation bounding box vs the reference's adapter (golden fixture), and
  vs the oracle on a larger event.
"""

import numpy as np
import pytest

import soilb200
from oracle import fixed_point as fx
from oracle import relax as R

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def relax_golden():
    return np.load(GOLDEN / "relax.npz")


def test_fp64_relax_critical_slope_bitwise(relax_golden):
    for name in relax_golden["full_names"]:
        h = relax_golden[f"full/{name}/h"]
        spacing = tuple(relax_golden[f"full/{name}/spacing"])
        angle = float(relax_golden[f"full/{name}/angle"])
        out, st = soilb200.relax_critical_slope(h, spacing, angle, 20000, 1e-8, precision="fp64")
        assert st.iterations == int(relax_golden[f"full/{name}/iterations"]), name
        assert st.converged
        assert np.array_equal(out, relax_golden[f"full/{name}/out"]), name
        assert st.volume_after == pytest.approx(st.volume_before, rel=1e-12)
        assert st.max_slope <= np.tan(np.deg2rad(angle)) + 1e-6


def test_fx32_relax_critical_slope_matches_mirror(relax_golden):
    for name in relax_golden["full_names"]:
        h = relax_golden[f"full/{name}/h"]
        spacing = tuple(relax_golden[f"full/{name}/spacing"])
        angle = float(relax_golden[f"full/{name}/angle"])
        out, st = soilb200.relax_critical_slope(h, spacing, angle, 20000, 1e-8, precision="fx32")
        k, datum = soilb200.choose_quantization(h)
        hq, it, conv = R.relax_critical_slope_fixed(fx.quantize(h, datum, k), spacing,
                                                    float(np.tan(np.deg2rad(angle))), 2.0 ** -k)
        assert st.iterations == it and st.converged == conv, name
        assert np.array_equal(out, fx.dequantize(hq, datum, k)), name
        assert int(np.sum(hq)) == int(np.sum(fx.quantize(h, datum, k).astype(np.int64)))
        assert np.abs(out - relax_golden[f"full/{name}/out"]).max() <= 1e-6, name


def test_fp64_frontier_matches_reference_cpu_adapter(relax_golden):
    for name in relax_golden["event_names"]:
        h = relax_golden[f"event/{name}/h"]
        seeds = relax_golden[f"event/{name}/seeds"]
        tile = int(relax_golden[f"event/{name}/tile"])
        angle = float(relax_golden[f"event/{name}/angle"])
        hxy = np.ascontiguousarray(h.T)
        sxy = np.ascontiguousarray(seeds.T)
        grid = soilb200.DeviceGrid(hxy.shape, 0.05, 0.05, precision="fp64", tile_size=tile)
        grid.upload("b_eff", hxy)
        front = soilb200.FrontierRelaxation(grid, spacing=(0.05, 0.05), weighted=False)
        front.seed_mask(sxy)
        st = front.run(float(np.tan(np.deg2rad(angle))), 1e-8)
        out = grid.download("b_eff").T
        assert st.rounds == int(relax_golden[f"event/{name}/iterations"]), name
        assert np.array_equal(out, relax_golden[f"event/{name}/out"]), name
        assert not grid.download("frontier_reached").any()
        grid.close()


def _event(shape, seed):
    rng = np.random.default_rng(seed)
    ys, xs = np.indices(shape)
    h = 0.5 + 0.15 * np.sin(xs / 7.0) + 0.002 * rng.random(shape)
    seeds = np.zeros(shape, dtype=bool)
    for _ in range(4):
        r, c = rng.integers(2, shape[0] - 3), rng.integers(2, shape[1] - 3)
        h[r - 2:r + 3, c - 2:c + 3] += rng.uniform(0.2, 0.4)
        seeds[r - 2:r + 3, c - 2:c + 3] = True
    h[0, :3] += 0.3  # corner / edge vertices exercise the boundary weights
    seeds[0, :3] = True
    return h, seeds


@pytest.mark.parametrize("shape,tile", [((70, 90), 16), ((45, 33), 8)])
def test_fp64_weighted_frontier_matches_oracle(shape, tile):
    h, seeds = _event(shape, shape[0])
    crit = float(np.tan(np.deg2rad(33.0)))
    w = R.vertex_weights(shape, 0.05, 0.05)
    want, reached, rounds, _ = R.frontier_relax(h, seeds, R.seed_tiles(seeds, tile), tile=tile,
                                                spacing=(0.05, 0.05), crit_tan=crit,
                                                tolerance=1e-8, weights=w)
    grid = soilb200.DeviceGrid(shape, 0.05, 0.05, precision="fp64", tile_size=tile)
    grid.upload("b_eff", h)
    front = soilb200.FrontierRelaxation(grid, weighted=True)
    front.seed_mask(seeds)
    st = front.run(crit, 1e-8)
    assert st.rounds == rounds
    out = grid.download("b_eff")
    assert np.array_equal(out, want)
    assert float(np.sum(out * w)) == pytest.approx(float(np.sum(h * w)), rel=1e-13)
    grid.close()


@pytest.mark.parametrize("shape,tile", [((70, 90), 16), ((64, 64), 32)])
def test_fx32_weighted_frontier_matches_mirror_exactly(shape, tile):
    h, seeds = _event(shape, shape[1])
    crit = float(np.tan(np.deg2rad(33.0)))
    k, datum = soilb200.choose_quantization(h)
    hq = fx.quantize(h, datum, k).astype(np.int64)
    w6 = R.vertex_weights6(shape)
    want, reached, rounds, _ = R.frontier_relax(hq, seeds, R.seed_tiles(seeds, tile), tile=tile,
                                                spacing=(0.05, 0.05), crit_tan=crit,
                                                tolerance=1e-8, weights=w6, fixed_point=True,
                                                quantum=2.0 ** -k)
    grid = soilb200.DeviceGrid(shape, 0.05, 0.05, precision="fx32", tile_size=tile,
                               height_exponent=k, datum_m=datum)
    grid.upload("b_eff", h)
    front = soilb200.FrontierRelaxation(grid, weighted=True)
    front.seed_mask(seeds)
    st = front.run(crit, 1e-8)
    assert st.rounds == rounds
    out = grid.download("b_eff")
    assert np.array_equal(out, fx.dequantize(want, datum, k))
    assert int(np.sum(want * w6)) == int(np.sum(hq * w6))  # exact sum(w*h)
    grid.close()


def test_frontier_round_cap_raises_nonconvergence():
    h, seeds = _event((40, 40), 3)
    grid = soilb200.DeviceGrid((40, 40), 0.05, 0.05, precision="fp64", tile_size=8)
    grid.upload("b_eff", h)
    front = soilb200.FrontierRelaxation(grid)
    front.seed_mask(seeds)
    with pytest.raises(soilb200.NumericalNonconvergenceError, match="NUMERICAL_NONCONVERGENCE"):
        front.run(float(np.tan(np.deg2rad(33.0))), 1e-8, max_rounds=1)
    grid.close()


def test_relax_validation_messages():
    with pytest.raises(ValueError, match="non-negative"):
        soilb200.relax_critical_slope(-np.ones((4, 4)), (0.05, 0.05))
    with pytest.raises(ValueError, match="between 0 and 90"):
        soilb200.relax_critical_slope(np.ones((4, 4)), (0.05, 0.05), 95.0)
    with pytest.raises(ValueError, match="both dimensions >= 2"):
        soilb200.relax_critical_slope(np.ones((1, 4)), (0.05, 0.05))


class _Grid:
    def __init__(self, nx, ny, dx, dy):
        self.nx, self.ny, self.dx, self.dy = int(nx), int(ny), float(dx), float(dy)


def test_event_driven_adapter_bit_identical_to_reference():
    """soilb200.EventDrivenMinimumSlopeAdapter (sb_relax_reached) against the
    reference's EventDrivenMinimumSlopeAdapter.solve (golden fixture): stable
    heights bit for bit, equal iteration counts, the same classification and
    propagation bounding box; volume unchanged."""
    g = np.load(GOLDEN / "event.npz")
    for name in g["names"]:
        nx, ny, dx, dy = g[f"{name}/grid"]
        thr = int(g[f"{name}/threshold"])
        cfg = soilb200.MiniSlopeConfig(critical_angle_deg=float(g[f"{name}/angle"]),
                                       tolerance=1e-8, large_avalanche_iteration_threshold=thr,
                                       numerical_safety_max_iterations=max(10_000, thr))
        solver = soilb200.EventDrivenMinimumSlopeAdapter(_Grid(nx, ny, dx, dy), cfg, tile_size=8)
        solver.set_reference_height(g[f"{name}/base"])
        res = solver.solve(g[f"{name}/initial"])
        assert res.converged, name
        assert res.iteration_count == int(g[f"{name}/iterations"]), name
        assert np.array_equal(res.heightmap_stable, g[f"{name}/stable"]), name
        d = res.diagnostics
        assert d["avalanche_classification"] == str(g[f"{name}/classification"]), name
        assert d["propagation_bbox_yx"] == [int(v) for v in g[f"{name}/propagation_bbox"]], name
        assert res.volume_after_m3 == pytest.approx(res.volume_before_m3, rel=1e-12)
        # a second solve of the stable state has nothing to do
        again = solver.solve(res.heightmap_stable)
        assert again.iteration_count == 0
        assert d["avalanche_classification"] != solver.NO_EVENT
        solver.close()


def test_event_driven_adapter_matches_oracle_on_a_larger_event():
    """A 300 x 260 event (many 32-cell tiles, most of them never reached, so
    the kernel's bounding-box skip is exercised) against oracle.relax.reached_relax."""
    rng = np.random.default_rng(21)
    ny, nx = 300, 260
    base = 0.4 + 0.002 * rng.random((ny, nx))
    init = base.copy()
    for _ in range(5):
        r, c = rng.integers(20, ny - 20), rng.integers(20, nx - 20)
        init[r - 3:r + 4, c - 3:c + 4] += rng.uniform(0.2, 0.5)
    seeds = np.abs(init - base) > 1e-8
    crit = float(np.tan(np.deg2rad(32.0)))
    want, reached, it = R.reached_relax(init.T, seeds.T, (0.05, 0.05), crit, 1e-8)
    cfg = soilb200.MiniSlopeConfig(critical_angle_deg=32.0, tolerance=1e-8)
    solver = soilb200.EventDrivenMinimumSlopeAdapter(_Grid(nx, ny, 0.05, 0.05), cfg)
    solver.set_reference_height(base)
    res = solver.solve(init)
    assert res.iteration_count == it
    assert np.array_equal(res.heightmap_stable, want.T)
    assert res.diagnostics["reached_cell_count"] == int(reached.sum())
    solver.close()


def test_event_driven_adapter_safety_limit_raises():
    g = np.load(GOLDEN / "event.npz")
    name = "toe65"
    nx, ny, dx, dy = g[f"{name}/grid"]
    cfg = soilb200.MiniSlopeConfig(critical_angle_deg=30.0, tolerance=1e-8,
                                   large_avalanche_iteration_threshold=10,
                                   numerical_safety_max_iterations=20)
    solver = soilb200.EventDrivenMinimumSlopeAdapter(_Grid(nx, ny, dx, dy), cfg, tile_size=8)
    solver.set_reference_height(g[f"{name}/base"])
    with pytest.raises(soilb200.NumericalNonconvergenceError, match="NUMERICAL_NONCONVERGENCE"):
        solver.solve(g[f"{name}/initial"])
    solver.close()


def test_weighted_frontier_compacted_list_beyond_one_wave():
    """More active tiles than the list-driven kernels have CTAs (a 512^2 grid of
    8-cell tiles, 4096 tiles, events scattered over all of it): the ballot-
    compacted tile list with appended stencil tiles must still reproduce the
    oracle's compact-frontier schedule bit for bit, with equal round counts."""
    rng = np.random.default_rng(99)
    shape = (512, 512)
    h = 0.5 + 0.003 * rng.random(shape)
    seeds = np.zeros(shape, dtype=bool)
    for _ in range(1500):
        r, c = rng.integers(2, shape[0] - 3), rng.integers(2, shape[1] - 3)
        h[r - 1:r + 2, c - 1:c + 2] += rng.uniform(0.1, 0.25)
        seeds[r - 1:r + 2, c - 1:c + 2] = True
    tile = 8
    crit = float(np.tan(np.deg2rad(33.0)))
    w = R.vertex_weights(shape, 0.05, 0.05)
    want, reached, rounds, hist = R.frontier_relax(h, seeds, R.seed_tiles(seeds, tile), tile=tile,
                                                   spacing=(0.05, 0.05), crit_tan=crit,
                                                   tolerance=1e-8, weights=w, record=True)
    assert len(hist[0]["active"]) > 1184  # more list entries than CTAs in the first round
    grid = soilb200.DeviceGrid(shape, 0.05, 0.05, precision="fp64", tile_size=tile)
    grid.upload("b_eff", h)
    front = soilb200.FrontierRelaxation(grid, weighted=True)
    front.seed_mask(seeds)
    st = front.run(crit, 1e-8)
    assert st.rounds == rounds
    assert np.array_equal(grid.download("b_eff"), want)
    assert not grid.download("frontier_reached").any()
    grid.close()


@pytest.mark.parametrize("precision", ["fp64", "fx32"])
def test_host_driven_sweeps_equal_sweep_graph(relax_golden, precision, monkeypatch):
    """SOILB200_NO_GRAPH=1 (sweeps launched from the host, the mode profilers
    use) gives the sweep graph's heights and iteration count."""
    for name in relax_golden["full_names"][:3]:
        h = relax_golden[f"full/{name}/h"]
        spacing = tuple(relax_golden[f"full/{name}/spacing"])
        angle = float(relax_golden[f"full/{name}/angle"])
        monkeypatch.delenv("SOILB200_NO_GRAPH", raising=False)
        a, sa = soilb200.relax_critical_slope(h, spacing, angle, 20000, 1e-8, precision=precision)
        monkeypatch.setenv("SOILB200_NO_GRAPH", "1")
        b, sb = soilb200.relax_critical_slope(h, spacing, angle, 20000, 1e-8, precision=precision)
        monkeypatch.delenv("SOILB200_NO_GRAPH")
        assert np.array_equal(a, b), name
        assert sa.iterations == sb.iterations, name
