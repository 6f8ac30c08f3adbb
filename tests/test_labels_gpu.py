"""GPU parity of the large-avalanche labelling kernels (through the C ABI).

Labels are compared bit for bit: every unstable cell must carry the minimum
flat index of its component (oracle: scipy component labelling + per-component
minimum), and region count / largest size / largest mask must equal the
reference's ``_largest_connected_region`` outputs (golden fixtures).
"""

import numpy as np
import pytest

import soilb200
from oracle import fixed_point as fx
from oracle import labels as L

from conftest import GOLDEN

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def labels_golden():
    return np.load(GOLDEN / "labels.npz")


def test_mask_labels_match_reference_and_canonical_oracle(labels_golden):
    for name in labels_golden["mask_names"]:
        conn = int(str(name).split("/c")[1])
        mask = labels_golden[f"{name}/mask"]
        largest, regions, size = soilb200.largest_connected_region(mask, conn)
        assert regions == int(labels_golden[f"{name}/regions"]), name
        assert size == int(labels_golden[f"{name}/largest_size"]), name
        assert np.array_equal(largest, labels_golden[f"{name}/largest"]), name
        if mask.any():
            grid = soilb200.DeviceGrid(mask.shape, 1.0, 1.0)
            labels, st = soilb200.label_mask(grid, mask, conn)
            assert np.array_equal(labels, L.canonical_labels(mask, conn)), name
            grid.close()


@pytest.mark.parametrize("shape,p,conn", [((257, 300), 0.55, 8), ((129, 97), 0.45, 4),
                                          ((701, 701), 0.58, 8), ((64, 1030), 0.6, 4)])
def test_random_masks_canonical_labels(shape, p, conn):
    rng = np.random.default_rng(shape[0] * 7 + shape[1])
    mask = rng.random(shape) < p
    grid = soilb200.DeviceGrid(shape, 0.05, 0.05)
    labels, st = soilb200.label_mask(grid, mask, conn)
    want = L.canonical_labels(mask, conn)
    assert np.array_equal(labels, want)
    regions, largest, winner, total = L.component_summary(want)
    assert st.connected_region_count == regions
    assert st.largest_connected_cell_count == largest
    assert st.winner_root == winner
    assert st.unstable_cell_count == total
    grid.close()


def _material(start=38.0, stop=30.0, cohesion=0.0):
    return soilb200.MaterialScenario("golden", 1370.0, 29.8, cohesion, 0.5, start, stop, 0.35)


def test_fp64_yield_labels_match_reference_detector(labels_golden):
    resting = labels_golden["yield/resting"]
    grid = soilb200.DeviceGrid(resting.shape, 0.05, 0.05, precision="fp64")
    grid.upload("b_eff", resting)
    grid.upload("z_base", np.zeros_like(resting))
    bridge = soilb200.B200LargeAvalancheBridge(grid, _material())
    st = bridge.label()
    labels = bridge.labels()
    assert np.array_equal(labels >= 0, labels_golden["yield/start_mask"])
    assert st.connected_region_count == int(labels_golden["yield/regions"])
    assert st.largest_connected_cell_count == int(labels_golden["yield/largest_size"])
    assert np.array_equal(labels == st.winner_root, labels_golden["yield/largest"])
    slope = grid.download("slope")
    assert np.abs(slope - labels_golden["yield/slope_rad"]).max() <= 1e-12
    grid.close()


def test_fx32_yield_labels_equal_fixed_point_oracle():
    rng = np.random.default_rng(5)
    ny, nx = 150, 170
    ys, xs = np.indices((ny, nx))
    b = 0.6 + 0.5 * np.sin(xs / 9.0) * np.cos(ys / 7.0) + 0.02 * rng.random((ny, nx))
    z = b - 0.05 - 0.1 * rng.random((ny, nx))
    h = np.where(rng.random((ny, nx)) < 0.2, 0.01 * rng.random((ny, nx)), 0.0)
    k, datum = soilb200.choose_quantization(b, z, mobile=h)
    grid = soilb200.DeviceGrid((ny, nx), 0.05, 0.05, precision="fx32", height_exponent=k,
                               datum_m=datum)
    for name, arr in (("b_eff", b), ("z_base", z), ("mobile", h)):
        grid.upload(name, arr)
    mat = _material()
    bridge = soilb200.B200LargeAvalancheBridge(grid, mat)
    st = bridge.label(release_settled_latches=False)
    labels = bridge.labels()
    bq, zq, hq = fx.quantize(b, datum, k), fx.quantize(z, datum, k), fx.quantize(h, 0.0, k)
    start, stop = np.deg2rad(38.0), np.deg2rad(30.0)
    y = L.yield_init(bq, zq, hq, None, None, dx=0.05, dy=0.05, tan_start=np.tan(start),
                     tan_stop=np.tan(stop), density=1370.0, gravity=9.81, cohesion=0.0,
                     mobilization_depth=0.08, dry=1e-8, fixed_point=True, quantum=2.0 ** -k)
    want = L.canonical_labels(y["unstable"], 8)
    assert np.array_equal(labels, want)
    # the float32 yield fields bit for bit, and the slope within the arc
    # tangent's bound of the double-precision angle of the same gradient
    slope = grid.download("slope").astype(np.float32)
    assert np.array_equal(slope, y["slope"])
    assert np.array_equal(grid.download("severity").astype(np.float32), y["severity"])
    exact = np.arctan(np.hypot(y["gx"].astype(np.float64), y["gy"].astype(np.float64)))
    assert np.abs(slope - exact).max() <= 3.0e-7
    regions, largest, winner, total = L.component_summary(want)
    assert (st.connected_region_count, st.largest_connected_cell_count, st.winner_root) == \
        (regions, largest, winner)
    # exact integer area of the winner (Triangle-A-C weights in units of dx*dy/6)
    from oracle.relax import vertex_weights6
    area6 = int(vertex_weights6((ny, nx))[want == winner].sum())
    assert st.largest_connected_area_m2 == pytest.approx(area6 * 0.05 * 0.05 / 6.0, rel=1e-15)
    grid.close()


@pytest.mark.parametrize("n", [65, 257, 701])
def test_whole_domain_plane_acceptance(n):
    # tools/run_gpu_large_avalanche_acceptance.py:35-62: a 42 deg plane is one
    # connected above-start region covering every cell.
    cols = np.indices((n, n))[1].astype(np.float64)
    resting = 1.0 + np.tan(np.deg2rad(42.0)) * cols * 0.05
    for precision in ("fp64", "fx32"):
        k, datum = soilb200.choose_quantization(resting)
        grid = soilb200.DeviceGrid((n, n), 0.05, 0.05, precision=precision, height_exponent=k,
                                   datum_m=datum)
        grid.upload("b_eff", resting)
        grid.upload("z_base", np.zeros((n, n)))
        bridge = soilb200.B200LargeAvalancheBridge(
            grid, _material(), soilb200.LargeAvalancheTransitionConfig(persistence_time_s=1 / 60))
        d = bridge.observe(1.0 / 60.0)
        assert d.connected_region_count == 1
        assert d.largest_connected_cell_count == n * n
        assert d.classification == bridge.LARGE_AVALANCHE_MOBILE_PATH
        assert np.all(bridge.labels() == 0)
        grid.close()


def test_local_instability_seeds_frontier_tiles():
    n = 96
    b = np.full((n, n), 1.0)
    b[40:44, 50:53] += 0.6  # a small steep bump: local instability only
    grid = soilb200.DeviceGrid((n, n), 0.05, 0.05, precision="fp64", tile_size=32)
    grid.upload("b_eff", b)
    grid.upload("z_base", np.zeros((n, n)))
    bridge = soilb200.B200LargeAvalancheBridge(grid, _material())
    d = bridge.observe(1.0 / 60.0)
    assert d.classification == bridge.LOCAL_STATIC_INSTABILITY
    labels = bridge.labels()
    winner = labels == d.winner_label
    reached = grid.download("frontier_reached").astype(bool)
    assert np.array_equal(reached, winner)
    tiles = soilb200.FrontierRelaxation(grid).active_tiles()
    rows, cols = np.nonzero(winner)
    want = np.unique((rows // 32) * 3 + cols // 32)
    assert np.array_equal(tiles, want)
    grid.close()
