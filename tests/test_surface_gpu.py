"""GPU tests of surface publication: dirty tiles after a mutation, tile
downloads with their one-cell overlap, and batched bilinear queries (FP64:
equal bit for bit to the reference's CPU sampler on its golden queries, and
to the oracle's clamped restatement of the reference query kernel, which is
pinned to that sampler, on queries outside the grid)."""

import numpy as np
import pytest

from conftest import GOLDEN
from oracle.surface import bilinear as _bilinear

from soilb200.bulk_state import B200BulkState

pytestmark = pytest.mark.gpu

DX = 0.05


@pytest.mark.parametrize("precision", ["fp64", "fx32"])
def test_dirty_tiles_downloads_and_queries(precision):
    rng = np.random.default_rng(3)
    ny, nx = 70, 90
    b = 0.5 + 0.1 * rng.random((ny, nx))
    st = B200BulkState((ny, nx), DX, DX, b, precision=precision, tile_size=16,
                       mobile_headroom_m=0.5)
    st.capture_surface_for_dirty_tracking()
    assert st.collect_surface_dirty_tiles().size == 0
    idx = np.asarray([20 * nx + 40, 20 * nx + 41, 65 * nx + 5], dtype=np.int32)
    st.entrain_host_indices(idx, np.full(3, 0.05), reason="test")   # b + h unchanged
    assert st.collect_surface_dirty_tiles().size == 0
    mob = st.grid.download("mobile")
    mob[33, 70] += 0.02
    st.grid.upload("mobile", mob)
    tiles = st.collect_surface_dirty_tiles()
    assert tiles.tolist() == [(33 // 16) * 6 + 70 // 16]
    surface = st.grid.download("b_eff") + st.grid.download("mobile")
    got = st.download_dirty_tiles()
    t = int(tiles[0])
    r0, c0 = (t // 6) * 16, (t % 6) * 16
    assert np.array_equal(got[t], surface[r0:r0 + 17, c0:c0 + 17])
    assert st.consume_dirty_tile_ids().size == 0
    q = np.column_stack([rng.uniform(-2, ny + 2, 500), rng.uniform(-2, nx + 2, 500)])
    vals = st.sample_surface_bilinear(q, source="test")
    ref = _bilinear(surface, q[:, 0], q[:, 1])
    if precision == "fp64":
        assert np.array_equal(vals, ref)
    else:
        assert np.abs(vals - ref).max() <= 1e-12
    with pytest.raises(ValueError):
        st.sample_surface_bilinear(np.zeros((2, 3)), source="test")
    st.close()


@pytest.mark.parametrize("precision", ["fp64", "fx32"])
def test_surface_queries_match_reference_sampler(precision):
    z = np.load(GOLDEN / "surface.npz")
    resting, mobile, q = z["resting"], z["mobile"], z["queries"]
    st = B200BulkState(resting.shape, DX, DX, resting, precision=precision, tile_size=16,
                       mobile_headroom_m=0.5)
    st.grid.upload("mobile", mobile)
    vals = st.sample_surface_bilinear(q, source="test")
    if precision == "fp64":
        assert np.array_equal(vals, z["values"])
    else:  # heights held in int32 quanta: within one quantum per corner
        assert np.abs(vals - z["values"]).max() <= 4.0 * st.grid.quantum
    st.close()


def test_surface_query_known_answers():
    """The reference's own device-state test (tests/test_device_bulk_state.py:
    116-126): resting heights 0..255 on a 16 x 16 grid."""
    grid = np.arange(256, dtype=np.float64).reshape(16, 16)
    st = B200BulkState(grid.shape, DX, DX, grid, precision="fp64", tile_size=4)
    vals = st.sample_surface_bilinear(np.asarray([[1.0, 2.0], [2.5, 3.5]]), source="test")
    assert vals.tolist() == [18.0, 43.5]
    st.close()
