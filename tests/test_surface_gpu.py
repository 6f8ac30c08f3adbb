"""GPU tests of surface publication: dirty tiles after a mutation, tile
downloads with their one-cell overlap, and batched bilinear queries
(FP64: equal to the reference kernel's arithmetic restated in NumPy)."""

import numpy as np
import pytest

from soilb200.bulk_state import B200BulkState

pytestmark = pytest.mark.gpu

DX = 0.05


def _bilinear(surface, rows, cols):
    ny, nx = surface.shape
    row = np.clip(rows, 0.0, ny - 1.0)
    col = np.clip(cols, 0.0, nx - 1.0)
    r0 = np.floor(row).astype(int)
    c0 = np.floor(col).astype(int)
    r1 = np.minimum(r0 + 1, ny - 1)
    c1 = np.minimum(c0 + 1, nx - 1)
    fr, fc = row - r0, col - c0
    return ((1.0 - fr) * (1.0 - fc) * surface[r0, c0] + (1.0 - fr) * fc * surface[r0, c1]
            + fr * (1.0 - fc) * surface[r1, c0] + fr * fc * surface[r1, c1])


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
