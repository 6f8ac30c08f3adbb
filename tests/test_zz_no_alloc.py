"""GPU test of the allocation-free entry point ``sb_label_mask_static``.

Some callers cannot allocate device memory while running: a simulator
plugin's frame callback that works inside a fixed memory budget handed over at
start-up, where cudaMalloc could block or synchronise the device.  This entry
point labels a caller-provided device mask into
caller-provided device labels with its scratch in a static device array.  The
test calls it through the C ABI twice in a row (the scratch keeps the previous
call's contents) and checks labels and statistics against the context-based
entry point ``sb_label_mask`` on the same masks (labels are integers, so the
tolerance is exact equality), and that the device's free memory
(``cudaMemGetInfo``, which also sees allocations made outside torch) is the
same before and after a call.  The file name makes pytest collect it last.
"""

import numpy as np
import pytest
import torch

import soilb200
from soilb200 import _lib

pytestmark = pytest.mark.gpu


def _reference(mask, conn):
    grid = soilb200.DeviceGrid(mask.shape, 0.05, 0.05)
    try:
        labels, st = soilb200.label_mask(grid, mask, conn)
    finally:
        grid.close()
    return labels, st


@pytest.mark.parametrize("conn", [8, 4])
def test_static_scratch_labels_match_context_entry_point_twice(conn):
    rng = np.random.default_rng(31 + conn)
    masks = [rng.random((701, 701)) < 0.58, rng.random((257, 300)) < 0.45]
    for mask in masks:  # two calls in a row, different sizes and contents
        want, st_ref = _reference(mask, conn)
        d_mask = torch.from_numpy(mask.astype(np.int32)).cuda()
        d_labels = torch.full(mask.shape, 12345, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        st = soilb200.label_mask_preallocated(d_mask.data_ptr(), d_labels.data_ptr(), mask.shape,
                                              conn, dx_m=0.05, dy_m=0.05)
        got = d_labels.cpu().numpy()
        assert np.array_equal(got, want)
        assert st.connected_region_count == st_ref.connected_region_count
        assert st.largest_connected_cell_count == st_ref.largest_connected_cell_count
        assert st.winner_root == st_ref.winner_root
        assert st.unstable_cell_count == st_ref.unstable_cell_count
        assert st.largest_connected_area_m2 == st_ref.largest_connected_area_m2


def test_static_scratch_call_allocates_no_device_memory():
    rng = np.random.default_rng(77)
    mask = rng.random((512, 640)) < 0.55
    d_mask = torch.from_numpy(mask.astype(np.int32)).cuda()
    d_labels = torch.empty(mask.shape, dtype=torch.int32, device="cuda")
    soilb200.label_mask_preallocated(d_mask.data_ptr(), d_labels.data_ptr(), mask.shape, 8)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        soilb200.label_mask_preallocated(d_mask.data_ptr(), d_labels.data_ptr(), mask.shape, 8)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_static_scratch_rejects_grids_beyond_capacity():
    d = torch.zeros((725, 725), dtype=torch.int32, device="cuda")  # 525625 > 524288 cells
    with pytest.raises(ValueError, match="exceeds the static scratch capacity"):
        soilb200.label_mask_preallocated(d.data_ptr(), d.data_ptr(), d.shape, 8)
    st = _lib.LabelStats()
    rc = _lib.load().sb_label_mask_static(d.data_ptr(), d.data_ptr(), 725, 725, 8, 1.0, 1.0,
                                          0, st)
    assert rc == _lib.SB_ERR_CAPACITY
