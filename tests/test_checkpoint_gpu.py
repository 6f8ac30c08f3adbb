"""GPU test of the device checkpoint boundary (reference npz replay format).

A state is advanced (entrainment, Mobile V2, deposition, avalanche
activation), written, restored into a fresh state, and both must hold the
same fields bit for bit; the archive carries the reference's field names,
schema and terrain hash, and an archive lacking the optional fields (as
older reference checkpoints do) restores with the reference's defaults.
"""

import json

import numpy as np
import pytest

import soilb200
from soilb200 import checkpoint as ck
from soilb200.bulk_state import B200BulkState, B200DepositionOperator, B200ProductionMobileV2Solver

pytestmark = pytest.mark.gpu

DX = 0.05
FIELDS = ("z_base", "b_eff", "mobile", "momentum_x", "momentum_y", "latch", "activation_count",
          "r2m_cumulative", "m2r_cumulative", "owned_surface", "first_activation_time",
          "frontier_reached", "previous_component")


def _advanced_state(precision):
    n = 80
    ys, xs = np.indices((n, n), dtype=np.float64)
    b0 = np.maximum(0.0, 1.4 - 1.0 * np.hypot(xs - n / 2, ys - n / 2) * DX)
    st = B200BulkState(b0.shape, DX, DX, b0, precision=precision, mobile_headroom_m=1.0)
    mat = soilb200.MaterialScenario("pile", 1600.0, 35.0, 0.0, 0.5, 38.0, 30.0, 0.55)
    idx = np.arange(30 * n + 10, 30 * n + 30, dtype=np.int32)
    st.entrain_host_indices(idx, np.full(idx.size, 0.05), reason="cut")
    solver = B200ProductionMobileV2Solver(state=st, config=soilb200.MobileV2Config())
    solver.bind_device_state(st, mat)
    solver.step_resident(1.0 / 60.0)
    dep = B200DepositionOperator()
    dep.bind_device_state(st)
    dep.step_resident(mat, 1.0 / 60.0)
    cfg = soilb200.LargeAvalancheTransitionConfig(persistence_time_s=1e-3)
    br = soilb200.B200LargeAvalancheBridge(st.grid, mat, cfg, state=st)
    br.observe_and_maybe_mobilize(1.0 / 60.0)
    st.advance_time(1.0 / 60.0)
    return st, br, b0, mat, cfg


@pytest.mark.parametrize("precision", ["fp64", "fx32"])
def test_checkpoint_round_trip(tmp_path, precision):
    st, br, b0, mat, cfg = _advanced_state(precision)
    rec = ck.write_device_checkpoint(st, tmp_path / "c.npz", provenance={"test": 1}, bridge=br)
    with np.load(tmp_path / "c.npz") as z:
        assert set(ck.FLOAT_FIELDS) | set(ck.INT_FIELDS) <= set(z.files)
        meta = json.loads(str(z["checkpoint_record_json"]))
        assert meta["schema"] == ck.SCHEMA
        assert meta["terrain_hash_sha256"] == ck.sha256_array(z["b_eff"])
    assert rec["checkpoint_hash_sha256"] == ck.sha256_file(tmp_path / "c.npz")
    kw = {}
    if precision == "fx32":
        kw = {"height_exponent": st.grid.height_exponent, "datum_m": st.grid.datum}
    st2 = B200BulkState(b0.shape, DX, DX, np.zeros_like(b0), precision=precision, **kw)
    br2 = soilb200.B200LargeAvalancheBridge(st2.grid, mat, cfg, state=st2)
    ck.restore_device_checkpoint(st2, tmp_path / "c.npz", bridge=br2)
    for name in FIELDS:
        assert np.array_equal(st2.grid.download(name), st.grid.download(name)), name
    assert st2.timestamp_device_s == st.timestamp_device_s
    assert br2._persistence_s == br._persistence_s
    st.close()
    st2.close()


def test_restore_older_archive_defaults(tmp_path):
    n = 24
    b = 0.5 + 0.01 * np.arange(n * n, dtype=np.float64).reshape(n, n) / (n * n)
    rec = {"schema": ck.SCHEMA, "shape_yx": [n, n], "resolution_xy_m": [DX, DX],
           "device_timestamp_s": 2.5, "large_avalanche": {"persistence_s": 0.1, "has_previous": True}}
    np.savez(tmp_path / "old.npz", b_eff=b, mobile=np.full((n, n), 0.01),
             checkpoint_record_json=np.asarray(json.dumps(rec)))
    st = B200BulkState((n, n), DX, DX, np.zeros((n, n)), precision="fp64")
    ck.restore_device_checkpoint(st, tmp_path / "old.npz")
    assert np.array_equal(st.grid.download("b_eff"), b)
    assert np.array_equal(st.grid.download("z_base"), np.zeros((n, n)))
    assert np.array_equal(st.grid.download("owned_surface"), b + 0.01)
    assert st.timestamp_device_s == 2.5
    with pytest.raises(RuntimeError, match="DEVICE_CHECKPOINT_SHAPE_MISMATCH"):
        st_small = B200BulkState((n - 1, n), DX, DX, np.zeros((n - 1, n)), precision="fp64")
        try:
            ck.restore_device_checkpoint(st_small, tmp_path / "old.npz")
        finally:
            st_small.close()
    st.close()


class _Bridge:
    _persistence_s = 0.0
    _has_previous = False


def test_restore_archive_written_by_the_reference(tmp_path):
    """An archive written by the reference's write_device_checkpoint (golden
    fixture) restores into a B200BulkState: every modelled field bit for bit,
    the bridge's persistence state, the device time; written back by this
    library, the modelled fields and the terrain hash are unchanged."""
    from conftest import GOLDEN
    path = GOLDEN / "reference_checkpoint.npz"
    with np.load(path) as z:
        fields = {name: z[name].copy() for name in z.files if name != "checkpoint_record_json"}
    st = B200BulkState(fields["b_eff"].shape, DX, DX, fields["b_eff"], precision="fp64",
                       mobile_headroom_m=1.0)
    br = _Bridge()
    rec = ck.restore_device_checkpoint(st, path, bridge=br)
    assert br._persistence_s == 0.0833 and br._has_previous
    assert st.timestamp_device_s == rec["device_timestamp_s"]
    for name, dev in ck._DEVICE_NAME.items():
        if dev is None:
            continue
        got = st.grid.download(dev)
        assert np.array_equal(got, fields[name].astype(got.dtype)), name
    out = ck.write_device_checkpoint(st, tmp_path / "back.npz", provenance={}, bridge=br)
    assert out["terrain_hash_sha256"] == rec["terrain_hash_sha256"]
    with np.load(tmp_path / "back.npz") as z:
        for name, dev in ck._DEVICE_NAME.items():
            if dev is not None:
                assert np.array_equal(z[name], fields[name]), name
    st.close()
