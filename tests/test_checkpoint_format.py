"""CPU test of checkpoint interoperability with the reference.

``tests/golden/reference_checkpoint.npz`` was written by the reference's own
``write_device_checkpoint`` (runtime/device_checkpoint.py:65-124) from a stub
core (``tests/golden/make_golden.py --checkpoint``).  This library's format
module must read it: the same field names and dtypes, the record schema, and
the terrain hash recomputed by ``soilb200.checkpoint.sha256_array``.  An
archive written by this library carries every record key the reference
writes.
"""

import json

import numpy as np

from soilb200 import checkpoint as ck

from conftest import GOLDEN


def test_reference_written_archive_has_this_library_s_layout():
    with np.load(GOLDEN / "reference_checkpoint.npz", allow_pickle=False) as z:
        files = set(z.files)
        assert set(ck.FLOAT_FIELDS) | set(ck.INT_FIELDS) | {"checkpoint_record_json"} == files
        record = json.loads(str(z["checkpoint_record_json"]))
        for name in ck.FLOAT_FIELDS:
            assert z[name].dtype == np.float64, name
            assert z[name].shape == tuple(record["shape_yx"]), name
        for name in ck.INT_FIELDS:
            assert z[name].dtype == np.int32, name
        assert record["schema"] == ck.SCHEMA
        assert record["terrain_hash_sha256"] == ck.sha256_array(z["b_eff"])
        assert record["large_avalanche"] == {"persistence_s": 0.0833, "has_previous": True}
        assert record["minislope"]["active_tiles"] == [0, 2]
        assert record["terrain_state_semantics"]["H_free"] == "b_eff + mobile"
    # every key of the reference's record is one this library writes
    ours = {"schema", "terrain_state_semantics", "runtime_backend", "state_authority",
            "shape_yx", "resolution_xy_m", "device_timestamp_s", "metadata", "large_avalanche",
            "minislope", "dirty_tiles", "terrain_hash_sha256", "provenance", "precision"}
    assert set(record) <= ours
