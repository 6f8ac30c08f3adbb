"""Device checkpoint boundary: the reference's npz replay format.

Same archive layout as runtime/device_checkpoint.py:21-45 and :65-124 -- one
array per field name (``FLOAT_FIELDS`` float64, ``INT_FIELDS`` int32, shape
(ny, nx)) plus ``checkpoint_record_json`` (schema
``390F_PRODUCTION_DEVICE_CHECKPOINT/v2``, shape, resolution, device time,
large-avalanche persistence, frontier state, terrain hash), so checkpoints
move between the reference and this library for replay.  Fields this library
does not model (``track_rut``, ``active_mask``, ``deposition_mask``,
``mobile_flux_export_cumulative``) are written as zeros and ignored on
restore.  Full-field transfers happen only here, at a named boundary.
"""

from __future__ import annotations

import hashlib
import json
from pathlib import Path
from typing import Any, Mapping

import numpy as np

SCHEMA = "390F_PRODUCTION_DEVICE_CHECKPOINT/v2"

FLOAT_FIELDS = (
    "z_base", "b_eff", "mobile", "momentum_x", "momentum_y", "track_rut",
    "avalanche_first_activation_time", "avalanche_last_activation_time",
    "avalanche_owned_surface", "avalanche_owned_export_baseline", "mobile_export_cumulative",
    "mobile_flux_export_cumulative", "avalanche_r2m_cumulative", "avalanche_m2r_cumulative",
)
INT_FIELDS = (
    "active_mask", "material_mask", "frontier_reached", "avalanche_latch",
    "avalanche_previous_component", "avalanche_activation_count", "deposition_mask",
)

# archive name -> device field name (None: not modelled, zeros on write)
_DEVICE_NAME = {
    "z_base": "z_base", "b_eff": "b_eff", "mobile": "mobile", "momentum_x": "momentum_x",
    "momentum_y": "momentum_y", "track_rut": None,
    "avalanche_first_activation_time": "first_activation_time",
    "avalanche_last_activation_time": "last_activation_time",
    "avalanche_owned_surface": "owned_surface",
    "avalanche_owned_export_baseline": "owned_export_baseline",
    "mobile_export_cumulative": "export_cumulative", "mobile_flux_export_cumulative": None,
    "avalanche_r2m_cumulative": "r2m_cumulative", "avalanche_m2r_cumulative": "m2r_cumulative",
    "active_mask": None, "material_mask": "forcing", "frontier_reached": "frontier_reached",
    "avalanche_latch": "latch", "avalanche_previous_component": "previous_component",
    "avalanche_activation_count": "activation_count", "deposition_mask": None,
}


def sha256_file(path) -> str:
    digest = hashlib.sha256()
    with Path(path).open("rb") as stream:
        for block in iter(lambda: stream.read(1024 * 1024), b""):
            digest.update(block)
    return digest.hexdigest()


def sha256_array(value: np.ndarray) -> str:
    """Hash of dtype name, shape (int64) and bytes, as the reference computes it."""
    array = np.ascontiguousarray(np.asarray(value))
    digest = hashlib.sha256()
    digest.update(str(array.dtype).encode("ascii"))
    digest.update(np.asarray(array.shape, dtype=np.int64).tobytes())
    digest.update(array.tobytes())
    return digest.hexdigest()


def write_device_checkpoint(state, path, *, provenance: Mapping[str, Any], bridge=None,
                            frontier_active_tiles=(), frontier_iterations: int = 0,
                            relaxation_pending: bool = False, metadata=None) -> dict:
    """Persist the replay-relevant state of a B200BulkState (and optionally the
    large-avalanche bridge's persistence) to ``path``."""
    grid = state.grid
    arrays = {}
    for name in FLOAT_FIELDS:
        dev = _DEVICE_NAME[name]
        arrays[name] = (grid.download(dev).astype(np.float64) if dev else
                        np.zeros(state.shape, np.float64))
    for name in INT_FIELDS:
        dev = _DEVICE_NAME[name]
        arrays[name] = (grid.download(dev).astype(np.int32) if dev else
                        np.zeros(state.shape, np.int32))
    record = {
        "schema": SCHEMA,
        "terrain_state_semantics": {
            "authoritative": ["z_base", "b_eff", "mobile", "momentum_x", "momentum_y"],
            "H_free": "b_eff + mobile",
            "h_resting": "b_eff - z_base",
        },
        "runtime_backend": "GPU_RUNTIME",
        "state_authority": "DEVICE",
        "shape_yx": list(state.shape),
        "resolution_xy_m": [grid.dx, grid.dy],
        "device_timestamp_s": float(state.timestamp_device_s),
        "metadata": dict(metadata or {}),
        "large_avalanche": {
            "persistence_s": float(getattr(bridge, "_persistence_s", 0.0)),
            "has_previous": bool(getattr(bridge, "_has_previous", False)),
        },
        "minislope": {
            "active_tiles": [int(t) for t in frontier_active_tiles],
            "iterations": int(frontier_iterations),
            "pending": bool(relaxation_pending),
        },
        "dirty_tiles": [],
        "terrain_hash_sha256": sha256_array(arrays["b_eff"]),
        "provenance": dict(provenance),
        "precision": state.precision,
    }
    target = Path(path)
    target.parent.mkdir(parents=True, exist_ok=True)
    np.savez_compressed(target, **arrays, checkpoint_record_json=np.asarray(
        json.dumps(record, sort_keys=True, separators=(",", ":"))))
    result = dict(record)
    result["checkpoint_path"] = str(target)
    result["checkpoint_hash_sha256"] = sha256_file(target)
    return result


def restore_device_checkpoint(state, path, *, bridge=None) -> dict:
    """Restore a checkpoint (written here or by the reference) into ``state``."""
    source = Path(path)
    with np.load(source, allow_pickle=False) as archive:
        record = json.loads(str(archive["checkpoint_record_json"]))
        if tuple(record["shape_yx"]) != tuple(state.shape):
            raise RuntimeError("DEVICE_CHECKPOINT_SHAPE_MISMATCH")
        if [float(v) for v in record["resolution_xy_m"]] != [state.grid.dx, state.grid.dy]:
            raise RuntimeError("DEVICE_CHECKPOINT_RESOLUTION_MISMATCH")
        fields = {name: np.asarray(archive[name]).copy()
                  for name in (*FLOAT_FIELDS, *INT_FIELDS) if name in archive.files}
    if "b_eff" not in fields:
        raise RuntimeError("DEVICE_CHECKPOINT_MISSING_STATIC_BED")
    fields.setdefault("z_base", np.zeros_like(fields["b_eff"]))
    fields.setdefault("avalanche_owned_surface",
                      fields["b_eff"] + fields.get("mobile", np.zeros_like(fields["b_eff"])))
    grid = state.grid
    for name, values in fields.items():
        dev = _DEVICE_NAME.get(name)
        if dev is None:
            continue
        grid.upload(dev, values)
    state._timestamp_device_s = float(record["device_timestamp_s"])
    if bridge is not None:
        bridge._persistence_s = float(record["large_avalanche"]["persistence_s"])
        bridge._has_previous = bool(record["large_avalanche"]["has_previous"])
    return record
