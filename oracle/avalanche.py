"""CPU restatement of large-avalanche activation -- TEST INFRASTRUCTURE.

Restates the reference's device kernels ``mobilize`` and
``reduce_persistence`` (runtime/gpu_large_avalanche.py:308-451) in float64
NumPy, applied to labels / severity / latches read back from the GPU; used
only by the tests as the checker of sb_avalanche_mobilize and
sb_avalanche_persistence.
"""

from __future__ import annotations

import numpy as np

from .deposition import vertex_weights


def mobilize(b, z, h, labels, winner, latch, severity, *, dx, dy, depth, dry, time_s,
             act_count, r2m):
    """Returns (b, h, latch, act_count, r2m, sums) after activating the winner component."""
    b = np.asarray(b, np.float64).copy()
    h = np.asarray(h, np.float64).copy()
    latch = np.asarray(latch).copy()
    act_count = np.asarray(act_count).copy()
    r2m = np.asarray(r2m, np.float64).copy()
    w = vertex_weights(b.shape, dx, dy)
    sel = (np.asarray(labels) == winner) & (latch == 0)
    transfer = np.minimum(np.maximum(b - z, 0.0), depth * severity)
    go = sel & (transfer > dry)
    t = np.where(go, transfer, 0.0)
    b = np.where(go, b - t, b)
    h = np.where(go, h + t, h)
    latch = np.where(go, 1, latch)
    weighted = t * w
    first = go & (act_count == 0)
    again = go & (act_count > 0)
    act_count = np.where(go, act_count + 1, act_count)
    r2m = np.where(go, r2m + weighted, r2m)
    sums = {"transferred": float(weighted.sum()), "new_volume": float(weighted[first].sum()),
            "re_volume": float(weighted[again].sum()), "new_area": float(w[first].sum()),
            "re_area": float(w[again].sum()), "cells": int(go.sum())}
    return b, h, latch, act_count, r2m, sums


def persistence(b0, b, h, qx, qy, slope, unstable, latch, act_count, r2m, m2r, *, dx, dy,
                start_rad, stop_rad, dry, activity_speed, tile_size):
    """The reference's lifecycle sums (reduce_persistence + _persistence_summary)."""
    w = vertex_weights(b.shape, dx, dy)
    wet = h > dry
    safe = np.where(wet, h, 1.0)
    speed = np.where(wet, np.sqrt((qx / safe) ** 2 + (qy / safe) ** 2), 0.0)
    moving = wet & (speed > activity_speed)
    active = np.asarray(unstable, bool) | moving
    ny, nx = b.shape
    rows, cols = np.nonzero(active)
    tiles = np.unique((rows // tile_size) * ((nx + tile_size - 1) // tile_size) + cols // tile_size)
    delta = (b + h) - b0
    act = act_count > 0
    sl = np.where(act, slope, 0.0)
    retired = act & ~wet & (slope <= stop_rad) & (latch == 0)
    return {
        "unique": int(act.sum()), "reactivated": int((act_count > 1).sum()),
        "wet": int(wet.sum()), "retired": int(retired.sum()), "tiles": int(tiles.size),
        "r2m": float(r2m.sum()), "m2r": float(m2r.sum()), "unique_area": float(w[act].sum()),
        "re_area": float(w[act_count > 1].sum()), "mobile_volume": float((h * w)[wet].sum()),
        "max_speed": float(speed.max(initial=0.0)), "net_change": float((delta * w).sum()),
        "net_transfer": float((np.abs(delta) * w * 0.5).sum()), "slope_sum": float(sl.sum()),
        "slope_max": float(sl.max(initial=0.0)),
        "minus_stop": float(np.where(act, slope - stop_rad, 0.0).sum()),
        "start_minus": float(np.where(act, start_rad - slope, 0.0).sum()),
        "retired_area": float(w[retired].sum()), "moving_volume": float((h * w)[moving].sum()),
    }
