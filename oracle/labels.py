"""CPU restatement of large-avalanche (FailureZone) labelling -- TEST INFRASTRUCTURE.

* ``yield_init`` follows the device ``initialize`` kernel of
  ``runtime/gpu_large_avalanche.py`` (:58-162): free-surface gradient with
  one-sided differences at the borders, slope angle, cohesive start/stop
  margins over a failure layer ``min(max(b_eff - z_base, 0), depth)``,
  severity, unstable mask and latch release.  ``fixed_point=True`` mirrors the
  production arithmetic (integer height differences, exact).
* ``canonical_labels`` gives every connected unstable cell the minimum flat
  index of its component -- the converged state of the device union-find
  (:27-56, :164-198), where roots only ever hook to smaller roots.  Computed
  here with ``scipy.ndimage.label`` (third-party, SciPy 1.18 in this image)
  followed by a per-component minimum.
* ``component_summary`` restates ``aggregate_components`` /
  ``reduce_components`` / ``select_winner`` / ``winner_diagnostics``
  (:200-275): region count, largest count, winner = smallest root among the
  largest components, area/volume/excess of the winner.
"""

from __future__ import annotations

import numpy as np
from scipy import ndimage


def gradient_device_order(free_l, free_r, denom):
    return (free_r - free_l) / denom


def yield_init(b, z, h, qx, qy, *, dx, dy, tan_start, tan_stop, density, gravity, cohesion,
               mobilization_depth, dry, activity_speed=0.05, fixed_point=False, quantum=1.0,
               latch=None, owned_export_baseline=None, export_cumulative=None, weights=None,
               release_settled_latches=True):
    """Returns dict(gx, gy, slope, severity, unstable, latch)."""
    ny, nx = np.shape(b)
    rows, cols = np.indices((ny, nx))
    left = np.where(cols > 0, cols - 1, cols)
    right = np.where(cols + 1 < nx, cols + 1, cols)
    down = np.where(rows > 0, rows - 1, rows)
    up = np.where(rows + 1 < ny, rows + 1, rows)
    denx = np.where((cols > 0) & (cols + 1 < nx), 2.0 * dx, dx)
    deny = np.where((rows > 0) & (rows + 1 < ny), 2.0 * dy, dy)
    if fixed_point:
        H = np.asarray(b, dtype=np.int64) + np.asarray(h, dtype=np.int64)
        gx = ((H[rows, right] - H[rows, left]).astype(np.float64) * quantum) / denx
        gy = ((H[up, cols] - H[down, cols]).astype(np.float64) * quantum) / deny
        depth_q = np.maximum(np.asarray(b, np.int64) - np.asarray(z, np.int64), 0)
        layer = np.minimum(depth_q.astype(np.float64) * quantum, mobilization_depth)
        mob = np.asarray(h, np.float64) * quantum
    else:
        b = np.asarray(b, np.float64)
        h = np.asarray(h, np.float64)
        # device order: ((r[R] + m[R]) - r[L]) - m[L]
        gx = (((b[rows, right] + h[rows, right]) - b[rows, left]) - h[rows, left]) / denx
        gy = (((b[up, cols] + h[up, cols]) - b[down, cols]) - h[down, cols]) / deny
        layer = np.minimum(np.maximum(b - np.asarray(z, np.float64), 0.0), mobilization_depth)
        mob = h
    mag = np.sqrt(gx * gx + gy * gy)
    slope = np.arctan(mag)
    norm = np.sqrt(1.0 + mag * mag)
    drive = density * gravity * layer * mag / norm
    normal = density * gravity * layer / norm
    start_margin = drive - (cohesion + normal * tan_start)
    stop_margin = drive - (cohesion + normal * tan_stop)
    severity = np.clip(stop_margin / np.maximum(normal * (tan_start - tan_stop), 1.0e-12), 0.0, 1.0)
    unstable = (layer > dry) & (start_margin > 0.0)
    out_latch = None
    if latch is not None:
        qx = np.asarray(qx, np.float64)
        qy = np.asarray(qy, np.float64)
        wet = mob > dry
        vx = np.divide(qx, mob, out=np.zeros_like(mob), where=wet)
        vy = np.divide(qy, mob, out=np.zeros_like(mob), where=wet)
        speed = np.where(wet, np.sqrt(vx * vx + vy * vy), 0.0)
        exported = np.asarray(export_cumulative) - np.asarray(owned_export_baseline)
        resolved = exported > dry * np.asarray(weights)
        release = (bool(release_settled_latches) & (speed <= activity_speed)
                   & (resolved | (stop_margin <= 0.0)))
        out_latch = np.where(release, 0, np.asarray(latch)).astype(np.int32)
    return {"gx": gx, "gy": gy, "slope": slope, "severity": severity,
            "unstable": unstable, "latch": out_latch, "stop_margin": stop_margin}


def canonical_labels(mask: np.ndarray, connectivity: int) -> np.ndarray:
    """-1 outside the mask, else the minimum flat index of the cell's component."""
    mask = np.asarray(mask, dtype=bool)
    structure = (np.ones((3, 3), dtype=bool) if connectivity == 8
                 else ndimage.generate_binary_structure(2, 1))
    lab, n = ndimage.label(mask, structure=structure)
    out = np.full(mask.shape, -1, dtype=np.int64)
    if n == 0:
        return out.astype(np.int32)
    flat = np.arange(mask.size, dtype=np.int64).reshape(mask.shape)
    mins = ndimage.minimum(flat, labels=lab, index=np.arange(1, n + 1))
    lut = np.concatenate(([-1], np.asarray(mins, dtype=np.int64)))
    out = lut[lab]
    return out.astype(np.int32)


def component_summary(labels: np.ndarray):
    """(region_count, largest_count, winner_root, total_unstable)."""
    lab = np.asarray(labels).ravel()
    on = lab >= 0
    if not np.any(on):
        return 0, 0, -1, 0
    roots, counts = np.unique(lab[on], return_counts=True)
    largest = int(counts.max())
    winner = int(roots[counts == largest].min())
    return int(roots.size), largest, winner, int(on.sum())
