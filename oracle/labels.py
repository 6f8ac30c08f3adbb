"""CPU restatement of large-avalanche (FailureZone) labelling -- TEST INFRASTRUCTURE.

* ``yield_init`` follows the device ``initialize`` kernel of
  ``runtime/gpu_large_avalanche.py`` (:58-162): free-surface gradient with
  one-sided differences at the borders, slope angle, cohesive start/stop
  margins over a failure layer ``min(max(b_eff - z_base, 0), depth)``,
  severity, unstable mask and latch release.  ``fixed_point=True`` mirrors the
  production arithmetic bit for bit (integer height differences, the yield in
  float32, the slope angle by Abramowitz & Stegun 4.4.49).
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
        y = _yield_fx32(b, z, h, rows, cols, left, right, down, up, dx=dx, dy=dy,
                        tan_start=tan_start, tan_stop=tan_stop, density=density,
                        gravity=gravity, cohesion=cohesion,
                        mobilization_depth=mobilization_depth, dry=dry, quantum=quantum)
        gx, gy, slope, severity, unstable, stop_margin = y
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
        severity = np.clip(stop_margin / np.maximum(normal * (tan_start - tan_stop), 1.0e-12),
                           0.0, 1.0)
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


_F = np.float32
# Abramowitz & Stegun, Handbook of Mathematical Functions, 4.4.49 (Hastings):
# atan(x) = x (1 + a2 x^2 + ... + a16 x^16) on [0, 1], |error| <= 2e-8.
ATAN_A = (-0.3333314528, 0.1999355085, -0.1420889944, 0.1065626393, -0.0752896400,
          0.0429096138, -0.0161657367, 0.0028662257)


def atan_as4449(x):
    """float32 arc tangent of x >= 0, evaluated as the fixed-point labelling
    kernel does (Horner in float32, separate multiplies and adds; x > 1 via
    pi/2 - atan(1/x)), so the bits agree with the device's."""
    x = np.asarray(x, dtype=_F)
    inv = x > _F(1.0)
    t = np.where(inv, _F(1.0) / np.where(inv, x, _F(1.0)), x).astype(_F)
    t2 = t * t
    p = _F(ATAN_A[-1])
    for a in ATAN_A[-2::-1]:
        p = _F(a) + t2 * p
    p = _F(1.0) + t2 * p
    r = t * p
    return np.where(inv, _F(np.pi / 2) - r, r).astype(_F)


def _yield_fx32(b, z, h, rows, cols, left, right, down, up, *, dx, dy, tan_start, tan_stop,
                density, gravity, cohesion, mobilization_depth, dry, quantum):
    """The fixed-point labelling kernel's yield in float32: integer free-surface
    differences, each constant one rounding of its double expression, the same
    operation order as the device (no fused multiply-adds)."""
    H = np.asarray(b, dtype=np.int64) + np.asarray(h, dtype=np.int64)
    inx = (cols > 0) & (cols + 1 < np.shape(b)[1])
    iny = (rows > 0) & (rows + 1 < np.shape(b)[0])
    sx = np.where(inx, _F(quantum / (2.0 * dx)), _F(quantum / dx)).astype(_F)
    sy = np.where(iny, _F(quantum / (2.0 * dy)), _F(quantum / dy)).astype(_F)
    gx = (H[rows, right] - H[rows, left]).astype(_F) * sx
    gy = (H[up, cols] - H[down, cols]).astype(_F) * sy
    mag = np.sqrt(gx * gx + gy * gy)
    depth_q = np.maximum(np.asarray(b, np.int64) - np.asarray(z, np.int64), 0)
    layer = np.minimum(depth_q.astype(_F) * _F(quantum), _F(mobilization_depth))
    norm = np.sqrt(_F(1.0) + mag * mag)
    rg = _F(density * gravity)
    drive = rg * layer * mag / norm
    normal = rg * layer / norm
    start_margin = drive - (_F(cohesion) + normal * _F(tan_start))
    stop_margin = drive - (_F(cohesion) + normal * _F(tan_stop))
    severity = np.minimum(np.maximum(
        stop_margin / np.maximum(normal * _F(tan_start - tan_stop), _F(1.0e-12)), _F(0.0)),
        _F(1.0))
    unstable = (layer > _F(dry)) & (start_margin > _F(0.0))
    return gx, gy, atan_as4449(mag), severity, unstable, stop_margin


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
