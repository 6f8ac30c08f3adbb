"""CPU restatement of the device deposition step -- TEST INFRASTRUCTURE.

Follows the reference's device kernel ``deposit`` and ``weighted_sum``
(bulk_interaction/warp_deposition.py:23-130) with every cell reading the
pre-step state (the device kernel reads neighbours while they are being
written; the free surface it reads is unchanged by deposition up to that
race).  Used only by the tests as the checker of ``sb_deposition_step``; it
is pinned against the reference's CPU ``DepositionOperator.apply``
(bulk_interaction/deposition.py:67-160) on the fixtures of
tests/golden/deposition.npz, where both give the same result.
"""

from __future__ import annotations

import numpy as np


def vertex_weights(shape, dx: float, dy: float) -> np.ndarray:
    """Triangle-A-C vertex weights (runtime/bulk_state_authority.py:612-634) in m^2."""
    from .relax import vertex_weights6
    return vertex_weights6(shape).astype(np.float64) * (dx * dy / 6.0)


def step(b, h, qx, qy, *, dx, dy, dt, density, cohesion, stop_angle_deg, settle_tail=False,
         forcing=None, rate=0.30, threshold=0.18, gravity=9.81):
    """One deposition step in float64; returns (b, h, qx, qy, volume, momentum_x, momentum_y)."""
    b = np.asarray(b, np.float64).copy()
    h = np.asarray(h, np.float64).copy()
    qx = np.asarray(qx, np.float64).copy()
    qy = np.asarray(qy, np.float64).copy()
    ny, nx = h.shape
    w = vertex_weights(h.shape, dx, dy)
    forced = np.zeros(h.shape, bool) if forcing is None else np.asarray(forcing, bool)
    candidate = (h > 0.0) & ~forced
    amount = np.zeros_like(h)
    if settle_tail:
        amount = np.where(candidate, h, 0.0)
    else:
        safe = np.where(candidate, h, 1.0)
        vx = qx / safe
        vy = qy / safe
        slow = ~(np.sqrt(vx * vx + vy * vy) > threshold)
        rows, cols = np.indices(h.shape)
        left = np.where(cols > 0, cols - 1, cols)
        right = np.where(cols + 1 < nx, cols + 1, cols)
        down = np.where(rows > 0, rows - 1, rows)
        up = np.where(rows + 1 < ny, rows + 1, rows)
        hx = np.where((cols == 0) | (cols + 1 == nx), dx, 2.0 * dx)
        hy = np.where((rows == 0) | (rows + 1 == ny), dy, 2.0 * dy)
        sx = (((b[rows, right] + h[rows, right]) - b[rows, left]) - h[rows, left]) / hx
        sy = (((b[up, cols] + h[up, cols]) - b[down, cols]) - h[down, cols]) / hy
        t = np.sqrt(sx * sx + sy * sy)
        norm = np.sqrt(1.0 + t * t)
        drive = density * gravity * h * t / norm
        resist = cohesion + density * gravity * h * np.tan(np.deg2rad(stop_angle_deg)) / norm
        settle = candidate & slow & ~(drive > resist)
        amount = np.where(settle, np.minimum(h, rate * dt), 0.0)
    moved = amount != 0.0
    safe = np.where(moved, h, 1.0)
    if settle_tail:
        rx = np.where(moved, qx, 0.0)
        ry = np.where(moved, qy, 0.0)
        b = np.where(moved, b + h, b)
        qx = np.where(moved, 0.0, qx)
        qy = np.where(moved, 0.0, qy)
        h = np.where(moved, 0.0, h)
    else:
        frac_removed = amount / safe
        rx = np.where(moved, qx * frac_removed, 0.0)
        ry = np.where(moved, qy * frac_removed, 0.0)
        b = np.where(moved, b + amount, b)
        fraction = (safe - amount) / safe
        h = np.where(moved, h - amount, h)
        qx = np.where(moved, qx * fraction, qx)
        qy = np.where(moved, qy * fraction, qy)
    volume = float(np.sum(amount * w))
    return b, h, qx, qy, volume, float(np.sum(density * rx * w)), float(np.sum(density * ry * w))
