"""CPU restatement of the bilinear free-surface query -- TEST INFRASTRUCTURE
(the checker of the GPU sampler, never shipped).

The Warp query kernel (runtime/bulk_state_authority.py:201-228) clamps each
(row, column) query to the grid, then blends the four corner values of
resting + mobile; the reference's CPU sampler (bulk_exchange/airborne.py:
587-600) is the same blend without the clamp.  Pinned to the CPU sampler's
outputs in ``tests/golden/surface.npz`` and to the reference test's known
answers (tests/test_device_bulk_state.py:116-126).
"""

import numpy as np


def bilinear(surface: np.ndarray, rows, cols) -> np.ndarray:
    """Clamped bilinear samples of ``surface`` ([ny, nx] float64)."""
    ny, nx = surface.shape
    row = np.clip(np.asarray(rows, dtype=np.float64), 0.0, ny - 1.0)
    col = np.clip(np.asarray(cols, dtype=np.float64), 0.0, nx - 1.0)
    r0 = np.floor(row).astype(np.int64)
    c0 = np.floor(col).astype(np.int64)
    r1 = np.minimum(r0 + 1, ny - 1)
    c1 = np.minimum(c0 + 1, nx - 1)
    fr, fc = row - r0, col - c0
    return ((1.0 - fr) * (1.0 - fc) * surface[r0, c0] + (1.0 - fr) * fc * surface[r0, c1]
            + fr * (1.0 - fc) * surface[r1, c0] + fr * fc * surface[r1, c1])
