"""CPU restatement of the learned repose proposal -- TEST INFRASTRUCTURE.

Only the tests use this module: it is the checker of the tensor-core
convolution kernels and of the training gradients, never part of the product
path.  The learned proposal has no counterpart in the reference (its repose
relaxation is the plain sweep of slope_model.py:273-343 alone), so this module
states the network's own specification in float64 NumPy:

* ``conv3x3``: O[y, x, co] = sum_{dy, dx, ci} I[y+dy-1, x+dx-1, ci] W[dy, dx, ci, co]
  with zero padding (cross-correlation, no bias).
* ``features``: per edge k of cell (r, c) -- east (r, c+1), north (r+1, c),
  north-east (r+1, c+1), north-west (r+1, c-1) -- the height drop
  (H[c] - H[n_k]) / (L_k tan_crit), 0 where the edge leaves the grid.
* ``divergence``: height change of fluxes F (transfer F * tan_crit * dx along
  each edge): dH[c] = -sum_k t_k(c) + sum_k t_k(c - d_k).
* ``forward`` / ``loss_and_grads``: the 4-layer net (ReLU between layers),
  mean squared error of dH against a target change, and its gradients by
  hand-written back-propagation.
"""

from __future__ import annotations

import numpy as np

EDGES = ((0, 1), (1, 0), (1, 1), (1, -1))  # (dr, dc) of east, north, north-east, north-west


def conv3x3(x: np.ndarray, w: np.ndarray) -> np.ndarray:
    """x [B, H, W, Ci], w [3, 3, Ci, Co] -> [B, H, W, Co] (float64)."""
    b, h, wd, _ = x.shape
    xp = np.zeros((b, h + 2, wd + 2, x.shape[3]))
    xp[:, 1:-1, 1:-1] = x
    out = np.zeros((b, h, wd, w.shape[3]))
    for dy in range(3):
        for dx in range(3):
            out += np.einsum("bhwc,cd->bhwd", xp[:, dy:dy + h, dx:dx + wd], w[dy, dx])
    return out


def conv3x3_wgrad(x: np.ndarray, g: np.ndarray) -> np.ndarray:
    """dW[dy, dx, ci, co] = sum I[y+dy-1, x+dx-1, ci] G[y, x, co]."""
    b, h, wd, ci = x.shape
    xp = np.zeros((b, h + 2, wd + 2, ci))
    xp[:, 1:-1, 1:-1] = x
    dw = np.zeros((3, 3, ci, g.shape[3]))
    for dy in range(3):
        for dx in range(3):
            dw[dy, dx] = np.einsum("bhwc,bhwd->cd", xp[:, dy:dy + h, dx:dx + wd], g)
    return dw


def flip_transpose(w: np.ndarray) -> np.ndarray:
    """Weights of the data gradient: W'[dy, dx, co, ci] = W[2-dy, 2-dx, ci, co]."""
    return np.ascontiguousarray(w[::-1, ::-1].transpose(0, 1, 3, 2))


def features(height: np.ndarray, dx: float, dy: float, tan_crit: float) -> np.ndarray:
    """height [B, H, W] -> [B, H, W, 4]."""
    b, h, wd = height.shape
    out = np.zeros((b, h, wd, 4))
    diag = np.sqrt(dx * dx + dy * dy)
    for k, (dr, dc) in enumerate(EDGES):
        L = dx if k == 0 else (dy if k == 1 else diag)
        r0, r1 = 0, h - dr
        c0, c1 = max(0, -dc), wd - max(0, dc)
        out[:, r0:r1, c0:c1, k] = (height[:, r0:r1, c0:c1]
                                   - height[:, r0 + dr:r1 + dr, c0 + dc:c1 + dc]) / (L * tan_crit)
    return out


def divergence(flux: np.ndarray, scale: float) -> np.ndarray:
    """flux [B, H, W, >=4] -> dH [B, H, W]; transfers flux * scale, inside the grid only."""
    b, h, wd = flux.shape[:3]
    dh = np.zeros((b, h, wd))
    for k, (dr, dc) in enumerate(EDGES):
        r1 = h - dr
        c0, c1 = max(0, -dc), wd - max(0, dc)
        t = flux[:, 0:r1, c0:c1, k] * scale
        dh[:, 0:r1, c0:c1] -= t
        dh[:, dr:r1 + dr, c0 + dc:c1 + dc] += t
    return dh


def forward(x: np.ndarray, weights):
    """Activations [x, a0, a1, a2] and the output fluxes."""
    acts = [x]
    a = x
    for i, w in enumerate(weights):
        z = conv3x3(a, w)
        a = z if i == len(weights) - 1 else np.maximum(z, 0.0)
        acts.append(a)
    return acts[:-1], acts[-1]


def loss_and_grads(x, weights, target_dh, scale: float, norm: float):
    """Loss = sum((dH - target)^2) * norm; returns (loss, [dW per layer], dflux)."""
    acts, flux = forward(x, weights)
    e = divergence(flux, scale) - target_dh
    loss = float(np.sum(e * e) * norm)
    # d loss / d flux[c, k] = 2 norm scale (e[n_k] - e[c]) for edges inside the grid
    dflux = np.zeros_like(flux)
    b, h, wd = e.shape
    for k, (dr, dc) in enumerate(EDGES):
        r1 = h - dr
        c0, c1 = max(0, -dc), wd - max(0, dc)
        dflux[:, 0:r1, c0:c1, k] = 2.0 * norm * scale * (
            e[:, dr:r1 + dr, c0 + dc:c1 + dc] - e[:, 0:r1, c0:c1])
    grads = [None] * len(weights)
    g = dflux
    for i in range(len(weights) - 1, -1, -1):
        grads[i] = conv3x3_wgrad(acts[i], g)
        if i > 0:
            g = conv3x3(g, flip_transpose(weights[i])) * (acts[i] > 0)
    return loss, grads, dflux
