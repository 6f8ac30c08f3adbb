"""CPU restatement of the reference's repose relaxations -- TEST INFRASTRUCTURE.

Two schedules, both on a generic 2-D array whose axis 0 uses spacing s0 and
axis 1 spacing s1 (the reference's ``relax_critical_slope(height,
grid_spacing)`` convention, ``slope_model.py:273-343``):

* ``relax_critical_slope`` -- full domain.  Per iteration, for each neighbour
  direction of ``_neighbor_pairs`` (:744-750) and each parity (axis-0
  coordinate if the direction steps axis 0, else axis-1 coordinate), every
  pair of the active parity moves half its excess over ``tan(angle)*L``
  (Jacobi inside a sub-phase, Gauss-Seidel across the 8 sub-phases).  The
  iteration's max excess is taken over *all* pairs of each sub-phase before
  its update; convergence when it is <= tolerance.
* ``reached_relax`` -- the event-driven reached-bbox backend: the same
  sub-phase schedule gated by a growing reached mask, with a confirming scan
  before it stops (``solvers/event_driven_slope.py:166-302``).
* ``frontier_relax`` -- the production compact-frontier round schedule
  (``runtime/v2_physics_core.py:1172-1254`` over
  ``solvers/warp_compact_frontier.py:56-130`` and the edge ownership of
  ``solvers/sparse_tile_slope.py:167-220``): edges owned by active tiles (tile
  of endpoint ``a``), reached-gated weighted transfers, 3x3-cell tile
  activation around moved endpoints (:28-54), phase tiles growing within a
  round, a final scan whose unstable owner tiles become the next round's
  active set; ``reached`` is cleared when the frontier empties.

``fixed_point=True`` variants mirror the production int32-quanta arithmetic
(transfers rounded up to whole weight-compatible quanta so the pair ends at or
below critical, exact conservation of sum(w*h)).
"""

from __future__ import annotations

import math

import numpy as np


def neighbor_pairs(s0: float, s1: float):
    """(d0, d1, distance) -- slope_model._neighbor_pairs (:744-750)."""
    diag = float(np.hypot(s0, s1))
    return [(1, 0, float(s0)), (0, 1, float(s1)), (1, 1, diag), (1, -1, diag)]


def paired_views(h: np.ndarray, d0: int, d1: int):
    """slope_model._paired_views (:753-764)."""
    if (d0, d1) == (1, 0):
        return h[:-1, :], h[1:, :]
    if (d0, d1) == (0, 1):
        return h[:, :-1], h[:, 1:]
    if (d0, d1) == (1, 1):
        return h[:-1, :-1], h[1:, 1:]
    if (d0, d1) == (1, -1):
        return h[:-1, 1:], h[1:, :-1]
    raise ValueError("unsupported neighbour offset")


def max_neighbor_slope(h: np.ndarray, spacing) -> float:
    m = 0.0
    for d0, d1, dist in neighbor_pairs(*spacing):
        a, b = paired_views(h, d0, d1)
        m = max(m, float(np.max(np.abs(a - b) / dist)))
    return m


def relax_critical_slope(height, grid_spacing, critical_angle_deg=34.0, max_iterations=20000,
                         tolerance=1e-8):
    """Returns (h, iterations, converged, volume_before, volume_after)."""
    height = np.asarray(height)
    if height.ndim != 2 or min(height.shape) < 2:
        raise ValueError("height must be a 2-D array with both dimensions >= 2")
    if np.any(height < 0):
        raise ValueError("soil heights must be non-negative")
    if not 0.0 < critical_angle_deg < 90.0:
        raise ValueError("critical_angle_deg must be between 0 and 90")
    h = np.asarray(height, dtype=float).copy()
    s0, s1 = grid_spacing
    if s0 <= 0 or s1 <= 0:
        raise ValueError("grid spacing must be positive")
    area = s0 * s1
    vol0 = float(h.sum() * area)
    crit = float(np.tan(np.deg2rad(critical_angle_deg)))
    phases = []
    for d0, d1, dist in neighbor_pairs(s0, s1):
        a, _ = paired_views(h, d0, d1)
        coord = (np.arange(a.shape[0])[:, None] if d0 else np.arange(a.shape[1])[None, :])
        even = (coord & 1) == 0
        phases.append((d0, d1, dist, (even, ~even)))
    converged = False
    it = 0
    for it in range(1, max_iterations + 1):
        worst = 0.0
        for d0, d1, dist, masks in phases:
            for active in masks:
                a, b = paired_views(h, d0, d1)
                diff = a - b
                excess = np.maximum(np.abs(diff) - crit * dist, 0)
                t = 0.5 * excess * np.sign(diff)
                t *= active
                a -= t
                b += t
                worst = max(worst, float(excess.max(initial=0.0)))
        if worst <= tolerance:
            converged = True
            break
    return h, it, converged, vol0, float(h.sum() * area)


def relax_critical_slope_fixed(hq, grid_spacing, crit_tan: float, quantum: float,
                               max_iterations=20000, tolerance=1e-8):
    """Fixed-point mirror of the production full-domain kernel.

    Heights are integer quanta; each active pair with excess e > 0 (in quanta)
    moves ceil(e/2) quanta, so the pair ends at or below critical; the
    convergence max is taken in quanta.  Returns (hq, iterations, converged).
    """
    h = np.asarray(hq, dtype=np.int64).copy()
    s0, s1 = grid_spacing
    pairs = neighbor_pairs(s0, s1)
    crit_q = [(crit_tan * dist) / quantum for _, _, dist in pairs]
    tol_q = tolerance / quantum
    it = 0
    converged = False
    for it in range(1, max_iterations + 1):
        worst = 0.0
        for d, (d0, d1, _) in enumerate(pairs):
            a, b = paired_views(h, d0, d1)
            coord = (np.arange(a.shape[0])[:, None] if d0 else np.arange(a.shape[1])[None, :])
            for par in (0, 1):
                a, b = paired_views(h, d0, d1)
                diff = a - b
                ex = np.abs(diff).astype(np.float64) - crit_q[d]
                worst = max(worst, float(ex.max(initial=0.0)))
                active = ((coord & 1) == par) & (ex > 0.0)
                t = np.where(active, np.ceil(ex * 0.5), 0.0).astype(np.int64)
                st = np.where(diff < 0, -t, t)
                a -= st
                b += st
        if worst <= tol_q:
            converged = True
            break
    return h, it, converged


# ---------------------------------------------------------------------------
# Reached-gated sweep (event-driven reached-bbox backend)
# ---------------------------------------------------------------------------
def reached_relax(height, seeds, spacing, crit_tan: float, tolerance: float,
                  max_iterations: int = 1_000_000):
    """``EventDrivenMinimumSlopeAdapter._relax_dynamic_frontier``
    (solvers/event_driven_slope.py:166-302), closed boundary, on a generic
    [axis 0, axis 1] array (the reference's H[x, y]).

    The reference crops every sub-phase to the reached-tile envelope plus one
    cell; every edge with a reached endpoint lies inside that window, so the
    crop only saves work and is left out here.  Per iteration and sub-phase
    (direction, parity): excess = max(|a - b| - crit * L, 0) over all pairs;
    the iteration maximum takes the reachable pairs (a or b reached) before
    the sub-phase's update; pairs of the active parity that are reachable move
    half their excess (0.5 * excess * sign(a - b)) and both endpoints of a
    moved pair become reached.  When the iteration's maximum is <= tolerance
    the post-iteration state is scanned once more (all reachable pairs) and
    the solve ends if that is <= tolerance too.  Returns (h, reached,
    iterations).
    """
    h = np.array(height, dtype=np.float64, copy=True)
    reached = np.array(seeds, dtype=bool, copy=True)
    pairs = neighbor_pairs(*spacing)
    iterations = 0
    while True:
        iterations += 1
        if iterations > max_iterations:
            raise RuntimeError("NUMERICAL_NONCONVERGENCE: reached-bbox MiniSlope exceeded the "
                               "numerical safety limit")
        worst = 0.0
        for d0, d1, dist in pairs:
            crit = crit_tan * dist
            for parity in (0, 1):
                a, b = paired_views(h, d0, d1)
                ra, rb = paired_views(reached, d0, d1)
                diff = a - b
                excess = np.maximum(np.abs(diff) - crit, 0.0)
                reach = ra | rb
                if np.any(reach):
                    worst = max(worst, float(excess[reach].max()))
                if d0:
                    coord = np.arange(a.shape[0])[:, None]
                else:
                    coord = np.arange(a.shape[1])[None, :]
                go = ((coord & 1) == parity) & reach & (excess > 0.0)
                t = np.where(go, 0.5 * excess * np.sign(diff), 0.0)
                a -= t
                b += t
                ra |= go
                rb |= go
        if worst <= tolerance:
            remaining = 0.0
            for d0, d1, dist in pairs:
                a, b = paired_views(h, d0, d1)
                ra, rb = paired_views(reached, d0, d1)
                reach = ra | rb
                if np.any(reach):
                    remaining = max(remaining,
                                    float((np.abs(a - b) - crit_tan * dist)[reach].max()))
            if remaining <= tolerance:
                return h, reached, iterations


# ---------------------------------------------------------------------------
# Compact frontier (production schedule)
# ---------------------------------------------------------------------------
def vertex_weights(shape, s0: float, s1: float) -> np.ndarray:
    """Triangle-A-C vertex weights (runtime/bulk_state_authority.py:612-621)."""
    w = np.zeros(shape, dtype=np.float64)
    f = s0 * s1 / 6.0
    w[:-1, :-1] += 2.0 * f
    w[:-1, 1:] += f
    w[1:, 1:] += 2.0 * f
    w[1:, :-1] += f
    return w


def vertex_weights6(shape) -> np.ndarray:
    """Same weights in integer units of s0*s1/6."""
    w = np.zeros(shape, dtype=np.int64)
    w[:-1, :-1] += 2
    w[:-1, 1:] += 1
    w[1:, 1:] += 2
    w[1:, :-1] += 1
    return w


def tile_ids_of(i, j, tile: int, tiles1: int):
    return (np.asarray(i) // tile) * tiles1 + np.asarray(j) // tile


def tiles_around(i, j, shape, tile: int) -> np.ndarray:
    """3x3-cell stencil tile activation (sparse_tile_slope.py:138-165)."""
    i = np.asarray(i, dtype=np.int64).ravel()
    j = np.asarray(j, dtype=np.int64).ravel()
    if i.size == 0:
        return np.empty(0, dtype=np.int32)
    tiles1 = (shape[1] + tile - 1) // tile
    out = []
    for oi in (-1, 0, 1):
        for oj in (-1, 0, 1):
            ci, cj = i + oi, j + oj
            ok = (ci >= 0) & (ci < shape[0]) & (cj >= 0) & (cj < shape[1])
            out.append(tile_ids_of(ci[ok], cj[ok], tile, tiles1))
    return np.unique(np.concatenate(out)).astype(np.int32)


def owned_edges(tiles: np.ndarray, shape, tile: int, d0: int, d1: int, parity: int):
    """Edges (a, b=a+(d0,d1)) whose a lies in one of ``tiles`` (edge_batch :167-220)."""
    tiles = np.unique(np.asarray(tiles, dtype=np.int64))
    if tiles.size == 0:
        e = np.empty(0, dtype=np.int64)
        return e, e, e, e, e
    tiles1 = (shape[1] + tile - 1) // tile
    li, lj = np.indices((tile, tile))
    li, lj = li.ravel(), lj.ravel()
    tr, tc = tiles // tiles1, tiles % tiles1
    ai = (tr[:, None] * tile + li[None, :]).ravel()
    aj = (tc[:, None] * tile + lj[None, :]).ravel()
    own = np.repeat(tiles, li.size)
    bi, bj = ai + d0, aj + d1
    coord = ai if d0 else aj
    ok = ((ai < shape[0]) & (aj < shape[1]) & (bi >= 0) & (bi < shape[0]) & (bj >= 0)
          & (bj < shape[1]) & ((coord & 1) == parity))
    return own[ok], ai[ok], aj[ok], bi[ok], bj[ok]


def _transfer_fp64(ha, hb, wa, wb, excess, diff):
    signed = np.where(diff < 0.0, -excess, excess)
    wsum = wa + wb
    return signed * wb / wsum, signed * wa / wsum


def frontier_relax(h, reached, active_tiles, *, tile: int, spacing, crit_tan: float,
                   tolerance: float, weights=None, max_rounds: int = 4096,
                   fixed_point: bool = False, quantum: float | None = None,
                   record: bool = False):
    """Run frontier rounds until no active tile remains.

    ``h`` is float64 (or int64 quanta when ``fixed_point``); ``weights`` are
    float64 vertex weights (``fixed_point``: integer weights, e.g. units of
    s0*s1/6).  Returns (h, reached, rounds, history) where history holds the
    per-round active/phase/unstable tile lists when ``record``.
    """
    h = np.array(h, copy=True)
    reached = np.array(reached, dtype=bool, copy=True)
    shape = h.shape
    active = np.unique(np.asarray(active_tiles, dtype=np.int32))
    pairs = neighbor_pairs(*spacing)
    if weights is None:
        weights = np.ones(shape, dtype=np.int64 if fixed_point else np.float64)
    history = []
    rounds = 0
    while active.size:
        rounds += 1
        if rounds > max_rounds:
            raise RuntimeError("NUMERICAL_NONCONVERGENCE: frontier round limit exceeded")
        phase = active
        rec = {"active": active.copy(), "moved": []}
        for d0, d1, dist in pairs:
            crit = crit_tan * dist
            for parity in (0, 1):
                _, ai, aj, bi, bj = owned_edges(phase, shape, tile, d0, d1, parity)
                if ai.size == 0:
                    rec["moved"].append(0)
                    continue
                reach = reached[ai, aj] | reached[bi, bj]
                ha, hb = h[ai, aj], h[bi, bj]
                wa, wb = weights[ai, aj], weights[bi, bj]
                if fixed_point:
                    diff = ha.astype(np.int64) - hb.astype(np.int64)
                    crit_q = crit / quantum
                    exq = np.abs(diff).astype(np.float64) - crit_q
                    moved = reach & (exq > 0.0)
                    g = np.gcd(wa, wb)
                    ua, ub = wb // g, wa // g
                    k = np.ceil(exq / (ua + ub)).astype(np.int64)
                    sgn = np.where(diff < 0, -1, 1)
                    ta = np.where(moved, sgn * k * ua, 0)
                    tb = np.where(moved, sgn * k * ub, 0)
                else:
                    diff = ha - hb
                    excess = np.abs(diff) - crit
                    moved = reach & (excess > 0.0)
                    ta, tb = _transfer_fp64(ha, hb, wa, wb, excess, diff)
                    ta = np.where(moved, ta, 0.0)
                    tb = np.where(moved, tb, 0.0)
                rec["moved"].append(int(np.count_nonzero(moved)))
                if not np.any(moved):
                    continue
                mi, mj, ni, nj = ai[moved], aj[moved], bi[moved], bj[moved]
                h[mi, mj] = h[mi, mj] - ta[moved]
                h[ni, nj] = h[ni, nj] + tb[moved]
                reached[mi, mj] = True
                reached[ni, nj] = True
                trig = tiles_around(np.concatenate((mi, ni)), np.concatenate((mj, nj)), shape, tile)
                phase = np.union1d(phase, trig).astype(np.int32)
        rec["phase"] = phase.copy()
        owners = []
        for d0, d1, dist in pairs:
            crit = crit_tan * dist
            for parity in (0, 1):
                own, ai, aj, bi, bj = owned_edges(phase, shape, tile, d0, d1, parity)
                if ai.size == 0:
                    continue
                reach = reached[ai, aj] | reached[bi, bj]
                if fixed_point:
                    exq = (np.abs(h[ai, aj].astype(np.int64) - h[bi, bj].astype(np.int64))
                           .astype(np.float64) - crit / quantum)
                    bad = reach & (exq > tolerance / quantum)
                else:
                    bad = reach & ((np.abs(h[ai, aj] - h[bi, bj]) - crit) > tolerance)
                if np.any(bad):
                    owners.append(own[bad])
        active = (np.unique(np.concatenate(owners)).astype(np.int32) if owners
                  else np.empty(0, dtype=np.int32))
        rec["unstable"] = active.copy()
        if record:
            history.append(rec)
        if active.size == 0:
            reached[:] = False
    return h, reached, rounds, history


def seed_tiles(seed_mask: np.ndarray, tile: int) -> np.ndarray:
    i, j = np.nonzero(seed_mask)
    return tiles_around(i, j, seed_mask.shape, tile)


def critical_quanta_ok(crit_tan: float, spacing, quantum: float) -> bool:
    """The fixed-point transfer rule needs crit*L >= 8 quanta (see module doc)."""
    return crit_tan * min(spacing) / quantum >= 8.0 and math.isfinite(crit_tan)
