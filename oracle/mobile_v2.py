"""FP64 NumPy restatement of the reference Mobile V2 finite-volume step.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

Follows ``src/isaac_bulk_pipeline/experimental/mobile_v2_reference.py`` of the
reference project:

* configuration defaults/validation  -> ``MobileV2Config`` (:16-38)
* substep loop, CFL, positivity, dry zeroing, external source, Coulomb
  friction                            -> ``MobileV2ReferenceSolver.step`` (:191-314)
* static short-circuit                -> ``_globally_static_below_start`` (:353-363)
* hydrostatic reconstruction + Rusanov face update
                                      -> ``_face_updates`` (:365-431)
* physical flux                       -> ``_physical_flux`` (:433-449)
* ledger/energy terms                 -> ``mass/momentum/energy_terms`` (:104-127)
* result accounting                   -> ``_result`` (:316-351)

Every floating-point operation is evaluated in the same order as the
reference so that element-wise results are bit-identical; only the scalar
diagnostics built from ``np.sum`` depend on summation order.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class OracleConfig:
    """Same keys and defaults as the reference ``MobileV2Config`` (:16-27)."""

    dx_m: float = 0.05
    dy_m: float = 0.05
    gravity_m_s2: float = 9.81
    earth_pressure_coefficient: float = 0.45
    cfl: float = 0.18
    dry_tolerance_m: float = 1.0e-10
    start_angle_deg: float = 34.0
    stop_angle_deg: float = 30.0
    basal_friction_coefficient: float = 0.55
    maximum_substeps: int = 4096


@dataclass
class OracleStep:
    b: np.ndarray
    h: np.ndarray
    q: np.ndarray
    dt_s: float
    substeps: int
    maximum_cfl: float
    mass_before: float
    mass_after: float
    momentum_before: np.ndarray
    momentum_after: np.ndarray
    conservative_impulse: np.ndarray
    friction_impulse: np.ndarray
    external_impulse: np.ndarray
    energy_before: tuple
    energy_after: tuple
    friction_dissipation: float
    external_work: float
    minimum_h: float
    substep_dts: list = field(default_factory=list)

    @property
    def energy_residual(self) -> float:
        return (self.energy_after[3] - self.energy_before[3]
                - self.external_work + self.friction_dissipation)

    @property
    def momentum_residual(self) -> np.ndarray:
        return (self.momentum_after - self.momentum_before
                - (self.conservative_impulse + self.friction_impulse
                   + self.external_impulse))


def _safe_div(num: np.ndarray, den: np.ndarray, wet: np.ndarray) -> np.ndarray:
    """num/den where ``wet`` else 0 (the reference's ``np.divide(where=)``)."""
    out = np.zeros(np.broadcast(num, den).shape, dtype=np.float64)
    np.divide(num, den, out=out, where=wet)
    return out


def mass(cfg: OracleConfig, h: np.ndarray) -> float:
    # reference :104-105
    return float(np.sum(h, dtype=np.float64) * cfg.dx_m * cfg.dy_m)


def momentum(cfg: OracleConfig, q: np.ndarray) -> np.ndarray:
    # reference :107-108
    return np.sum(q, axis=(0, 1), dtype=np.float64) * cfg.dx_m * cfg.dy_m


def energy_terms(cfg: OracleConfig, b: np.ndarray, h: np.ndarray, q: np.ndarray):
    """(kinetic, gravitational, internal, total) per unit density (:110-127)."""
    area = cfg.dx_m * cfg.dy_m
    wet = h > cfg.dry_tolerance_m
    speed2 = _safe_div(np.sum(q * q, axis=-1), h * h, wet)
    kinetic = float(0.5 * np.sum(h * speed2, dtype=np.float64) * area)
    grav = float(cfg.gravity_m_s2 * np.sum(h * b, dtype=np.float64) * area)
    internal = float(0.5 * cfg.earth_pressure_coefficient * cfg.gravity_m_s2
                     * np.sum(h * h, dtype=np.float64) * area)
    return kinetic, grav, internal, kinetic + grav + internal


def globally_static(cfg: OracleConfig, b: np.ndarray, h: np.ndarray, q: np.ndarray) -> bool:
    """Static short-circuit (:353-363): no discharge and |grad(b+h)| <= tan(start)."""
    if np.max(np.abs(q), initial=0.0) > 1.0e-14:
        return False
    gy, gx = np.gradient(b + h, cfg.dy_m, cfg.dx_m)
    limit = np.tan(np.deg2rad(cfg.start_angle_deg)) + 1.0e-14
    return bool(np.max(np.hypot(gx, gy), initial=0.0) <= limit)


def _flux_of(cfg: OracleConfig, hs: np.ndarray, qs: np.ndarray, normal: int) -> np.ndarray:
    """Physical flux of a reconstructed state (:433-449)."""
    vel = _safe_div(qs, hs[..., None], hs[..., None] > cfg.dry_tolerance_m)
    qn = qs[..., normal]
    out = np.empty(hs.shape + (3,), dtype=np.float64)
    out[..., 0] = qn
    out[..., 1] = qn * vel[..., 0]
    out[..., 2] = qn * vel[..., 1]
    out[..., 1 + normal] += (0.5 * cfg.earth_pressure_coefficient
                             * cfg.gravity_m_s2 * hs * hs)
    return out


def face_pass(cfg: OracleConfig, b, h, q, dt, dh, dq, axis: int) -> None:
    """One direction of the unsplit face update (:365-431), accumulating in place.

    ``axis=1`` visits x faces (between columns), ``axis=0`` y faces.
    """
    K = cfg.earth_pressure_coefficient
    g = cfg.gravity_m_s2
    dry = cfg.dry_tolerance_m
    if axis == 1:
        lo = (slice(None), slice(None, -1))
        hi = (slice(None), slice(1, None))
        spacing, normal = cfg.dx_m, 0
    else:
        lo = (slice(None, -1), slice(None))
        hi = (slice(1, None), slice(None))
        spacing, normal = cfg.dy_m, 1
    bl, br = b[lo], b[hi]
    hl, hr = h[lo], h[hi]
    ql, qr = q[lo], q[hi]
    # Hydrostatic reconstruction on the steady head b + K h.
    bface = np.maximum(bl, br)
    hsl = np.maximum(((bl + K * hl) - bface) / K, 0.0)
    hsr = np.maximum(((br + K * hr) - bface) / K, 0.0)
    qsl = ql * _safe_div(hsl, hl, hl > dry)[..., None]
    qsr = qr * _safe_div(hsr, hr, hr > dry)[..., None]
    fl = _flux_of(cfg, hsl, qsl, normal)
    fr = _flux_of(cfg, hsr, qsr, normal)
    unl = _safe_div(qsl[..., normal], hsl, hsl > dry)
    unr = _safe_div(qsr[..., normal], hsr, hsr > dry)
    speed = np.maximum(np.abs(unl) + np.sqrt(K * g * hsl),
                       np.abs(unr) + np.sqrt(K * g * hsr))
    state_l = np.concatenate((hsl[..., None], qsl), axis=-1)
    state_r = np.concatenate((hsr[..., None], qsr), axis=-1)
    flux = 0.5 * (fl + fr) - 0.5 * speed[..., None] * (state_r - state_l)
    # Pressure-difference corrections, one per side of the face.
    minus = flux.copy()
    plus = flux.copy()
    minus[..., 1 + normal] += 0.5 * K * g * hl * hl - 0.5 * K * g * hsl * hsl
    plus[..., 1 + normal] += 0.5 * K * g * hr * hr - 0.5 * K * g * hsr * hsr
    lam = dt / spacing
    dh[lo] -= lam * minus[..., 0]
    dh[hi] += lam * plus[..., 0]
    dq[lo] -= lam * minus[..., 1:]
    dq[hi] += lam * plus[..., 1:]


def step(cfg: OracleConfig, b: np.ndarray, h: np.ndarray, q: np.ndarray,
         dt_s: float, external: np.ndarray | None = None) -> OracleStep:
    """One physics step of ``dt_s`` seconds (:191-314)."""
    dt = float(dt_s)
    if not np.isfinite(dt) or dt <= 0.0:
        raise ValueError("dt must be finite/positive")
    b = np.array(b, dtype=np.float64)
    h = np.array(h, dtype=np.float64)
    q = np.array(q, dtype=np.float64)
    ext = (np.zeros(q.shape) if external is None
           else np.broadcast_to(np.asarray(external, dtype=np.float64), q.shape).copy())
    area = cfg.dx_m * cfg.dy_m
    e0 = energy_terms(cfg, b, h, q)
    m0 = mass(cfg, h)
    p0 = momentum(cfg, q)
    cons = np.zeros(2)
    fric = np.zeros(2)
    extimp = np.zeros(2)
    fdiss = 0.0
    ework = 0.0
    remaining = dt
    substeps = 0
    max_cfl = 0.0
    dts: list[float] = []
    dry = cfg.dry_tolerance_m
    spacing_min = min(cfg.dx_m, cfg.dy_m)
    if (np.max(np.abs(ext), initial=0.0) <= 1.0e-14
            and globally_static(cfg, b, h, q)):
        return OracleStep(b, h, q, dt, 0, 0.0, m0, m0, p0, p0, cons, fric, extimp,
                          e0, e0, 0.0, 0.0, float(np.min(h, initial=0.0)), dts)
    while remaining > 1.0e-14:
        if substeps >= cfg.maximum_substeps:
            raise RuntimeError("MobileV2 maximum_substeps exceeded")
        vel = _safe_div(q, h[..., None], h[..., None] > dry)
        wave = np.linalg.norm(vel, axis=-1) + np.sqrt(
            cfg.earth_pressure_coefficient * cfg.gravity_m_s2 * np.maximum(h, 0.0))
        wmax = float(np.max(wave, initial=0.0))
        stable = remaining if wmax <= 1.0e-14 else cfg.cfl * spacing_min / wmax
        sub = min(remaining, stable)
        max_cfl = max(max_cfl, wmax * sub / spacing_min)
        dts.append(sub)
        q_sum_before = np.sum(q, axis=(0, 1), dtype=np.float64)
        dh = np.zeros_like(h)
        dq = np.zeros_like(q)
        face_pass(cfg, b, h, q, sub, dh, dq, axis=1)
        face_pass(cfg, b, h, q, sub, dh, dq, axis=0)
        hn = h + dh
        qn = q + dq
        if np.min(hn, initial=0.0) < -2.0e-13:
            raise RuntimeError("MobileV2 positivity failure")
        hn = np.maximum(hn, 0.0)
        qn[hn <= dry] = 0.0
        cons += (np.sum(qn, axis=(0, 1), dtype=np.float64) - q_sum_before) * area
        wet = hn[..., None] > dry
        v0 = _safe_div(qn, hn[..., None], wet)
        qe = qn + hn[..., None] * ext * sub
        ve = _safe_div(qe, hn[..., None], wet)
        extimp += np.sum(qe - qn, axis=(0, 1)) * area
        ework += float(np.sum(hn * np.sum(0.5 * (v0 + ve) * ext, axis=-1),
                              dtype=np.float64) * area * sub)
        spd = np.linalg.norm(ve, axis=-1)
        dec = cfg.basal_friction_coefficient * cfg.gravity_m_s2 * sub
        factor = np.maximum(0.0, 1.0 - dec / np.maximum(spd, 1.0e-15))
        va = ve * factor[..., None]
        qa = hn[..., None] * va
        fric += np.sum(qa - qe, axis=(0, 1)) * area
        fdiss += float(0.5 * np.sum(hn * (spd * spd - np.sum(va * va, axis=-1)),
                                    dtype=np.float64) * area)
        h, q = hn, qa
        remaining -= sub
        substeps += 1
    e1 = energy_terms(cfg, b, h, q)
    return OracleStep(b, h, q, dt, substeps, max_cfl, m0, mass(cfg, h), p0,
                      momentum(cfg, q), cons, fric, extimp, e0, e1, fdiss, ework,
                      float(np.min(h, initial=0.0)), dts)


def physical_entrainment(cfg: OracleConfig, b, h, q, depth, velocity=None):
    """Resting->Mobile exchange keeping b+h invariant (:142-167)."""
    depth = np.asarray(depth, dtype=np.float64)
    if depth.shape != np.shape(h) or np.any(depth < 0.0):
        raise ValueError("entrainment depth invalid")
    if np.any(depth > np.asarray(b) + 1.0e-14):
        raise ValueError("entrainment exceeds available support")
    vel = (np.zeros(np.shape(q)) if velocity is None
           else np.broadcast_to(np.asarray(velocity, dtype=np.float64), np.shape(q)))
    e_before = energy_terms(cfg, b, h, q)[3]
    b2 = np.asarray(b) - depth
    h2 = np.asarray(h) + depth
    q2 = np.asarray(q) + depth[..., None] * vel
    return (b2, h2, q2), energy_terms(cfg, b2, h2, q2)[3] - e_before


def physical_deposition(cfg: OracleConfig, b, h, q, depth):
    """Mobile->Resting exchange keeping b+h invariant (:169-189)."""
    depth = np.asarray(depth, dtype=np.float64)
    h = np.asarray(h, dtype=np.float64)
    if depth.shape != h.shape or np.any(depth < 0.0):
        raise ValueError("deposition depth invalid")
    if np.any(depth > h + 1.0e-14):
        raise ValueError("deposition exceeds Mobile thickness")
    e_before = energy_terms(cfg, b, h, q)[3]
    keep = _safe_div(h - depth, h, h > cfg.dry_tolerance_m)
    b2 = np.asarray(b) + depth
    h2 = np.maximum(h - depth, 0.0)
    q2 = np.asarray(q) * keep[..., None]
    return (b2, h2, q2), energy_terms(cfg, b2, h2, q2)[3] - e_before


# ---------------------------------------------------------------------------
# Production record (reference bulk_interaction/warp_mobile_v2.py).
# ---------------------------------------------------------------------------
def vertex_weights(ny: int, nx: int, dx: float, dy: float) -> np.ndarray:
    """Triangle-A-C vertex weights (runtime/bulk_state_authority.py:624-633)."""
    w = np.zeros((ny, nx), dtype=np.float64)
    f = dx * dy / 6.0
    w[:-1, :-1] += 2.0 * f
    w[:-1, 1:] += f
    w[1:, 1:] += 2.0 * f
    w[1:, :-1] += f
    return w


def production_summary(cfg: OracleConfig, density: float, b, h, q) -> np.ndarray:
    """The seven weighted sums of the production ``summarize`` kernel
    (warp_mobile_v2.py:28-54): volume, momentum x/y, max speed, kinetic,
    potential and internal (pressure) energy."""
    ny, nx = h.shape
    w = vertex_weights(ny, nx, cfg.dx_m, cfg.dy_m)
    wet = h > cfg.dry_tolerance_m
    vel = _safe_div(q, h[..., None], wet[..., None])
    spd = np.linalg.norm(vel, axis=-1)
    g, K = cfg.gravity_m_s2, cfg.earth_pressure_coefficient
    return np.asarray([
        float(np.sum(h * w)),
        float(np.sum(density * q[..., 0] * w)),
        float(np.sum(density * q[..., 1] * w)),
        float(np.max(np.where(wet, spd, 0.0), initial=0.0)),
        float(np.sum(np.where(wet, 0.5 * density * h * spd * spd * w, 0.0))),
        float(np.sum(density * g * h * b * w)),
        float(np.sum(density * 0.5 * K * g * h * h * w)),
    ])


def production_record(cfg: OracleConfig, density: float, b0, h0, q0, st: OracleStep) -> dict:
    """The WarpMobileStep fields of one production step (warp_mobile_v2.py:
    151-245) from the state before it and the oracle's step.  The impulse and
    dissipation totals are the reference solver's (``step`` above); the Warp
    diagnostic kernel of the production path (mobile_v2_warp.py:178-232)
    sums the same quantities and differs only in a cell that dries out within
    a substep, where it adds the face update before the momentum is zeroed."""
    before = production_summary(cfg, density, b0, h0, q0)
    bp = np.asarray([before[1], before[2], 0.0])
    if st.substeps == 0:
        return dict(volume_before_m3=before[0], volume_after_m3=before[0],
                    momentum_before_terrain_kg_m_s=bp, momentum_after_terrain_kg_m_s=bp,
                    gravity_pressure_impulse_terrain_ns=np.zeros(3),
                    basal_friction_impulse_terrain_ns=np.zeros(3),
                    numerical_dissipative_impulse_terrain_ns=np.zeros(3),
                    maximum_speed_m_s=before[3], substeps=0, cfl_limited=False,
                    kinetic_energy_before_j=before[4], kinetic_energy_after_j=before[4],
                    gravity_pressure_work_j=0.0, basal_friction_work_j=0.0,
                    transport_numerical_energy_residual_j=0.0, transport_mass_residual_m3=0.0)
    after = production_summary(cfg, density, st.b, st.h, st.q)
    ap = np.asarray([after[1], after[2], 0.0])
    gravity = np.asarray([st.conservative_impulse[0], st.conservative_impulse[1], 0.0]) * density
    friction = np.asarray([st.friction_impulse[0], st.friction_impulse[1], 0.0]) * density
    fwork = st.friction_dissipation * density
    remaining, cfl_limited = st.dt_s, False
    for sub in st.substep_dts:  # warp_mobile_v2.py:193-194
        cfl_limited |= sub < remaining - 1.0e-14
        remaining -= sub
    return dict(volume_before_m3=before[0], volume_after_m3=after[0],
                momentum_before_terrain_kg_m_s=bp, momentum_after_terrain_kg_m_s=ap,
                gravity_pressure_impulse_terrain_ns=gravity,
                basal_friction_impulse_terrain_ns=friction,
                numerical_dissipative_impulse_terrain_ns=ap - bp - gravity - friction,
                maximum_speed_m_s=after[3], substeps=st.substeps, cfl_limited=cfl_limited,
                kinetic_energy_before_j=before[4], kinetic_energy_after_j=after[4],
                gravity_pressure_work_j=(after[5] + after[6]) - (before[5] + before[6]),
                basal_friction_work_j=fwork,
                transport_numerical_energy_residual_j=(after[4] + after[5] + after[6])
                - (before[4] + before[5] + before[6]) + fwork,
                transport_mass_residual_m3=after[0] - before[0])
