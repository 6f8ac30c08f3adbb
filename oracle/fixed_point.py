"""CPU mirror of the 32-bit production Mobile V2 arithmetic -- TEST INFRASTRUCTURE.

The production CUDA path stores heights (``b_eff``, ``z_base``, ``h``) as int32
multiples of a power-of-two quantum ``Q = 2**-k`` metres (``b``/``z`` relative
to a datum) and momentum as float32.  Every face mass flux is rounded to whole
quanta once, so both neighbours move the same integer and mass is conserved
exactly; each donor may lose at most ``floor(h/4)`` quanta per face, so heights
can never become negative (the reference equations are positivity-preserving
for CFL <= 0.25, where this cap never binds; it only limits faces at CFL 0.4).

The operation order below is the specification of the FX instantiation of
the kernel in ``csrc/sb_fv.cuh``.  Velocities are computed once per cell
(u = q * (1/h)) and reused by its faces: the reference's reconstructed
discharge q * (hs/h) equals u * hs and its face velocity qs/hs equals u, so
this is the same mathematics with no division per face.  All float32 operations are single
IEEE operations (the library is compiled with ``-fmad=false``), so this mirror
and the kernel agree bit for bit.

Equations follow the reference ``experimental/mobile_v2_reference.py``
(``_face_updates`` :365-431, ``step`` :236-307) with three stated deviations:
hydrostatic depth uses the exact integer support difference, a donor cap
replaces the positivity raise/clip, and the wave speed uses float32.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

F32 = np.float32


@dataclass
class FixedParams:
    dx: float
    dy: float
    gravity: float = 9.81
    K: float = 0.45
    cfl: float = 0.18
    dry: float = 1.0e-10
    mu: float = 0.55
    start_angle_deg: float = 34.0
    exponent: int = 28
    maximum_substeps: int = 4096

    @property
    def quantum(self) -> float:
        return 2.0 ** (-self.exponent)


def choose_exponent(span_m: float) -> int:
    """Largest k <= 30 with span * 2**k * 4 <= 2**31 (4x headroom for growth)."""
    span = max(float(span_m), 1.0e-6)
    k = int(np.floor(np.log2(2.0 ** 29 / span)))
    return int(min(30, max(12, k)))


def quantize(x: np.ndarray, datum: float, exponent: int) -> np.ndarray:
    return np.rint((np.asarray(x, dtype=np.float64) - datum) * 2.0 ** exponent).astype(np.int32)


def dequantize(xq: np.ndarray, datum: float, exponent: int) -> np.ndarray:
    return np.asarray(xq, dtype=np.float64) * 2.0 ** (-exponent) + datum


def _div(num, den, wet):
    out = np.zeros(np.broadcast(num, den).shape, dtype=F32)
    np.divide(num, den, out=out, where=wet)
    return out


def cell_velocity(p: FixedParams, hq, qx, qy):
    """Per-cell velocity q/h (0 where h == 0) and celerity sqrt(K g h)."""
    QF = F32(p.quantum)
    hf = hq.astype(F32) * QF
    inv = _div(np.ones_like(hf), hf, hq > 0)
    return qx * inv, qy * inv, np.sqrt(F32(p.K * p.gravity) * hf)


def face_fluxes(p: FixedParams, lam: np.float32, bl, br, hlq, hrq, unl, utl, unr, utr, cl, cr):
    """Fluxes of one face family from cell velocities (un, ut) and celerities c.

    Returns (mass quanta int32, Fn_minus, Fn_plus, Ft)."""
    KGF = F32(p.K * p.gravity)
    HKGF = F32(0.5 * p.K * p.gravity)
    QF = F32(p.quantum)
    QKF = F32(p.quantum / p.K)
    INVQ = F32(2.0 ** p.exponent)
    DRYF = F32(p.dry)
    zero = F32(0)
    bface = np.maximum(bl, br)
    dl = (bface - bl).astype(np.int32)
    dr = (bface - br).astype(np.int32)
    hl = hlq.astype(F32) * QF
    hr = hrq.astype(F32) * QF
    low_l, low_r = dl != 0, dr != 0
    hsl = np.where(low_l, np.maximum(hl - dl.astype(F32) * QKF, zero), hl)
    hsr = np.where(low_r, np.maximum(hr - dr.astype(F32) * QKF, zero), hr)
    csl = np.where(low_l, np.sqrt(KGF * hsl), cl)
    csr = np.where(low_r, np.sqrt(KGF * hsr), cr)
    corl = np.where(low_l, (HKGF * hl) * hl - (HKGF * hsl) * hsl, zero)
    corr = np.where(low_r, (HKGF * hr) * hr - (HKGF * hsr) * hsr, zero)
    qnsl, qtsl = unl * hsl, utl * hsl
    qnsr, qtsr = unr * hsr, utr * hsr
    wl, wr = hsl > DRYF, hsr > DRYF
    vnl, vtl = np.where(wl, unl, zero), np.where(wl, utl, zero)
    vnr, vtr = np.where(wr, unr, zero), np.where(wr, utr, zero)
    fnl = qnsl * vnl + (HKGF * hsl) * hsl
    fnr = qnsr * vnr + (HKGF * hsr) * hsr
    ftl = qnsl * vtl
    ftr = qnsr * vtr
    spd = np.maximum(np.abs(vnl) + csl, np.abs(vnr) + csr)
    half = F32(0.5) * spd
    fh = F32(0.5) * (qnsl + qnsr) - half * (hsr - hsl)
    fn = F32(0.5) * (fnl + fnr) - half * (qnsr - qnsl)
    ft = F32(0.5) * (ftl + ftr) - half * (qtsr - qtsl)
    m = np.rint((lam * fh) * INVQ)
    m = np.clip(m, F32(-(2.0 ** 30)), F32(2.0 ** 30)).astype(np.int32)
    m = np.where(m > 0, np.minimum(m, hlq >> 2), np.maximum(m, -(hrq >> 2))).astype(np.int32)
    return m, fn + corl, fn + corr, ft


def wave_speed(p: FixedParams, hq: np.ndarray, qx: np.ndarray, qy: np.ndarray) -> np.ndarray:
    """Wave speed of a state as evaluated by the step prologue."""
    QF = F32(p.quantum)
    KGF = F32(p.K * p.gravity)
    hn = hq.astype(F32) * QF
    wet = hn > F32(p.dry)
    inv = _div(np.ones_like(hn), hn, wet)
    vx = qx * inv
    vy = qy * inv
    return np.sqrt(vx * vx + vy * vy) + np.sqrt(KGF * hn)


def substep(p: FixedParams, bq, hq, qx, qy, sub_dt: float, ax=None, ay=None):
    """One substep on int32/float32 fields; returns new fields, FP64 diagnostics
    and the wave speed of the new state (which sets the next dt)."""
    ny, nx = hq.shape
    lamx = F32(sub_dt / p.dx)
    lamy = F32(sub_dt / p.dy)
    QF = F32(p.quantum)
    u, v, cel = cell_velocity(p, hq, qx, qy)
    # x faces: between (r, c) and (r, c+1); normal = x, tangential = y.
    mx, fnmx, fnpx, ftx = face_fluxes(p, lamx, bq[:, :-1], bq[:, 1:], hq[:, :-1], hq[:, 1:],
                                      u[:, :-1], v[:, :-1], u[:, 1:], v[:, 1:],
                                      cel[:, :-1], cel[:, 1:])
    # y faces: between (r, c) and (r+1, c); normal = y, tangential = x.
    my, fnmy, fnpy, fty = face_fluxes(p, lamy, bq[:-1, :], bq[1:, :], hq[:-1, :], hq[1:, :],
                                      v[:-1, :], u[:-1, :], v[1:, :], u[1:, :],
                                      cel[:-1, :], cel[1:, :])

    def pad_e(a):  # east face value per cell (zero on the last column)
        out = np.zeros((ny, nx), dtype=a.dtype)
        out[:, :-1] = a
        return out

    def pad_w(a):
        out = np.zeros((ny, nx), dtype=a.dtype)
        out[:, 1:] = a
        return out

    def pad_n(a):
        out = np.zeros((ny, nx), dtype=a.dtype)
        out[:-1, :] = a
        return out

    def pad_s(a):
        out = np.zeros((ny, nx), dtype=a.dtype)
        out[1:, :] = a
        return out

    dh = ((-pad_e(mx) + pad_w(mx)) - pad_n(my)) + pad_s(my)
    zero = F32(0)
    dqx = (((zero - lamx * pad_e(fnmx)) + lamx * pad_w(fnpx)) - lamy * pad_n(fty)) + lamy * pad_s(fty)
    dqy = (((zero - lamx * pad_e(ftx)) + lamx * pad_w(ftx)) - lamy * pad_n(fnmy)) + lamy * pad_s(fnpy)
    hnq = (hq + dh).astype(np.int32)
    assert int(hnq.min(initial=0)) >= 0
    hn = hnq.astype(F32) * QF
    wet = hn > F32(p.dry)
    qxn = np.where(wet, qx + dqx, zero)
    qyn = np.where(wet, qy + dqy, zero)
    inv = _div(np.ones_like(hn), hn, wet)
    vbx = qxn * inv
    vby = qyn * inv
    if ax is not None:
        dtf = F32(sub_dt)
        qex = np.where(wet, qxn + (hn * ax) * dtf, qxn)
        qey = np.where(wet, qyn + (hn * ay) * dtf, qyn)
        vex = qex * inv
        vey = qey * inv
    else:
        qex, qey, vex, vey = qxn, qyn, vbx, vby
    spd = np.sqrt(vex * vex + vey * vey)
    dec = F32(p.mu * p.gravity * sub_dt)
    fac = np.maximum(zero, F32(1) - dec / np.maximum(spd, F32(1.0e-15)))
    vax = vex * fac
    vay = vey * fac
    qxo = hn * vax
    qyo = hn * vay
    wave = spd * fac + np.sqrt(F32(p.K * p.gravity) * hn)
    h64 = hn.astype(np.float64)
    diag = {
        "cons": np.asarray([np.sum(qxn.astype(np.float64) - qx), np.sum(qyn.astype(np.float64) - qy)]),
        "ext": np.asarray([np.sum(qex.astype(np.float64) - qxn), np.sum(qey.astype(np.float64) - qyn)]),
        "fric": np.asarray([np.sum(qxo.astype(np.float64) - qex), np.sum(qyo.astype(np.float64) - qey)]),
        "fdiss": 0.5 * float(np.sum(h64 * (spd.astype(np.float64) ** 2
                                           - (vax.astype(np.float64) ** 2 + vay.astype(np.float64) ** 2)))),
        "wave": float(np.max(wave, initial=F32(0))),
    }
    return hnq, qxo.astype(F32), qyo.astype(F32), diag


def static_check(p: FixedParams, bq, hq, qx, qy) -> bool:
    if max(float(np.max(np.abs(qx), initial=0.0)), float(np.max(np.abs(qy), initial=0.0))) > 1.0e-14:
        return False
    H = bq.astype(np.int64) + hq.astype(np.int64)
    return bool(max_surface_gradient(p, H) <= np.tan(np.deg2rad(p.start_angle_deg)) + 1.0e-14)


def _diff_axis(H, axis, spacing, Q):
    """np.gradient's differences (central inside, one-sided at the edges, edge_order 1)
    of an integer surface, scaled by Q / (2 spacing) resp. Q / spacing as one
    rounded constant: (H[i+1] - H[i-1]) * (Q / (2 d))."""
    H = np.moveaxis(H, axis, 0)
    d = np.zeros(H.shape, dtype=np.float64)
    n = H.shape[0]
    if n < 2:
        return np.moveaxis(d, 0, axis)
    d[1:-1] = (H[2:] - H[:-2]).astype(np.float64) * (Q / (2.0 * spacing))
    d[0] = (H[1] - H[0]).astype(np.float64) * (Q / spacing)
    d[-1] = (H[-1] - H[-2]).astype(np.float64) * (Q / spacing)
    return np.moveaxis(d, 0, axis)


def max_surface_gradient(p: FixedParams, H) -> float:
    """Largest free-surface slope |grad(b + h)| of the fixed-point path (the
    static short-circuit of mobile_v2_reference.py:199-205 on quantised
    heights): the maximum of gx^2 + gy^2 is taken first, its square root last."""
    Q = p.quantum
    gx = _diff_axis(H, 1, p.dx, Q)
    gy = _diff_axis(H, 0, p.dy, Q)
    return float(np.sqrt(np.max(gx * gx + gy * gy, initial=0.0)))


def step(p: FixedParams, bq, hq, qx, qy, dt_s: float, ax=None, ay=None):
    """A full physics step of the fixed-point path; returns fields, substeps, dts."""
    bq = np.asarray(bq, dtype=np.int32)
    hq = np.asarray(hq, dtype=np.int32).copy()
    qx = np.asarray(qx, dtype=F32).copy()
    qy = np.asarray(qy, dtype=F32).copy()
    if ax is None and static_check(p, bq, hq, qx, qy):
        return hq, qx, qy, 0, []
    remaining = float(dt_s)
    smin = min(p.dx, p.dy)
    dts = []
    w = float(np.max(wave_speed(p, hq, qx, qy), initial=F32(0)))
    while remaining > 1.0e-14:
        if len(dts) >= p.maximum_substeps:
            raise RuntimeError("MobileV2 maximum_substeps exceeded")
        stable = remaining if w <= 1.0e-14 else p.cfl * smin / w
        sub = min(remaining, stable)
        hq, qx, qy, diag = substep(p, bq, hq, qx, qy, sub, ax, ay)
        w = diag["wave"]
        dts.append(sub)
        remaining -= sub
    return hq, qx, qy, len(dts), dts
