"""Pin the CPU oracle against the reference's own outputs (no GPU needed).

The golden fixtures were produced by running the reference's
``MobileV2ReferenceSolver`` (tests/golden/make_golden.py); the JSON values are
copied from the reports the reference ships
(``outputs/mobile_v2_reference/*.json``).
"""

import json

import numpy as np
import pytest

from oracle import fixed_point as fx
from oracle import mobile_v2 as m
from oracle import relax as R
from oracle import surface as Sf

from conftest import GOLDEN


def _cfg():
    return m.OracleConfig()


def test_fv_oracle_is_bitwise_equal_to_reference_on_contract_states(fv_golden):
    cfg = _cfg()
    for name in fv_golden["names"]:
        s = m.step(cfg, fv_golden[f"{name}/b"], fv_golden[f"{name}/h"], fv_golden[f"{name}/q"],
                   float(fv_golden[f"{name}/dt"]))
        assert s.substeps == int(fv_golden[f"{name}/substeps"]), name
        assert np.array_equal(s.h, fv_golden[f"{name}/h_out"]), name
        assert np.array_equal(s.q, fv_golden[f"{name}/q_out"]), name
        sc = fv_golden[f"{name}/scalars"]
        assert s.maximum_cfl == sc[0]
        assert s.energy_after[3] == pytest.approx(sc[6], rel=1e-14, abs=1e-15)


def test_fv_oracle_matches_shipped_contract_report(fv_golden):
    rep = json.loads((GOLDEN / "reference_reports.json").read_text())["cpu_contracts"]
    cfg = _cfg()
    for name, want in rep.items():
        s = m.step(cfg, fv_golden[f"{name}/b"], fv_golden[f"{name}/h"], fv_golden[f"{name}/q"],
                   float(fv_golden[f"{name}/dt"]))
        assert s.substeps == want["substeps"], name
        assert s.maximum_cfl == pytest.approx(want["maximum_CFL"], abs=1e-15)
        assert s.energy_after[3] == pytest.approx(want["energy_after"], rel=1e-13, abs=1e-15)
        assert s.energy_before[3] == pytest.approx(want["energy_before"], rel=1e-13, abs=1e-15)
        assert s.friction_dissipation == pytest.approx(want["friction_dissipation"], rel=1e-11,
                                                       abs=1e-15)
        assert abs(s.mass_after - s.mass_before) <= 2.0e-13


def test_device_equivalence_substep_counts(fv_golden):
    rep = json.loads((GOLDEN / "reference_reports.json").read_text())["device_equivalence"]
    for name, want in rep.items():
        assert int(fv_golden[f"{name}/substeps"]) == want["CPU_substeps"] == want["DEVICE_substeps"]


def test_fv_oracle_gate_cfl04_bitwise(gate_golden):
    cfg = m.OracleConfig(basal_friction_coefficient=float(np.tan(np.deg2rad(35.0))), cfl=0.4)
    b, h = gate_golden["b"], gate_golden["h"]
    q = np.zeros(h.shape + (2,))
    for k in range(6):
        s = m.step(cfg, b, h, q, 1.0 / 60.0)
        h, q = s.h, s.q
        assert s.substeps == gate_golden["substeps"][k]
        assert np.array_equal(h, gate_golden[f"h_{k}"])
        assert np.array_equal(q, gate_golden[f"q_{k}"])


def test_fixed_point_mirror_tracks_fp64_and_conserves_exactly(gate_golden):
    b, h = gate_golden["b"], gate_golden["h"]
    datum = 0.5 * (b.min() + b.max())
    k = fx.choose_exponent(max(b.max() - datum, h.max()))
    p = fx.FixedParams(dx=0.05, dy=0.05, cfl=0.4, mu=float(np.tan(np.deg2rad(35.0))), exponent=k)
    bq = fx.quantize(b, datum, k)
    hq = fx.quantize(h, 0.0, k)
    m0 = int(hq.sum(dtype=np.int64))
    qx = np.zeros(h.shape, np.float32)
    qy = qx.copy()
    for s in range(6):
        hq, qx, qy, n, _ = fx.step(p, bq, hq, qx, qy, 1.0 / 60.0)
        assert n == gate_golden["substeps"][s]
        err = np.abs(fx.dequantize(hq, 0.0, k) - gate_golden[f"h_{s}"]).max()
        assert err <= 1.0e-6
        assert int(hq.sum(dtype=np.int64)) == m0
        assert hq.min() >= 0


def test_fixed_point_donor_cap_keeps_heights_nonnegative():
    # A thin film on a steep ramp at CFL 0.4: the cap must keep h >= 0.
    rng = np.random.default_rng(3)
    ny, nx = 24, 31
    ys, xs = np.indices((ny, nx))
    b = 0.9 * xs * 0.05 + 0.01 * rng.random((ny, nx))
    h = np.where(rng.random((ny, nx)) < 0.3, 1e-6 * rng.random((ny, nx)), 0.0)
    k = fx.choose_exponent(1.0)
    p = fx.FixedParams(dx=0.05, dy=0.05, cfl=0.4, exponent=k)
    bq = fx.quantize(b, 0.5, k)
    hq = fx.quantize(h, 0.0, k)
    qx = (rng.normal(0, 1e-6, (ny, nx))).astype(np.float32)
    qy = np.zeros_like(qx)
    m0 = int(hq.sum(dtype=np.int64))
    hq, qx, qy, n, _ = fx.step(p, bq, hq, qx, qy, 0.05)
    assert hq.min() >= 0 and int(hq.sum(dtype=np.int64)) == m0


def test_config0_generator_matches_gate_fixture_inputs():
    """The 256x256 config-0 inputs are regenerated from the seed; the gate
    fixture records their exact sums."""
    from pathlib import Path

    from soilb200 import workloads

    z = np.load(Path(__file__).resolve().parent / "golden" / "gate0.npz")
    t = workloads.config0_terrain(256, seed=0, dx=0.05)
    assert float(t["b_eff"].sum()) == float(z["b0_sum"])
    assert float(t["h"].sum()) == float(z["h0_sum"])
    assert z["substeps"].shape == (300,) and z["relax_iterations"].shape == (300,)


def test_deposition_oracle_matches_reference_cpu_operator():
    """oracle/deposition.py (device-kernel semantics) equals the reference's CPU
    DepositionOperator.apply on its device-test scenarios (fixture)."""
    from oracle import deposition as D

    z = np.load(GOLDEN / "deposition.npz")
    m = z["material"]
    for n in z["names"]:
        q = z[f"{n}/momentum"]
        b, h, _, _, vol, _, _ = D.step(z[f"{n}/resting"], z[f"{n}/mobile"], q[..., 0], q[..., 1],
                                       dx=0.05, dy=0.05, dt=1.0 / 60.0, density=m[0],
                                       cohesion=m[2], stop_angle_deg=m[5],
                                       settle_tail=bool(z[f"{n}/tail"]))
        assert np.array_equal(b, z[f"{n}/resting_out"]), n
        assert np.array_equal(h, z[f"{n}/mobile_out"]), n
        assert vol == pytest.approx(float(z[f"{n}/volume"]), abs=1e-15), n


def test_reached_relax_bit_identical_to_event_driven_adapter():
    """oracle.relax.reached_relax == EventDrivenMinimumSlopeAdapter.solve
    (golden fixture written by the reference): stable heights bit for bit and
    equal iteration counts, seeds = cells that differ from the reference
    height by more than the tolerance."""
    g = np.load(GOLDEN / "event.npz")
    for name in g["names"]:
        nx, ny, dx, dy = g[f"{name}/grid"]
        base, init = g[f"{name}/base"], g[f"{name}/initial"]
        seeds = np.abs(init - base) > 1e-8
        crit = float(np.tan(np.deg2rad(float(g[f"{name}/angle"]))))
        h, reached, it = R.reached_relax(init.T, seeds.T, (dx, dy), crit, 1e-8)
        assert it == int(g[f"{name}/iterations"]), name
        assert np.array_equal(h.T, g[f"{name}/stable"]), name
        assert reached.T[seeds].all(), name


def test_surface_oracle_matches_reference_cpu_sampler():
    """The clamped bilinear query equals the reference's CPU sampler bit for
    bit on in-range queries, and the reference test's known answers."""
    z = np.load(GOLDEN / "surface.npz")
    field = z["resting"] + z["mobile"]
    q = z["queries"]
    assert np.array_equal(Sf.bilinear(field, q[:, 0], q[:, 1]), z["values"])
    grid = np.arange(256, dtype=np.float64).reshape(16, 16)
    assert Sf.bilinear(grid, [1.0, 2.5], [2.0, 3.5]).tolist() == [18.0, 43.5]


def test_fixed_point_yield_arc_tangent_within_its_bound():
    """The float32 arc tangent of the fixed-point labelling (Abramowitz &
    Stegun 4.4.49, |polynomial error| <= 2e-8) against the double arc
    tangent: within 2e-7 rad over [0, 1], beyond it and at the ends."""
    from oracle import labels as L
    x = np.concatenate([np.linspace(0.0, 1.0, 200001), np.linspace(1.0, 60.0, 200001),
                        np.logspace(-9, 9, 20001), [0.0, 1.0, np.inf]]).astype(np.float32)
    got = L.atan_as4449(x).astype(np.float64)
    want = np.arctan(x.astype(np.float64))
    assert np.abs(got - want).max() <= 2.0e-7
    assert got[-3] == 0.0 and got[-1] == np.float32(np.pi / 2)


def test_fixed_point_yield_tracks_the_fp64_yield():
    """The float32 fixed-point yield against the FP64 yield (the reference's
    arithmetic) on the same quantized surface: slope within 4e-7 rad,
    severity within 1e-5, and the unstable masks equal up to cells whose
    start margin lies within float rounding of zero (at most 0.1 %)."""
    from oracle import labels as L
    rng = np.random.default_rng(11)
    ny, nx = 120, 140
    ys, xs = np.indices((ny, nx))
    b = 0.8 + 0.6 * np.sin(xs / 7.0) * np.cos(ys / 5.0) + 0.05 * rng.random((ny, nx))
    z = b - 0.02 - 0.12 * rng.random((ny, nx))
    k = 24
    bq, zq = fx.quantize(b, 0.0, k), fx.quantize(z, 0.0, k)
    hq = np.zeros_like(bq)
    kw = dict(dx=0.05, dy=0.05, tan_start=np.tan(np.deg2rad(38.0)),
              tan_stop=np.tan(np.deg2rad(30.0)), density=1600.0, gravity=9.81, cohesion=20.0,
              mobilization_depth=0.08, dry=1e-8)
    y32 = L.yield_init(bq, zq, hq, None, None, fixed_point=True, quantum=2.0 ** -k, **kw)
    y64 = L.yield_init(fx.dequantize(bq, 0.0, k), fx.dequantize(zq, 0.0, k),
                       np.zeros((ny, nx)), None, None, **kw)
    assert np.abs(y32["slope"].astype(np.float64) - y64["slope"]).max() <= 4.0e-7
    assert np.abs(y32["severity"].astype(np.float64) - y64["severity"]).max() <= 1.0e-5
    assert 0 < int(y64["unstable"].sum()) < ny * nx
    diff = int(np.count_nonzero(y32["unstable"] != y64["unstable"]))
    assert diff <= int(1e-3 * ny * nx), diff
