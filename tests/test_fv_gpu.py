"""GPU parity of the Mobile V2 finite-volume kernels (through the C ABI).

* FP64 instantiation vs the reference's outputs (golden fixtures): fields are
  compared bit for bit and substep counts must be equal.
* FX32 mirror-exact variant (``SOILB200_FV_EXACT=1``: IEEE reciprocal, root
  and division, no FMA contraction) vs its CPU mirror (oracle/fixed_point.py):
  bit-identical int32 heights and float32 momentum, exactly zero mass change.
* FX32 production kernel (FMA contraction, approximate reciprocal/root): the
  same substep counts, exactly zero mass change, heights within 1e-6 m of the
  FP64 reference on the contract states (stated production bound: 1e-5 m
  after the 5 s gate) and within 1e-7 m of the mirror.
"""

import numpy as np
import pytest

import soilb200
from oracle import fixed_point as fx
from oracle import mobile_v2 as m

pytestmark = pytest.mark.gpu


def _state(g, name):
    return soilb200.MobileV2State(g[f"{name}/b"], g[f"{name}/h"], g[f"{name}/q"])


def test_fp64_kernel_bitwise_equals_reference(fv_golden):
    solver = soilb200.B200MobileV2Solver(soilb200.MobileV2Config(), precision="fp64")
    for name in fv_golden["names"]:
        step = solver.step(_state(fv_golden, name), float(fv_golden[f"{name}/dt"]))
        assert step.substeps == int(fv_golden[f"{name}/substeps"]), name
        assert np.array_equal(step.state.h_m, fv_golden[f"{name}/h_out"]), name
        assert np.array_equal(step.state.q_m2_s, fv_golden[f"{name}/q_out"]), name
        sc = fv_golden[f"{name}/scalars"]
        assert step.maximum_cfl == sc[0]
        assert step.energy_after_j_per_density == pytest.approx(sc[6], rel=1e-12, abs=1e-14)
        assert abs(step.mass_residual_m3) <= 2.0e-13
        assert float(np.max(np.abs(step.momentum_accounting_residual_m4_s))) <= 2.0e-12
    solver.close()


def test_fp64_kernel_gate_cfl04_six_steps(gate_golden):
    cfg = soilb200.MobileV2Config.unchecked(
        basal_friction_coefficient=float(np.tan(np.deg2rad(35.0))), cfl=0.4)
    solver = soilb200.B200MobileV2Solver(cfg, precision="fp64")
    state = soilb200.MobileV2State(gate_golden["b"], gate_golden["h"],
                                   np.zeros(gate_golden["h"].shape + (2,)))
    for k in range(6):
        step = solver.step(state, 1.0 / 60.0)
        state = step.state
        assert step.substeps == gate_golden["substeps"][k]
        assert np.array_equal(state.h_m, gate_golden[f"h_{k}"])
        assert np.array_equal(state.q_m2_s, gate_golden[f"q_{k}"])
    solver.close()


def _fx_run(solver, b, h, q, dt, steps, mu, cfl):
    """Run the kernel and the CPU mirror from the same quantized inputs."""
    state = soilb200.MobileV2State(b, h, q)
    st = solver.step(state, dt)
    k, datum = solver.last_quantization
    p = fx.FixedParams(dx=0.05, dy=0.05, cfl=cfl, mu=mu, exponent=k)
    bq = fx.quantize(b, datum, k)
    hq = fx.quantize(h, 0.0, k)
    qx = q[..., 0].astype(np.float32)
    qy = q[..., 1].astype(np.float32)
    hq, qx, qy, n, _ = fx.step(p, bq, hq, qx, qy, dt)
    return st, hq, qx, qy, n, k


def test_fx32_kernel_bitwise_equals_cpu_mirror(fv_golden, monkeypatch):
    cfg = soilb200.MobileV2Config()
    monkeypatch.setenv("SOILB200_FV_EXACT", "1")  # read when the solver creates its grids
    solver = soilb200.B200MobileV2Solver(cfg, precision="fx32")
    for name in fv_golden["names"]:
        b, h, q = fv_golden[f"{name}/b"], fv_golden[f"{name}/h"], fv_golden[f"{name}/q"]
        st, hq, qx, qy, n, k = _fx_run(solver, b, h, q, float(fv_golden[f"{name}/dt"]), 1,
                                       cfg.basal_friction_coefficient, cfg.cfl)
        assert st.substeps == n, name
        if n == 0:  # static short-circuit returns the caller's state untouched
            assert np.array_equal(st.state.h_m, h), name
            continue
        assert np.array_equal(st.state.h_m, fx.dequantize(hq, 0.0, k)), name
        assert np.array_equal(st.state.q_m2_s[..., 0], qx.astype(np.float64)), name
        assert np.array_equal(st.state.q_m2_s[..., 1], qy.astype(np.float64)), name
        assert st.mass_residual_m3 == 0.0
        # against the FP64 reference: well inside the 1e-5 m production bound
        assert np.abs(st.state.h_m - fv_golden[f"{name}/h_out"]).max() <= 1.0e-6, name
    solver.close()


def test_fx32_production_kernel_within_bounds(fv_golden):
    cfg = soilb200.MobileV2Config()
    solver = soilb200.B200MobileV2Solver(cfg, precision="fx32")
    for name in fv_golden["names"]:
        b, h, q = fv_golden[f"{name}/b"], fv_golden[f"{name}/h"], fv_golden[f"{name}/q"]
        st, hq, qx, qy, n, k = _fx_run(solver, b, h, q, float(fv_golden[f"{name}/dt"]), 1,
                                       cfg.basal_friction_coefficient, cfg.cfl)
        assert st.substeps == n, name
        assert st.mass_residual_m3 == 0.0, name
        if n == 0:
            assert np.array_equal(st.state.h_m, h), name
            continue
        assert np.abs(st.state.h_m - fx.dequantize(hq, 0.0, k)).max() <= 1.0e-7, name
        qscale = max(float(np.abs(qx).max()), float(np.abs(qy).max()), 1e-30)
        assert np.abs(st.state.q_m2_s[..., 0] - qx).max() <= 1e-4 * qscale, name
        assert np.abs(st.state.q_m2_s[..., 1] - qy).max() <= 1e-4 * qscale, name
        assert np.abs(st.state.h_m - fv_golden[f"{name}/h_out"]).max() <= 1.0e-6, name
    solver.close()


def test_fx32_gate_tracks_fp64_with_exact_mass(gate_golden):
    mu = float(np.tan(np.deg2rad(35.0)))
    cfg = soilb200.MobileV2Config.unchecked(basal_friction_coefficient=mu, cfl=0.4)
    solver = soilb200.B200MobileV2Solver(cfg, precision="fx32")
    state = soilb200.MobileV2State(gate_golden["b"], gate_golden["h"],
                                   np.zeros(gate_golden["h"].shape + (2,)))
    m0 = None
    for k in range(6):
        step = solver.step(state, 1.0 / 60.0)
        state = step.state
        assert step.mass_residual_m3 == 0.0
        m0 = step.mass_before_m3 if m0 is None else m0
        assert step.mass_after_m3 == m0
        assert np.abs(state.h_m - gate_golden[f"h_{k}"]).max() <= 1.0e-5
    solver.close()


@pytest.mark.parametrize("shape", [(2, 2), (3, 200), (150, 5), (65, 129), (17, 19)])
def test_fx32_and_fp64_ragged_shapes(shape, monkeypatch):
    rng = np.random.default_rng(sum(shape))
    ny, nx = shape
    ys, xs = np.indices(shape)
    b = 0.2 + 0.3 * np.sin(xs / 4.0) * np.cos(ys / 3.0) + 0.05 * rng.random(shape)
    h = np.maximum(0.0, 0.1 * rng.random(shape) - 0.02)
    q = h[..., None] * rng.normal(0, 0.4, shape + (2,))
    cfg = soilb200.MobileV2Config()
    ref = m.step(m.OracleConfig(), b, h, q, 0.02)
    s64 = soilb200.B200MobileV2Solver(cfg, precision="fp64")
    st = s64.step(soilb200.MobileV2State(b, h, q), 0.02)
    assert st.substeps == ref.substeps
    assert np.array_equal(st.state.h_m, ref.h)
    assert np.array_equal(st.state.q_m2_s, ref.q)
    s64.close()
    monkeypatch.setenv("SOILB200_FV_EXACT", "1")  # read when the solver creates its grid
    s32 = soilb200.B200MobileV2Solver(cfg, precision="fx32")
    st2, hq, qx, qy, n, k = _fx_run(s32, b, h, q, 0.02, 1, cfg.basal_friction_coefficient, cfg.cfl)
    assert st2.substeps == n
    assert np.array_equal(st2.state.h_m, fx.dequantize(hq, 0.0, k))
    assert np.array_equal(st2.state.q_m2_s[..., 0], qx.astype(np.float64))
    assert st2.mass_residual_m3 == 0.0
    s32.close()
    monkeypatch.delenv("SOILB200_FV_EXACT")
    fast = soilb200.B200MobileV2Solver(cfg, precision="fx32")  # production kernel
    st3 = fast.step(soilb200.MobileV2State(b, h, q), 0.02)
    assert st3.substeps == n
    assert st3.mass_residual_m3 == 0.0
    assert np.abs(st3.state.h_m - ref.h).max() <= 1.0e-6
    fast.close()


def test_substep_cap_and_dt_errors_match_reference():
    shape = (16, 16)
    b = np.zeros(shape)
    h = np.full(shape, 0.2)
    q = np.zeros(shape + (2,))
    q[..., 0] = 0.4
    cfg = soilb200.MobileV2Config(maximum_substeps=1)
    solver = soilb200.B200MobileV2Solver(cfg, precision="fp64")
    with pytest.raises(RuntimeError, match="MobileV2 maximum_substeps exceeded"):
        solver.step(soilb200.MobileV2State(b, h, q), 0.5)
    with pytest.raises(ValueError, match="dt must be finite/positive"):
        solver.step(soilb200.MobileV2State(b, h, q), -1.0)
    solver.close()


def test_static_short_circuit_returns_input_unchanged(fv_golden):
    for precision in ("fp64", "fx32"):
        solver = soilb200.B200MobileV2Solver(soilb200.MobileV2Config(), precision=precision)
        for name in ("STATIC_FLAT", "STATIC_SLOPE"):
            st = solver.step(_state(fv_golden, name), 0.05)
            assert st.substeps == 0
            assert np.array_equal(st.state.h_m, fv_golden[f"{name}/h"])
            assert np.max(np.abs(st.state.q_m2_s)) == 0.0
        solver.close()


def test_external_acceleration_matches_oracle():
    shape = (20, 24)
    rng = np.random.default_rng(11)
    b = 0.1 * rng.random(shape)
    h = 0.05 + 0.05 * rng.random(shape)
    q = np.zeros(shape + (2,))
    ext = np.zeros(shape + (2,))
    ext[..., 0] = 2.0
    ext[..., 1] = -1.0
    ref = m.step(m.OracleConfig(), b, h, q, 0.02, external=ext)
    solver = soilb200.B200MobileV2Solver(soilb200.MobileV2Config(), precision="fp64")
    st = solver.step(soilb200.MobileV2State(b, h, q), 0.02, external_acceleration_m_s2=ext)
    assert st.substeps == ref.substeps
    assert np.array_equal(st.state.h_m, ref.h)
    assert np.array_equal(st.state.q_m2_s, ref.q)
    assert st.external_work_j_per_density == pytest.approx(ref.external_work, rel=1e-10)
    solver.close()
