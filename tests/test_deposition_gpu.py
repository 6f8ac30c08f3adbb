"""GPU tests of the Mobile -> Resting deposition operator (sb_deposition_step).

* FP64: fields bit-identical to the CPU oracle (device-kernel semantics,
  pinned to the reference's CPU DepositionOperator) and within 1e-13 m / m^3
  of the reference's own outputs, the bound the reference's device tests use
  (tests/test_device_bulk_state.py:150-230).
* FX32: b_eff + h unchanged cell by cell and the settled volume exact in
  quanta; forced cells untouched; moving cells do not settle.
"""

import numpy as np
import pytest

import soilb200
from soilb200.bulk_state import B200BulkState, B200DepositionOperator
from oracle import deposition as D

pytestmark = pytest.mark.gpu

GOLDEN = __import__("pathlib").Path(__file__).resolve().parent / "golden" / "deposition.npz"


def _material(m):
    return soilb200.MaterialScenario("device_state", *[float(v) for v in m])


def _state(resting, mobile, q, precision):
    st = B200BulkState(resting.shape, 0.05, 0.05, resting, z_base_m=np.zeros_like(resting),
                       precision=precision, mobile_headroom_m=0.5)
    st.grid.upload("mobile", mobile)
    st.grid.upload("momentum_x", q[..., 0])
    st.grid.upload("momentum_y", q[..., 1])
    return st


@pytest.mark.parametrize("precision", ["fp64", "fx32"])
def test_deposition_matches_reference_scenarios(precision):
    z = np.load(GOLDEN)
    mat = _material(z["material"])
    for n in z["names"]:
        r, h, q = z[f"{n}/resting"], z[f"{n}/mobile"], z[f"{n}/momentum"]
        st = _state(r, h, q, precision)
        op = B200DepositionOperator()
        op.bind_device_state(st)
        rec = op.step_resident(mat, 1.0 / 60.0, settle_subcell_tail=bool(z[f"{n}/tail"]))
        b_out = st.grid.download("b_eff")
        h_out = st.grid.download("mobile")
        if precision == "fp64":
            ob, oh, oqx, oqy, vol, mx, my = D.step(
                r, h, q[..., 0], q[..., 1], dx=0.05, dy=0.05, dt=1.0 / 60.0,
                density=mat.assumed_bulk_density_kg_m3, cohesion=mat.cohesion_proxy_pa,
                stop_angle_deg=mat.stop_angle_deg, settle_tail=bool(z[f"{n}/tail"]))
            assert np.array_equal(b_out, ob), n
            assert np.array_equal(h_out, oh), n
            assert np.array_equal(st.grid.download("momentum_x"), oqx), n
            assert rec.deposited_volume_m3 == pytest.approx(vol, rel=1e-13, abs=1e-16), n
            assert rec.removed_mobile_momentum_terrain_kg_m_s[0] == pytest.approx(mx, rel=1e-12,
                                                                                  abs=1e-15)
            tol = 1e-13
        else:
            tol = 2e-8  # fixed-point heights: a few quanta of the grid's quantum
        assert np.abs(b_out - z[f"{n}/resting_out"]).max() <= tol, n
        assert np.abs(h_out - z[f"{n}/mobile_out"]).max() <= tol, n
        assert rec.deposited_volume_m3 == pytest.approx(float(z[f"{n}/volume"]), abs=max(tol, 1e-13))
        st.close()


def test_fx32_deposition_keeps_surface_and_exact_volume():
    rng = np.random.default_rng(5)
    shape = (48, 37)
    ys, xs = np.indices(shape)
    r = 0.5 + 0.03 * np.sin(xs / 3.0) * np.cos(ys / 5.0)
    h = np.where(rng.random(shape) < 0.7, 0.002 + 0.02 * rng.random(shape), 0.0)
    q = np.zeros(shape + (2,))
    q[5:9, 5:9, 0] = 0.5 * h[5:9, 5:9]   # 0.5 m/s > threshold: these do not settle
    st = _state(r, h, q, "fx32")
    forcing = np.zeros(shape, bool)
    forcing[20:30, 10:20] = True
    st.set_tool_forcing_mask(forcing)
    b0, h0 = st.grid.download("b_eff"), st.grid.download("mobile")
    r0 = st.reservoir_reduction(1600.0)
    op = B200DepositionOperator()
    op.bind_device_state(st)
    mat = soilb200.MaterialScenario("m", 1600.0, 35.0, 0.0, 0.5, 38.0, 30.0, 0.55)
    rec = op.step_resident(mat, 1.0 / 60.0)
    b1, h1 = st.grid.download("b_eff"), st.grid.download("mobile")
    assert np.array_equal(b1 + h1, b0 + h0)
    assert np.array_equal(h1[forcing], h0[forcing])
    moving = np.zeros(shape, bool)
    moving[5:9, 5:9] = h0[5:9, 5:9] > 0
    assert np.array_equal(h1[moving], h0[moving])
    r1 = st.reservoir_reduction(1600.0)
    moved_q = r1["resting_quanta_w6"] - r0["resting_quanta_w6"]
    assert moved_q == r0["mobile_quanta_w6"] - r1["mobile_quanta_w6"]
    assert moved_q > 0
    assert rec.deposited_volume_m3 == pytest.approx(r1["resting_volume_m3"] - r0["resting_volume_m3"],
                                                    rel=1e-12)
    m2r = st.grid.download("m2r_cumulative")
    assert m2r.sum() == pytest.approx(rec.deposited_volume_m3, rel=1e-12)
    st.close()


@pytest.mark.parametrize("precision", ["fp64", "fx32"])
def test_exchange_sums_are_reproducible(precision):
    """Entrained / deposited volumes and removed momentum come out bit for bit
    the same on every run of the same command (fixed-order block folds, no
    floating-point atomics), over a command spanning many blocks."""
    n = 256
    rng = np.random.default_rng(11)
    resting = 0.5 + 0.3 * rng.random((n, n))
    mobile = 0.05 * rng.random((n, n))
    q = 0.01 * rng.standard_normal((n, n, 2))
    idx = rng.choice(n * n, size=40000, replace=False).astype(np.int32)
    depth = 0.02 * rng.random(idx.size)
    results = []
    for _ in range(3):
        st = _state(resting, mobile, q, precision)
        v_in = st.entrain_host_indices(idx, depth, reason="cut")
        rec = st.deposit_host_indices(idx, 0.5 * depth, density_kg_m3=1600.0, reason="settle")
        results.append((v_in, rec["deposited_volume_m3"],
                        *rec["removed_mobile_momentum_kg_m_s"][:2]))
        st.close()
    assert results[0] == results[1] == results[2]
    assert results[0][0] > 0.0 and results[0][1] > 0.0
