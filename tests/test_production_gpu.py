"""The production solver's step record against the oracle.

``B200ProductionMobileV2Solver.step_resident`` returns the reference's
``WarpMobileStep`` (bulk_interaction/warp_mobile_v2.py:151-245): Triangle-A-C
weighted volume, momentum and energies before and after the step, the
impulse and work totals of its substeps, and the residuals built from them.
``oracle.mobile_v2.production_record`` restates that record on the oracle's
FP64 step; the FP64 fields are bit-identical (so substeps and the CFL flag
are equal), and every record value agrees to 1e-12 of the magnitudes it is
built from (the weighted sums are taken in a different order; the residual
fields are differences of totals ~1e3 times larger) over five steps of a config-0 mound,
plus the static short-circuit record of a resting mound.
"""

import numpy as np
import pytest

import soilb200
from oracle import mobile_v2 as M
from soilb200 import workloads
from soilb200.bulk_state import B200BulkState, B200ProductionMobileV2Solver

pytestmark = pytest.mark.gpu

DX = 0.05
DT = 1.0 / 60.0
DENSITY = 1600.0
FIELDS_VEC = ("momentum_before_terrain_kg_m_s", "momentum_after_terrain_kg_m_s",
              "gravity_pressure_impulse_terrain_ns", "basal_friction_impulse_terrain_ns",
              "numerical_dissipative_impulse_terrain_ns")
FIELDS_SCALAR = ("volume_before_m3", "volume_after_m3", "maximum_speed_m_s",
                 "kinetic_energy_before_j", "kinetic_energy_after_j", "gravity_pressure_work_j",
                 "basal_friction_work_j", "transport_numerical_energy_residual_j",
                 "transport_mass_residual_m3")


def _material():
    return soilb200.MaterialScenario("m", DENSITY, 35.0, 0.0, 0.5, 38.0, 30.0, 0.55)


def _compare(rec, want, k, energy_scale):
    """Record values to 1e-12 of the magnitudes they are built from: the
    residual fields are differences of totals ~1e3-1e4 times larger."""
    assert rec.substeps == want["substeps"], k
    assert rec.cfl_limited == want["cfl_limited"], k
    for name in FIELDS_SCALAR:
        got, ref = getattr(rec, name), want[name]
        scale = max(abs(ref), energy_scale) if name.endswith("_j") else abs(ref)
        if name == "transport_mass_residual_m3":
            scale = want["volume_before_m3"]
        assert abs(got - ref) <= 1e-12 * scale + 1e-18, (k, name, got, ref)
    mom = max(float(np.abs(np.asarray(want[n])).max()) for n in FIELDS_VEC)
    for name in FIELDS_VEC:
        got, ref = np.asarray(getattr(rec, name)), np.asarray(want[name])
        assert np.abs(got - ref).max() <= 1e-12 * mom + 1e-18, (k, name, got, ref)


def _energy_scale(cfg, b, h, q, o):
    """Largest energy total of the step (kinetic, potential, pressure)."""
    s0 = M.production_summary(cfg, DENSITY, b, h, q)
    s1 = M.production_summary(cfg, DENSITY, o.b, o.h, o.q)
    return float(max(np.abs(s0[4:]).max(), np.abs(s1[4:]).max(), 1.0))


def _solver(b, z, h, q=None):
    st = B200BulkState(b.shape, DX, DX, b, z_base_m=z, precision="fp64", mobile_headroom_m=1.0)
    st.grid.upload("mobile", h)
    if q is not None:
        st.grid.upload("momentum_x", q[..., 0])
        st.grid.upload("momentum_y", q[..., 1])
    solver = B200ProductionMobileV2Solver(state=st, config=soilb200.MobileV2Config(dx_m=DX,
                                                                                   dy_m=DX))
    solver.bind_device_state(st, _material())
    return st, solver


def test_production_record_matches_oracle_on_a_moving_mound():
    cfg0 = workloads.config0_terrain(96, seed=2, dx=DX)
    b, z, h = cfg0["b_eff"], cfg0["z_base"], cfg0["h"]
    q = np.stack([0.6 * h, -0.2 * h], axis=-1)  # a mound sliding down-slope: never static
    st, solver = _solver(b, z, h, q)
    ocfg = M.OracleConfig(dx_m=DX, dy_m=DX)
    for k in range(5):
        rec = solver.step_resident(DT)
        o = M.step(ocfg, b, h, q, DT)
        want = M.production_record(ocfg, DENSITY, b, h, q, o)
        _compare(rec, want, k, _energy_scale(ocfg, b, h, q, o))
        b, h, q = o.b, o.h, o.q
        assert np.array_equal(st.grid.download("mobile"), h), k
    assert rec.substeps > 0
    st.close()


def test_production_record_of_a_static_pile():
    n = 48
    ys, xs = np.indices((n, n), dtype=np.float64)
    b = 0.5 + 0.01 * np.tan(np.deg2rad(10.0)) * xs * DX  # far below the start angle
    h = np.zeros((n, n))
    st, solver = _solver(b, np.zeros_like(b), h)
    rec = solver.step_resident(DT)
    ocfg = M.OracleConfig(dx_m=DX, dy_m=DX)
    o = M.step(ocfg, b, h, np.zeros((n, n, 2)), DT)
    want = M.production_record(ocfg, DENSITY, b, h, np.zeros((n, n, 2)), o)
    assert o.substeps == 0
    _compare(rec, want, 0, _energy_scale(ocfg, b, h, np.zeros((n, n, 2)), o))
    st.close()
