"""GPU tests of large-avalanche activation (sb_avalanche_mobilize) and the
lifecycle summary (sb_avalanche_persistence) against oracle/avalanche.py,
applied to the labels, severity and latches the GPU labelling produced.

FP64: activated fields bit-identical, sums within 1e-12 relative (order of
summation differs).  FX32: volume moved exactly (quanta), b_eff + h unchanged.
"""

import numpy as np
import pytest

import soilb200
from soilb200.bulk_state import B200BulkState
from oracle import avalanche as A

pytestmark = pytest.mark.gpu

DX = 0.05


def _pile(n=96):
    ys, xs = np.indices((n, n), dtype=np.float64)
    r = np.hypot(xs - n / 2, ys - n / 2) * DX
    return np.maximum(0.0, 1.6 - 1.1 * r) + 0.02 * np.sin(xs / 3.0)


def _bridge(state):
    mat = soilb200.MaterialScenario("pile", 1600.0, 35.0, 0.0, 0.5, 38.0, 30.0, 0.55)
    cfg = soilb200.LargeAvalancheTransitionConfig(persistence_time_s=1e-3,
                                                  minimum_mean_excess_start_deg=0.0)
    return soilb200.B200LargeAvalancheBridge(state.grid, mat, cfg, state=state), mat, cfg


@pytest.mark.parametrize("precision", ["fp64", "fx32"])
def test_mobilize_and_persistence_match_oracle(precision):
    b0 = _pile()
    st = B200BulkState(b0.shape, DX, DX, b0, precision=precision, mobile_headroom_m=1.0)
    g = st.grid
    br, mat, cfg = _bridge(st)
    diag = br.observe(1.0 / 60.0)
    assert diag.transition_ready, diag
    labels = g.download("labels")
    sev = g.download("severity")
    latch = g.download("latch")
    b, z, h = g.download("b_eff"), g.download("z_base"), g.download("mobile")
    out = soilb200._lib.MobilizeStats()
    soilb200._lib.check(g.ctx, soilb200._lib.load().sb_avalanche_mobilize(
        g.ctx, 0.25, cfg.mobilization_depth_m, cfg.dry_tolerance_m, out))
    b1, h1 = g.download("b_eff"), g.download("mobile")
    assert out.cells > 0
    if precision == "fp64":
        ob, oh, olatch, ocount, or2m, sums = A.mobilize(
            b, z, h, labels, diag.winner_label, latch, sev, dx=DX, dy=DX,
            depth=cfg.mobilization_depth_m, dry=cfg.dry_tolerance_m, time_s=0.25,
            act_count=np.zeros(b.shape, np.int32), r2m=np.zeros(b.shape))
        assert np.array_equal(b1, ob)
        assert np.array_equal(h1, oh)
        assert np.array_equal(g.download("latch"), olatch)
        assert out.cells == sums["cells"]
        assert out.transferred_volume_m3 == pytest.approx(sums["transferred"], rel=1e-12)
        assert out.newly_activated_area_m2 == pytest.approx(sums["new_area"], rel=1e-12)
        assert out.reactivated_volume_m3 == 0.0
        per = soilb200._lib.PersistenceStats()
        start, stop = np.deg2rad(38.0), np.deg2rad(30.0)
        soilb200._lib.check(g.ctx, soilb200._lib.load().sb_avalanche_persistence(
            g.ctx, start, stop, cfg.dry_tolerance_m, cfg.mobile_activity_speed_m_s, per))
        ref = A.persistence(b0, b1, h1, g.download("momentum_x"), g.download("momentum_y"),
                            g.download("slope"), labels >= 0, g.download("latch"), ocount, or2m,
                            np.zeros(b.shape), dx=DX, dy=DX, start_rad=start, stop_rad=stop,
                            dry=cfg.dry_tolerance_m, activity_speed=cfg.mobile_activity_speed_m_s,
                            tile_size=st.tile_size)
        assert per.unique_cells_ever_activated == ref["unique"]
        assert per.current_mobile_cell_count == ref["wet"]
        assert per.active_tile_count == ref["tiles"]
        assert per.cumulative_r2m_m3 == pytest.approx(ref["r2m"], rel=1e-12)
        assert per.current_mobile_volume_m3 == pytest.approx(ref["mobile_volume"], rel=1e-12)
        assert per.net_spatial_transfer_m3 == pytest.approx(ref["net_transfer"], rel=1e-12)
        assert per.activated_slope_sum_rad == pytest.approx(ref["slope_sum"], rel=1e-12)
        assert abs(per.net_terrain_volume_change_m3) <= 1e-12
    else:
        assert np.array_equal(b1 + h1, b + h)
        r = st.reservoir_reduction(1600.0)
        assert r["mobile_quanta_w6"] == out.transferred_w6_quanta
    # a second activation finds the component latched: nothing moves
    out2 = soilb200._lib.MobilizeStats()
    soilb200._lib.check(g.ctx, soilb200._lib.load().sb_avalanche_mobilize(
        g.ctx, 0.5, cfg.mobilization_depth_m, cfg.dry_tolerance_m, out2))
    assert out2.cells == 0
    st.close()


def test_observe_and_maybe_mobilize_record():
    b0 = _pile(80)
    st = B200BulkState(b0.shape, DX, DX, b0, precision="fx32", mobile_headroom_m=1.0)
    br, _, _ = _bridge(st)
    res = br.observe_and_maybe_mobilize(1.0 / 60.0)
    assert res.classification == br.LARGE_AVALANCHE_MOBILE_PATH
    assert res.transitioned and res.transferred_volume_m3 > 0.0
    assert res.newly_activated_volume_m3 == pytest.approx(res.transferred_volume_m3, rel=1e-12)
    assert res.unique_cells_ever_activated > 0
    assert res.cumulative_resting_to_mobile_m3 == pytest.approx(res.transferred_volume_m3, rel=1e-9)
    assert res.current_mobile_volume_m3 == pytest.approx(res.transferred_volume_m3, rel=1e-9)
    st.close()


@pytest.mark.parametrize("name", ["pile64", "plane21"])
def test_observe_and_maybe_mobilize_matches_reference_cpu_controller(name):
    """B200LargeAvalancheBridge.observe_and_maybe_mobilize (FP64) against the
    reference's CPU LargeAvalancheTransitionController.observe_and_maybe_mobilize
    (golden fixture written by the reference), called repeatedly with no
    transport in between, z_base = 0: per call the transition flag, the
    persistence time, the unstable and largest-component counts and the
    transferred volume; after every call b_eff and mobile height bit for bit.
    (The CPU controller also gives the new mobile material a launch velocity,
    the device path a zero-momentum exchange as the reference's Warp kernel
    does, so momentum is not compared.)"""
    from conftest import GOLDEN
    g = np.load(GOLDEN / "avalanche.npz")
    dt = float(g["dt"])
    b0 = g[f"{name}/resting0"]
    st = B200BulkState(b0.shape, DX, DX, b0, precision="fp64", mobile_headroom_m=1.0)
    mat = soilb200.MaterialScenario("golden_pile", 1600.0, 35.0, 0.0, 0.5, 38.0, 30.0, 0.55)
    br = soilb200.B200LargeAvalancheBridge(st.grid, mat, soilb200.LargeAvalancheTransitionConfig(),
                                           state=st)
    for k, (transitioned, volume, persistence, unstable, largest) in enumerate(g[f"{name}/record"]):
        res = br.observe_and_maybe_mobilize(dt)
        assert res.transitioned == bool(transitioned), (name, k)
        assert res.transferred_volume_m3 == pytest.approx(volume, rel=1e-12, abs=1e-15), (name, k)
        assert res.persistence_s == pytest.approx(persistence, rel=1e-12, abs=1e-15), (name, k)
        assert res.unstable_cell_count == int(unstable), (name, k)
        assert res.largest_connected_cell_count == int(largest), (name, k)
        assert np.array_equal(st.grid.download("b_eff"), g[f"{name}/resting_{k}"]), (name, k)
        assert np.array_equal(st.grid.download("mobile"), g[f"{name}/mobile_{k}"]), (name, k)
    st.close()
