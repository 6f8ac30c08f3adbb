"""GPU tests of ``PlainPath.settle``: the site's resting surface relaxed to
repose in place after the cut steps, on the path's own resident grid.

* plain schedule: the relax_critical_slope sweep on the path's FX32 b_eff is
  bit-identical to the fixed-point CPU mirror of the reference's
  ``relax_critical_slope`` (``slope_model.py:273-343``), same sweep count;
* learned schedule (trained network + plain sweeps): converges to the same
  tolerance, every face of the end state is within tan(35 deg) * distance +
  tolerance (checked on the CPU over the reference's four neighbour pairs),
  and the volume ledger is exact;
* only the resting surface moves: the mobile layer and momenta are untouched.
"""

import numpy as np
import pytest

import soilb200
from oracle import fixed_point as fx
from oracle import relax as R
from soilb200 import learned, workloads
from soilb200.pipeline import PlainPath
from soilb200.train_repose import DEFAULT_WEIGHTS

pytestmark = pytest.mark.gpu

DX = 0.05
DT = 1.0 / 60.0
ANGLE = 35.0
TOL = 1.0e-4 * DX


def _material():
    return soilb200.MaterialScenario("settle_test", 1600.0, ANGLE, 0.0, 0.5, 38.0, 30.0, 0.55)


def _cut_path(n=256, steps=40, seed=3):
    b = workloads.noise_pile(n, seed, DX)
    cut = workloads.BucketCut((n, n), DX, b, start=(0.25 * n * DX, 0.5 * n * DX))
    path = PlainPath(b, np.zeros_like(b), dx=DX, material=_material(), tile_size=32)
    for k in range(steps):
        idx, tgt = cut.footprint((k + 1) * DT)
        path.step(DT, idx, tgt)
    return path


def _max_excess(h):
    tan = float(np.tan(np.deg2rad(ANGLE)))
    worst = 0.0
    for d0, d1, dist in R.neighbor_pairs(DX, DX):
        a, b = R.paired_views(h, d0, d1)
        worst = max(worst, float((np.abs(a - b) - tan * dist).max()))
    return worst


def test_settle_plain_schedule_matches_fixed_point_mirror():
    path = _cut_path()
    g = path.grid
    k, datum = g.height_exponent, g.datum
    start = g.download("b_eff")
    mobile = [g.download(f) for f in ("mobile", "momentum_x", "momentum_y")]
    hq = fx.quantize(start, datum, k)
    lr = learned.LearnedRelaxation(g, learned.ReposeNet.load(DEFAULT_WEIGHTS), ANGLE)
    st = path.settle(lr, TOL, learned.PLAIN)
    out_q, it, conv = R.relax_critical_slope_fixed(
        hq, (DX, DX), float(np.tan(np.deg2rad(ANGLE))), 2.0 ** -k, max_iterations=400000,
        tolerance=TOL)
    assert st.converged and conv
    assert int(st.iterations) == it
    assert np.array_equal(g.download("b_eff"), fx.dequantize(out_q, datum, k))
    for name, before in zip(("mobile", "momentum_x", "momentum_y"), mobile):
        assert np.array_equal(g.download(name), before), name
    path.close()


def test_settle_learned_schedule_reaches_repose_with_exact_ledger():
    assert DEFAULT_WEIGHTS.exists(), DEFAULT_WEIGHTS
    path = _cut_path()
    g = path.grid
    k, datum = g.height_exponent, g.datum
    start = g.download("b_eff")
    q0 = int(fx.quantize(start, datum, k).astype(np.int64).sum())
    assert _max_excess(start) > TOL  # the cut left faces above repose
    lr = learned.LearnedRelaxation(g, learned.ReposeNet.load(DEFAULT_WEIGHTS), ANGLE)
    st = path.settle(lr, TOL)
    out = g.download("b_eff")
    assert st.converged
    assert int(fx.quantize(out, datum, k).astype(np.int64).sum()) == q0
    assert _max_excess(out) <= TOL + 2.0 ** -k
    path.close()


def test_settle_rejects_a_relaxation_of_another_grid():
    path = _cut_path(n=96, steps=2)
    other = soilb200.DeviceGrid((96, 96), DX, DX, precision="fx32")
    lr = learned.LearnedRelaxation(other, learned.ReposeNet.load(DEFAULT_WEIGHTS), ANGLE)
    with pytest.raises(ValueError):
        path.settle(lr, TOL)
    other.close()
    path.close()
