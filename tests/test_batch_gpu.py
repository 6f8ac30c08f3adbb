"""GPU tests of the batched patch runtime (many Mobile V2 grids per launch).

Every patch of a batch must end bit-identical to the same patch stepped alone
on its own device grid (same quantum, FX32), with equal substep counts per
step, whatever the tile shape (rows per warp strip); volume is conserved in
exact quanta (sum of h); the autotuner leaves the state as it found it.
"""

import numpy as np
import pytest

import soilb200
from soilb200 import _lib, workloads
from soilb200.batch import B200PatchBatch
from soilb200.grid import DeviceGrid
from soilb200.mobile_v2 import mobile_params

pytestmark = pytest.mark.gpu

DT = 1.0 / 60.0


def _wavy(shape, seed):
    rng = np.random.default_rng(seed)
    ys, xs = np.indices(shape)
    b = 0.3 + 0.25 * np.sin(xs / 5.0) * np.cos(ys / 4.0) + 0.04 * rng.random(shape)
    h = np.maximum(0.0, 0.12 * rng.random(shape) - 0.03)
    q = h[..., None] * rng.normal(0.0, 0.5, shape + (2,))
    return b, h, q


def _patches():
    out = []
    for i, shape in enumerate([(40, 70), (64, 64), (33, 100), (130, 65), (2, 47), (31, 30)]):
        out.append(_wavy(shape, 11 + i))
    out.append(workloads.config2_patch(3))
    out.append(workloads.config2_patch(17))
    # a static patch (flat, still): the prologue's short-circuit, zero substeps
    out.append((np.ones((48, 52)), np.full((48, 52), 0.05), np.zeros((48, 52, 2))))
    return out


def _alone(b, h, q, k, datum, cfg, steps):
    grid = DeviceGrid(b.shape, cfg.dx_m, cfg.dy_m, precision="fx32", height_exponent=k,
                      datum_m=datum)
    for name, val in (("z_base", b), ("b_eff", b), ("mobile", h), ("momentum_x", q[..., 0]),
                      ("momentum_y", q[..., 1])):
        grid.upload(name, val)
    subs = []
    for _ in range(steps):
        st = _lib.MobileStats()
        _lib.check(grid.ctx, _lib.load().sb_mobile_step(grid.ctx, DT, mobile_params(cfg), st))
        subs.append(int(st.substeps))
    out = [grid.download(n) for n in ("mobile", "momentum_x", "momentum_y")]
    grid.close()
    return out, subs


def _batch(patches, cfg):
    states = [soilb200.MobileV2State(b, h, q) for b, h, q in patches]
    return B200PatchBatch(states, cfg)


@pytest.mark.parametrize("rows", [None, 4, 64])
def test_batch_equals_patches_stepped_alone(rows):
    cfg = soilb200.MobileV2Config()
    patches = _patches()
    batch = _batch(patches, cfg)
    if rows is not None:
        batch.rows = [rows] * batch.n_patches
    subs = []
    for _ in range(3):
        stats = batch.step_stats(DT)
        subs.append([int(s.substeps) for s in stats])
        for s in stats:  # fluxes move whole quanta between cells: sum(h) is exact
            assert s.after.mass_quanta == s.before.mass_quanta
    assert subs[0][-1] == 0  # the static patch
    assert max(subs[0]) > 1
    for i, (b, h, q) in enumerate(patches):
        k, datum = batch.quantization[i]
        fields, alone_subs = _alone(b, h, q, k, datum, cfg, 3)
        assert alone_subs == [s[i] for s in subs], i
        for name, ref in zip(("mobile", "momentum_x", "momentum_y"), fields):
            assert np.array_equal(batch.download(i, name), ref), (i, name)
    batch.close()


def test_batch_step_records_match_single_solver():
    cfg = soilb200.MobileV2Config()
    patches = _patches()[:3]
    batch = _batch(patches, cfg)
    steps = batch.step(DT)
    solver = soilb200.B200MobileV2Solver(cfg, precision="fx32")
    for i, (b, h, q) in enumerate(patches):
        ref = solver.step(soilb200.MobileV2State(b, h, q), DT)
        got = steps[i]
        assert got.substeps == ref.substeps
        assert np.array_equal(got.state.h_m, ref.state.h_m)
        assert np.array_equal(got.state.q_m2_s, ref.state.q_m2_s)
        assert got.mass_residual_m3 == 0.0
        assert got.mass_before_m3 == ref.mass_before_m3
        assert got.maximum_cfl == ref.maximum_cfl
        assert got.energy_after_j_per_density == pytest.approx(ref.energy_after_j_per_density,
                                                               rel=1e-9, abs=1e-12)
    solver.close()
    batch.close()


def test_autotune_restores_state_and_sets_rows():
    cfg = soilb200.MobileV2Config()
    patches = _patches()
    batch = _batch(patches, cfg)
    before = [batch.download(i, "mobile") for i in range(batch.n_patches)]
    ms = batch.autotune(DT, trials=1)
    assert ms > 0.0
    assert all(r in (4, 8, 16, 32, 64) for r in batch.rows)
    for i in range(batch.n_patches):
        assert np.array_equal(batch.download(i, "mobile"), before[i])
    # stepping after tuning still matches the patches stepped alone
    batch.step_stats(DT)
    b, h, q = patches[1]
    k, datum = batch.quantization[1]
    fields, _ = _alone(b, h, q, k, datum, cfg, 1)
    assert np.array_equal(batch.download(1, "mobile"), fields[0])
    batch.close()


def test_batch_argument_errors():
    cfg = soilb200.MobileV2Config()
    batch = _batch(_patches()[:2], cfg)
    with pytest.raises(ValueError):
        batch.rows = [2, 16]
    with pytest.raises(ValueError, match="dt must be finite/positive"):
        batch.step_stats(-1.0)
    with pytest.raises(ValueError):
        batch.upload(0, "mobile", np.zeros((3, 3)))
    batch.close()


def test_batch_labels_equal_patches_labelled_alone():
    """Config 2's label check: after three batched steps every patch's
    canonical labels and component statistics equal those of the same patch
    stepped and labelled alone on its own grid (bit for bit; the resting layer
    z_base = b_eff - 0.2 m gives the yield detector material to fail)."""
    cfg = soilb200.MobileV2Config()
    patches = _patches()[:-1]
    states = [soilb200.MobileV2State(b, h, q) for b, h, q in patches]
    zs = [b - 0.2 for b, _, _ in patches]
    batch = B200PatchBatch(states, cfg, z_base=zs)
    for _ in range(3):
        batch.step_stats(DT)
    mat = soilb200.MaterialScenario("batch", 1600.0, 35.0, 0.0, 0.5, 38.0, 30.0, 0.55)
    stats = batch.label(mat)
    assert sum(s.unstable_cell_count for s in stats) > 0
    for i, (b, h, q) in enumerate(patches):
        k, datum = batch.quantization[i]
        grid = DeviceGrid(b.shape, cfg.dx_m, cfg.dy_m, precision="fx32", height_exponent=k,
                          datum_m=datum)
        for name, val in (("z_base", zs[i]), ("b_eff", b), ("mobile", h),
                          ("momentum_x", q[..., 0]), ("momentum_y", q[..., 1])):
            grid.upload(name, val)
        for _ in range(3):
            st = _lib.MobileStats()
            _lib.check(grid.ctx, _lib.load().sb_mobile_step(grid.ctx, DT, mobile_params(cfg), st))
        bridge = soilb200.B200LargeAvalancheBridge(grid, mat)
        ref = bridge.label(release_settled_latches=False)
        assert np.array_equal(batch.labels(i), bridge.labels()), i
        got = stats[i]
        assert (got.unstable_cell_count, got.connected_region_count,
                got.largest_connected_cell_count, got.winner_root) == \
            (ref.unstable_cell_count, ref.connected_region_count,
             ref.largest_connected_cell_count, ref.winner_root), i
        assert got.largest_connected_area_m2 == ref.largest_connected_area_m2, i
        assert got.largest_connected_mobilizable_volume_m3 == \
            ref.largest_connected_mobilizable_volume_m3, i
        grid.close()
    batch.close()
