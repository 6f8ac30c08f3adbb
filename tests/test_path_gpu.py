"""GPU tests of the plain terrain step (config-1 path on a small grid).

* The fused step (one CUDA graph per physics step, classification and gating
  on the device) must reproduce the operator-by-operator path bit for bit:
  fields, substeps, classifications, residual rounds.
* FX32: the total material volume sum(w*(b-z)+) + sum(w*h) is conserved
  exactly (entrainment, transport and relaxation all move whole quanta).
"""

import numpy as np
import pytest

import soilb200
from soilb200 import workloads
from soilb200.pipeline import PlainPath

pytestmark = pytest.mark.gpu

DT = 1.0 / 60.0


def _material():
    return soilb200.MaterialScenario("path_test", 1600.0, 35.0, 0.0, 0.5, 38.0, 30.0, 0.55)


def _setup(n, seed=1):
    b = workloads.noise_pile(n, seed, 0.05)
    cut = workloads.BucketCut((n, n), 0.05, b, start=(0.25 * n * 0.05, 0.5 * n * 0.05))
    return b, cut


def _fields(path):
    g = path.grid
    return [g.download(k) for k in ("b_eff", "mobile", "momentum_x", "momentum_y")]


@pytest.mark.parametrize("precision,residual", [("fx32", "gated"), ("fx32", "always"),
                                                ("fp64", "always")])
def test_fused_step_equals_operator_path(precision, residual):
    n = 160
    b, cut = _setup(n)
    z = np.zeros_like(b)
    fused = PlainPath(b, z, dx=0.05, material=_material(), precision=precision, tile_size=32,
                      residual=residual, fused=True)
    ops = PlainPath(b, z, dx=0.05, material=_material(), precision=precision, tile_size=32,
                    residual=residual, fused=False)
    for k in range(24):
        idx, tgt = cut.footprint((k + 1) * DT)
        a = fused.step(DT, idx, tgt)
        o = ops.step(DT, idx, tgt)
        assert a.substeps == o.substeps, k
        assert a.classification == o.classification, k
        assert (a.unstable_cells, a.regions, a.largest) == (o.unstable_cells, o.regions, o.largest)
        assert a.residual_rounds == o.residual_rounds, k
        if k % 6 == 5:
            for fa, fo in zip(_fields(fused), _fields(ops)):
                assert np.array_equal(fa, fo), k
    fused.close()
    ops.close()


def test_fx32_path_conserves_total_volume_exactly():
    n = 192
    b, cut = _setup(n, seed=3)
    path = PlainPath(b, np.zeros_like(b), dx=0.05, material=_material(), precision="fx32",
                     tile_size=32, residual="always")
    r0 = path.state.reservoir_reduction(1600.0)
    total0 = r0["resting_quanta_w6"] + r0["mobile_quanta_w6"]
    moved = 0.0
    for k in range(40):
        idx, tgt = cut.footprint((k + 1) * DT)
        st = path.step(DT, idx, tgt)
        moved += st.entrained_m3
        r = path.state.reservoir_reduction(1600.0)
        assert r["resting_quanta_w6"] + r["mobile_quanta_w6"] == total0, k
    assert moved > 0.0
    assert path.state.reservoir_reduction(1600.0)["mobile_quanta_w6"] > 0
    path.close()


def test_host_driven_substep_loop_equals_graph(monkeypatch):
    """SOILB200_NO_GRAPH=1 (host-driven launches of the same kernels, one
    synchronisation per substep) gives the step graph's fields and records."""
    n = 96
    b, cut = _setup(n, seed=2)
    z = np.zeros_like(b)
    graph = PlainPath(b, z, dx=0.05, material=_material(), tile_size=32, residual="gated",
                      fused=False)
    monkeypatch.setenv("SOILB200_NO_GRAPH", "1")
    host = PlainPath(b, z, dx=0.05, material=_material(), tile_size=32, residual="gated",
                     fused=False)
    monkeypatch.delenv("SOILB200_NO_GRAPH")
    for k in range(12):
        idx, tgt = cut.footprint((k + 1) * DT)
        a = graph.step(DT, idx, tgt)
        o = host.step(DT, idx, tgt)
        assert a.substeps == o.substeps, k
        assert (a.unstable_cells, a.regions, a.largest) == (o.unstable_cells, o.regions, o.largest)
        sa, so = graph.mobile.last_stats, host.mobile.last_stats
        assert sa.friction_dissipation == pytest.approx(so.friction_dissipation, rel=1e-12, abs=1e-30)
        for j in range(2):
            assert sa.conservative_impulse_m4_s[j] == pytest.approx(
                so.conservative_impulse_m4_s[j], rel=1e-12, abs=1e-30)
        assert sa.before.mass_m3 == so.before.mass_m3
        assert sa.after.mass_m3 == so.after.mass_m3
        for fa, fo in zip(_fields(graph), _fields(host)):
            assert np.array_equal(fa, fo), k
    graph.close()
    host.close()


@pytest.mark.parametrize("precision", ["fx32", "fp64"])
def test_fused_step_cut_command_growth(precision):
    """Cut commands of varying length, one larger than the fused step's first
    command buffer (4096 cells), an empty one and a repeated one: the fused
    step still equals the operator path field for field."""
    n = 160
    b, _ = _setup(n, seed=3)
    z = np.zeros_like(b)
    fused = PlainPath(b, z, dx=0.05, material=_material(), precision=precision, tile_size=32,
                      residual="always", fused=True)
    ops = PlainPath(b, z, dx=0.05, material=_material(), precision=precision, tile_size=32,
                    residual="always", fused=False)
    rng = np.random.default_rng(7)
    sizes = [200, 0, 6000, 6000, 50, 9000, 0, 300]
    for k, m in enumerate(sizes):
        idx = rng.choice(n * n, size=m, replace=False).astype(np.int32)
        tgt = b.ravel()[idx] - rng.uniform(0.0, 0.05, size=m)
        a = fused.step(DT, idx, tgt)
        o = ops.step(DT, idx, tgt)
        assert a.substeps == o.substeps, k
        assert a.entrained_m3 == pytest.approx(o.entrained_m3, rel=1e-12, abs=1e-15), k
        assert a.residual_rounds == o.residual_rounds, k
        for fa, fo in zip(_fields(fused), _fields(ops)):
            assert np.array_equal(fa, fo), k
    fused.close()
    ops.close()


def test_fused_step_rejects_invalid_cut_commands():
    """A non-finite target, an index outside the grid and mismatched lengths
    raise ValueError with the reference's message; a later valid step works."""
    n = 64
    b, _ = _setup(n, seed=2)
    path = PlainPath(b, np.zeros_like(b), dx=0.05, material=_material(), tile_size=32,
                     fused=True)
    idx = np.array([n * n // 2 + n // 2 + k for k in range(3)], dtype=np.int32)  # on the pile
    with pytest.raises(ValueError, match="invalid entrainment request"):
        path.step(DT, idx, np.array([0.1, np.nan, 0.1]))
    with pytest.raises(ValueError, match="invalid entrainment request"):
        path.step(DT, idx, np.array([0.1, 0.1]))
    with pytest.raises(ValueError, match="entrainment index outside state"):
        path.step(DT, np.array([5, n * n], dtype=np.int32), np.array([0.1, 0.1]))
    st = path.step(DT, idx, b.ravel()[idx] - 0.01)
    assert st.entrained_m3 > 0.0
    path.close()
