"""GPU parity of the FX32 register-streaming substep kernel.

The streaming kernel (warps walk down 30-column strips, faces in registers)
in its mirror-exact variant (SOILB200_FV_EXACT=1) and the TMA tile kernel
(SOILB200_FV_TILE=1) must produce identical int32 heights and float32
momentum, and both must equal the CPU mirror (oracle/fixed_point.py), across
strip edges (nx around multiples of 30) and row-chunk edges
(SOILB200_FV_ROWS=r splits every strip into ceil(ny/r) balanced row chunks:
r = 1, 3 and 64).  The production variant (FMA contraction, approximate
reciprocal and root) must give the same fields for every row chunking (the
chunking never changes a cell's arithmetic) and stay within 1e-7 m of the
exact variant with the same substep counts and exact mass.
"""

import numpy as np
import pytest

import soilb200
from oracle import fixed_point as fx

pytestmark = pytest.mark.gpu

DT = 0.02


def _wavy(shape, seed):
    rng = np.random.default_rng(seed)
    ys, xs = np.indices(shape)
    b = 0.3 + 0.25 * np.sin(xs / 5.0) * np.cos(ys / 4.0) + 0.04 * rng.random(shape)
    h = np.maximum(0.0, 0.12 * rng.random(shape) - 0.03)
    q = h[..., None] * rng.normal(0.0, 0.5, shape + (2,))
    return b, h, q


def _run(monkeypatch, env, b, h, q, ext=None, steps=2):
    for key, val in env.items():
        monkeypatch.setenv(key, val)
    solver = soilb200.B200MobileV2Solver(soilb200.MobileV2Config(), precision="fx32")
    state = soilb200.MobileV2State(b, h, q)
    subs = []
    for _ in range(steps):
        st = solver.step(state, DT, external_acceleration_m_s2=ext)
        assert st.mass_residual_m3 == 0.0
        subs.append(st.substeps)
        state = st.state
    quant = solver.last_quantization
    solver.close()
    for key in env:
        monkeypatch.delenv(key)
    return state, subs, quant


@pytest.mark.parametrize("shape", [(257, 301), (64, 61), (33, 30), (100, 31), (9, 91), (2, 47)])
@pytest.mark.parametrize("rows", ["1", "3", "64"])
def test_stream_kernel_equals_tile_kernel(monkeypatch, shape, rows):
    b, h, q = _wavy(shape, sum(shape) + int(rows))
    tile, s_tile, _ = _run(monkeypatch, {"SOILB200_FV_TILE": "1"}, b, h, q)
    strm, s_strm, _ = _run(monkeypatch, {"SOILB200_FV_ROWS": rows, "SOILB200_FV_EXACT": "1"},
                           b, h, q)
    assert s_tile == s_strm
    assert np.array_equal(tile.h_m, strm.h_m)
    assert np.array_equal(tile.q_m2_s, strm.q_m2_s)


@pytest.mark.parametrize("shape,rows", [((67, 95), "5"), ((128, 121), "1"), ((40, 30), "64")])
def test_stream_kernel_equals_cpu_mirror_with_external(monkeypatch, shape, rows):
    b, h, q = _wavy(shape, 7 * shape[1])
    ext = np.zeros(shape + (2,))
    ext[..., 0] = 1.5
    ext[..., 1] = -0.75
    state, subs, (k, datum) = _run(monkeypatch, {"SOILB200_FV_ROWS": rows,
                                                 "SOILB200_FV_EXACT": "1"}, b, h, q, ext, steps=1)
    cfg = soilb200.MobileV2Config()
    p = fx.FixedParams(dx=cfg.dx_m, dy=cfg.dy_m, cfl=cfg.cfl, mu=cfg.basal_friction_coefficient,
                       exponent=k)
    bq = fx.quantize(b, datum, k)
    hq = fx.quantize(h, 0.0, k)
    ax = ext[..., 0].astype(np.float32)
    ay = ext[..., 1].astype(np.float32)
    hq, qx, qy, n, _ = fx.step(p, bq, hq, q[..., 0].astype(np.float32),
                               q[..., 1].astype(np.float32), DT, ax, ay)
    assert subs == [n]
    assert np.array_equal(state.h_m, fx.dequantize(hq, 0.0, k))
    assert np.array_equal(state.q_m2_s[..., 0], qx.astype(np.float64))
    assert np.array_equal(state.q_m2_s[..., 1], qy.astype(np.float64))


@pytest.mark.parametrize("shape", [(257, 301), (64, 61), (9, 91)])
def test_production_kernel_independent_of_row_chunks_and_near_exact(monkeypatch, shape):
    b, h, q = _wavy(shape, 3 * sum(shape))
    exact, s_exact, _ = _run(monkeypatch, {"SOILB200_FV_EXACT": "1"}, b, h, q)
    runs = [_run(monkeypatch, {"SOILB200_FV_ROWS": rows}, b, h, q) for rows in ("1", "3", "64")]
    for state, subs, _ in runs:
        assert subs == s_exact
        assert np.array_equal(state.h_m, runs[0][0].h_m)
        assert np.array_equal(state.q_m2_s, runs[0][0].q_m2_s)
    assert np.abs(runs[0][0].h_m - exact.h_m).max() <= 1.0e-7
