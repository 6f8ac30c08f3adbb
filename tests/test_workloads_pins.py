"""CPU pins of the synthetic workload generators against the reference.

``workloads.fractal_perlin_noise`` restates the reference's training-patch
generator ``slope_model.fractal_perlin_noise`` (slope_model.py:77-129); the
golden fixture ``tests/golden/fractal.npz`` holds that function's own output
(written by ``tests/golden/make_golden.py --fractal``).  The restatement
evaluates the same expressions in a different order, so the bound is a few
units in the last place (1e-14 on fields scaled to max |value| = 1).
"""

import numpy as np
import pytest

from soilb200 import workloads

from conftest import GOLDEN


def test_fractal_perlin_noise_matches_reference_generator():
    g = np.load(GOLDEN / "fractal.npz")
    for k in range(int(g["count"])):
        nx, ny, seed = (int(v) for v in g[f"{k}/args"])
        base_cells, octaves = (int(v) for v in g[f"{k}/kw"])
        persistence, lacunarity = (float(v) for v in g[f"{k}/kwf"])
        got = workloads.fractal_perlin_noise(nx, ny, seed, base_cells=base_cells,
                                             octaves=octaves, persistence=persistence,
                                             lacunarity=lacunarity)
        want = g[f"{k}/noise"]
        assert got.shape == want.shape
        assert np.abs(got - want).max() <= 1e-14, k


def test_fractal_noise_validation_and_config3_patch():
    with pytest.raises(ValueError, match="at least 2"):
        workloads.fractal_perlin_noise(1, 5, 0)
    with pytest.raises(ValueError, match="positive"):
        workloads.fractal_perlin_noise(5, 5, 0, octaves=0)
    p = workloads.config3_patch(11)
    assert p.shape == (128, 128) and p.min() == 0.0
    # steepest neighbour slope lies in [tan 45, tan 60]
    dx = 0.05
    diag = np.hypot(dx, dx)
    s = max(np.abs(np.diff(p, axis=0)).max() / dx, np.abs(np.diff(p, axis=1)).max() / dx,
            np.abs(p[1:, 1:] - p[:-1, :-1]).max() / diag,
            np.abs(p[1:, :-1] - p[:-1, 1:]).max() / diag)
    assert np.tan(np.deg2rad(45.0)) - 1e-9 <= s <= np.tan(np.deg2rad(60.0)) + 1e-9
