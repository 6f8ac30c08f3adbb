"""Seeded synthetic workloads of the benchmark configurations.

No public dataset is involved: every terrain is generated from
``numpy.random.default_rng(seed)``.

* config 0 -- 256^2, dx 0.05 m: z_base = 10 deg x-tilted plane + 8 Gaussian
  bumps (A ~ U[0.05, 0.3] m, sigma ~ U[0.2, 1.0] m); b_eff = z_base; centred
  Gaussian mound h (peak 0.4 m, sigma 1.5 m); q = 0.  g 9.81, mu tan 35 deg,
  K 0.45, CFL 0.4, dt 1/60 s, repose relaxation 35 deg every step.
* config 1 -- 701^2, dx 0.05 m: 6-octave value-noise pile (amplitude 2 m,
  persistence 0.5) in b_eff, z_base = 0, h = 0; a bucket cut (1.8 m wide
  footprint moving 6 m in a straight line at 0.5 m/s) entrains resting
  material down to 0.4 m below the initial surface; labelling at 38 deg,
  8-connected; 10 s simulated.
* config 2 -- 512 patches (seeds 1000 + i) with sides from
  {64, 96, 128, 192, 256, 384, 512} and aspect <= 2:1, each a config-0-style
  terrain (10 deg tilt + 8 bumps) with a mound of mobile material at a seeded
  position; every patch takes its own CFL substeps.
* config 3 -- 128^2 training patches (seed i): the reference's fractal
  gradient noise (``fractal_perlin_noise``) steepened to a maximum neighbour
  slope of U[45, 60] deg, relaxed to 35 deg by the plain sweep.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np


def config0_terrain(n: int = 256, seed: int = 0, dx: float = 0.05):
    rng = np.random.default_rng(seed)
    ys, xs = np.indices((n, n), dtype=np.float64)
    x, y = xs * dx, ys * dx
    z = np.tan(np.deg2rad(10.0)) * x
    for _ in range(8):
        amp = rng.uniform(0.05, 0.3)
        sig = rng.uniform(0.2, 1.0)
        cx, cy = rng.uniform(0.0, n * dx, size=2)
        z = z + amp * np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2.0 * sig * sig))
    c = (n - 1) * dx / 2.0
    h = 0.4 * np.exp(-((x - c) ** 2 + (y - c) ** 2) / (2.0 * 1.5 ** 2))
    return {"z_base": z.copy(), "b_eff": z.copy(), "h": h, "q": np.zeros((n, n, 2))}


def value_noise(shape, cells: int, rng: np.random.Generator) -> np.ndarray:
    """Lattice value noise in [0, 1] with quintic interpolation."""
    ny, nx = shape
    lattice = rng.random((cells + 1, cells + 1))
    u = np.linspace(0.0, cells, nx, endpoint=False) + 0.5 * cells / nx
    v = np.linspace(0.0, cells, ny, endpoint=False) + 0.5 * cells / ny
    iu = np.minimum(u.astype(int), cells - 1)
    iv = np.minimum(v.astype(int), cells - 1)
    fu = u - iu
    fv = v - iv
    su = fu ** 3 * (fu * (fu * 6.0 - 15.0) + 10.0)
    sv = fv ** 3 * (fv * (fv * 6.0 - 15.0) + 10.0)
    a = lattice[iv[:, None], iu[None, :]]
    b = lattice[iv[:, None], iu[None, :] + 1]
    c = lattice[iv[:, None] + 1, iu[None, :]]
    d = lattice[iv[:, None] + 1, iu[None, :] + 1]
    top = a + (b - a) * su[None, :]
    bot = c + (d - c) * su[None, :]
    return top + (bot - top) * sv[:, None]


def noise_pile(n: int = 701, seed: int = 1, dx: float = 0.05, amplitude: float = 2.0,
               octaves: int = 6, persistence: float = 0.5, base_cells: int = 12) -> np.ndarray:
    """2 m pile: parabolic envelope times (0.25 + 0.75 * fBm); with 12 base cells
    the finest octave has ~0.2 m features, so ~0.1% of cells exceed 38 deg
    (fragmented failure zones) and ~1% exceed 30 deg."""
    rng = np.random.default_rng(seed)
    acc = np.zeros((n, n))
    weight = 0.0
    amp = 1.0
    for o in range(octaves):
        acc += amp * value_noise((n, n), base_cells * 2 ** o, rng)
        weight += amp
        amp *= persistence
    fbm = acc / weight
    ys, xs = np.indices((n, n), dtype=np.float64)
    c = (n - 1) / 2.0
    r = np.hypot(xs - c, ys - c) / (0.5 * n)
    envelope = np.clip(1.0 - r * r, 0.0, 1.0)
    return amplitude * envelope * (0.25 + 0.75 * fbm)


@dataclass
class BucketCut:
    """Straight-line bucket cut entraining resting material (config 1).

    The footprint is ``width`` m across and ``length`` m along the path; its
    leading edge travels ``travel`` m at ``speed`` m/s from ``start`` along
    unit ``heading``.  Inside the footprint the resting surface is cut down to
    ``depth`` m below the initial surface (entrainment, b_eff + h invariant).
    """

    shape: tuple
    dx: float
    initial_surface: np.ndarray
    start: tuple = (8.0, 17.5)
    heading: tuple = (1.0, 0.0)
    width: float = 1.8
    length: float = 0.3
    travel: float = 6.0
    speed: float = 0.5
    depth: float = 0.4

    def __post_init__(self) -> None:
        ny, nx = self.shape
        ys, xs = np.indices((ny, nx), dtype=np.float64)
        self._x = xs.ravel() * self.dx
        self._y = ys.ravel() * self.dx
        hx, hy = self.heading
        norm = float(np.hypot(hx, hy))
        self._h = (hx / norm, hy / norm)
        self._target = (np.asarray(self.initial_surface, dtype=np.float64).ravel() - self.depth)

    def footprint(self, t_s: float):
        """(flat indices, target surfaces) of the cells under the bucket at time t."""
        s = min(self.speed * max(t_s, 0.0), self.travel)
        hx, hy = self._h
        px = self._x - self.start[0]
        py = self._y - self.start[1]
        along = px * hx + py * hy
        across = -px * hy + py * hx
        inside = (along <= s) & (along >= s - self.length) & (np.abs(across) <= 0.5 * self.width)
        idx = np.flatnonzero(inside).astype(np.int32)
        return idx, self._target[idx]

    @property
    def duration_s(self) -> float:
        return self.travel / self.speed


def config1(n: int = 701, seed: int = 1, dx: float = 0.05):
    b = noise_pile(n, seed, dx)
    cut = BucketCut((n, n), dx, b, start=(0.3 * n * dx, 0.5 * n * dx))
    return {"b_eff": b, "z_base": np.zeros((n, n)), "cut": cut}


C2_SIDES = (64, 96, 128, 192, 256, 384, 512)


def config2_patch(i: int, dx: float = 0.05):
    """Patch i of config 2: (b_eff, h, q) with shape (ny, nx), seed 1000 + i."""
    rng = np.random.default_rng(1000 + i)
    ny = int(rng.choice(C2_SIDES))
    nx = int(rng.choice([s for s in C2_SIDES if max(s, ny) <= 2 * min(s, ny)]))
    ys, xs = np.indices((ny, nx), dtype=np.float64)
    x, y = xs * dx, ys * dx
    z = np.tan(np.deg2rad(10.0)) * x
    for _ in range(8):
        amp = rng.uniform(0.05, 0.3)
        sig = rng.uniform(0.2, 1.0)
        cx = rng.uniform(0.0, nx * dx)
        cy = rng.uniform(0.0, ny * dx)
        z = z + amp * np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2.0 * sig * sig))
    mx = rng.uniform(0.2, 0.8) * (nx - 1) * dx
    my = rng.uniform(0.2, 0.8) * (ny - 1) * dx
    sm = min(1.5, 0.2 * min(ny, nx) * dx)
    h = 0.4 * np.exp(-((x - mx) ** 2 + (y - my) ** 2) / (2.0 * sm * sm))
    return z, h, np.zeros((ny, nx, 2))


def config2(n_patches: int = 512, dx: float = 0.05):
    """The config-2 patch list [(b_eff, h, q), ...]."""
    return [config2_patch(i, dx) for i in range(n_patches)]


def fractal_perlin_noise(nx: int, ny: int, seed=None, *, base_cells: int = 3, octaves: int = 5,
                         persistence: float = 0.52, lacunarity: float = 2.0) -> np.ndarray:
    """Seeded fractal gradient (Perlin) noise: the generator of the reference's
    training patches (``slope_model.fractal_perlin_noise``, slope_model.py:77-129).

    Same parameters and the same random draws (one ``(m+1, m+1)`` array of
    gradient angles per octave from ``default_rng(seed)``, m = round(cells of
    that octave)), so a seed gives the reference's field: per octave, unit
    gradients on an m x m lattice over [0, 1]^2, the dot products with the
    offsets to the four lattice corners blended by the quintic fade
    6t^5 - 15t^4 + 10t^3, octave weights normalised, then the field scaled to
    max |value| = 1.  Indexed [x, y] with shape (nx, ny), as the reference.
    """
    if nx < 2 or ny < 2:
        raise ValueError("noise dimensions must be at least 2")
    if base_cells < 1 or octaves < 1:
        raise ValueError("base_cells and octaves must be positive")
    rng = np.random.default_rng(seed)
    px = np.linspace(0.0, 1.0, nx)
    py = np.linspace(0.0, 1.0, ny)
    field = np.zeros((nx, ny))
    total = 0.0
    amp = 1.0
    freq = float(base_cells)

    def fade(t):
        return t * t * t * (t * (t * 6.0 - 15.0) + 10.0)

    for _ in range(octaves):
        m = max(1, int(round(freq)))
        theta = rng.uniform(0.0, 2.0 * np.pi, (m + 1, m + 1))
        gcos, gsin = np.cos(theta), np.sin(theta)
        cx = np.minimum((px * m).astype(int), m - 1)
        cy = np.minimum((py * m).astype(int), m - 1)
        ox = px * m - cx
        oy = py * m - cy
        ox[-1] = 1.0
        oy[-1] = 1.0
        X, Y = cx[:, None], cy[None, :]
        U, V = ox[:, None], oy[None, :]
        corner = {}
        for di in (0, 1):
            for dj in (0, 1):
                corner[di, dj] = gcos[X + di, Y + dj] * (U - di) + gsin[X + di, Y + dj] * (V - dj)
        fu, fv = fade(U), fade(V)
        lo = corner[0, 0] + fu * (corner[1, 0] - corner[0, 0])
        hi = corner[0, 1] + fu * (corner[1, 1] - corner[0, 1])
        field += amp * (lo + fv * (hi - lo))
        total += amp
        amp *= persistence
        freq *= lacunarity
    field /= max(total, 1e-12)
    peak = float(np.abs(field).max())
    return field / peak if peak > 0.0 else field


def config3_patch(i: int, n: int = 128, dx: float = 0.05) -> np.ndarray:
    """Training patch i of config 3: the reference generator's fractal noise
    (seed i) steepened to a seeded 45-60 deg maximum neighbour slope and
    shifted to non-negative heights."""
    h = fractal_perlin_noise(n, n, seed=i)
    target = np.tan(np.deg2rad(np.random.default_rng([i, 3]).uniform(45.0, 60.0)))
    # steepest of the four neighbour directions (slope_model.max_neighbor_slope's measure)
    diag = np.hypot(dx, dx)
    s = max(np.abs(np.diff(h, axis=0)).max() / dx, np.abs(np.diff(h, axis=1)).max() / dx,
            np.abs(h[1:, 1:] - h[:-1, :-1]).max() / diag, np.abs(h[1:, :-1] - h[:-1, 1:]).max() / diag)
    return (h - h.min()) * (target / s)


class SiteCut:
    """A config-1 bucket cut evaluated on a local window of a large grid
    (same footprint rule as ``BucketCut``; cost proportional to the window)."""

    def __init__(self, shape, dx: float, initial_surface: np.ndarray, start, heading,
                 width: float = 1.8, length: float = 0.3, travel: float = 6.0,
                 speed: float = 0.5, depth: float = 0.4) -> None:
        ny, nx = shape
        self.nx = nx
        self.speed, self.travel, self.length, self.width = speed, travel, length, width
        self.start = (float(start[0]), float(start[1]))
        hx, hy = heading
        norm = float(np.hypot(hx, hy))
        self._h = (hx / norm, hy / norm)
        reach = travel + width + length
        c0 = max(0, int((self.start[0] - reach) / dx) - 1)
        c1 = min(nx, int((self.start[0] + reach) / dx) + 2)
        r0 = max(0, int((self.start[1] - reach) / dx) - 1)
        r1 = min(ny, int((self.start[1] + reach) / dx) + 2)
        rows, cols = np.indices((r1 - r0, c1 - c0))
        rows, cols = rows + r0, cols + c0
        self._flat = (rows * nx + cols).ravel().astype(np.int64)
        px = cols.ravel() * dx - self.start[0]
        py = rows.ravel() * dx - self.start[1]
        self._along = px * self._h[0] + py * self._h[1]
        self._across = -px * self._h[1] + py * self._h[0]
        self._target = np.asarray(initial_surface, np.float64).ravel()[self._flat] - depth

    def footprint(self, t_s: float):
        s = min(self.speed * max(t_s, 0.0), self.travel)
        inside = ((self._along <= s) & (self._along >= s - self.length)
                  & (np.abs(self._across) <= 0.5 * self.width))
        return self._flat[inside], self._target[inside]


    def swept(self):
        """Flat indices of every cell the footprint covers over the whole
        travel (leading edge from 0 to ``travel``, trailing edge ``length``
        behind it) and their target surfaces."""
        inside = ((self._along <= self.travel) & (self._along >= -self.length)
                  & (np.abs(self._across) <= 0.5 * self.width))
        return self._flat[inside], self._target[inside]


def site_after_cuts(cfg) -> np.ndarray:
    """b_eff of a config-4 site after all its cuts have run their full travel
    (every swept cell lowered to its target surface)."""
    b = cfg["b_eff"].copy()
    flat = b.reshape(-1)
    for cut in cfg["cuts"]:
        idx, tgt = cut.swept()
        flat[idx] = np.minimum(flat[idx], tgt)
    return b


def merged_footprint(cuts, t_s: float):
    """Union of several cuts' footprints: each cell once, at its lowest target."""
    parts = [c.footprint(t_s) for c in cuts]
    idx = np.concatenate([p[0] for p in parts]) if parts else np.zeros(0, np.int64)
    tgt = np.concatenate([p[1] for p in parts]) if parts else np.zeros(0)
    if idx.size == 0:
        return idx.astype(np.int32), tgt
    order = np.lexsort((tgt, idx))
    idx, tgt = idx[order], tgt[order]
    first = np.ones(idx.size, bool)
    first[1:] = idx[1:] != idx[:-1]
    return idx[first].astype(np.int32), tgt[first]


def config4(n: int = 4096, seed: int = 4, dx: float = 0.05, n_cuts: int = 64):
    b = noise_pile(n, seed, dx, base_cells=max(12, round(12 * n / 701)))
    rng = np.random.default_rng(seed + 1)
    cuts = []
    for _ in range(n_cuts):
        x, y = rng.uniform(0.15, 0.85, size=2) * (n - 1) * dx
        ang = rng.uniform(0.0, 2.0 * np.pi)
        cuts.append(SiteCut((n, n), dx, b, (x, y), (np.cos(ang), np.sin(ang))))
    return {"b_eff": b, "z_base": np.zeros((n, n)), "cuts": cuts}

