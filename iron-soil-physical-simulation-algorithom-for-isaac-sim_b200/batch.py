"""Batched Mobile V2 patches: many independent terrain grids per launch.

A dig simulator runs many environments at once, each with its own terrain
patch of its own size.  ``B200PatchBatch`` keeps all of them resident on one
GPU and advances every patch by one physics step per :meth:`step` call, each
patch with its own CFL substeps (the reference steps one grid per call:
``MobileV2ReferenceSolver.step``, experimental/mobile_v2_reference.py:191-314,
and ``WarpProductionMobileV2Solver.step_resident``,
bulk_interaction/warp_mobile_v2.py:188-245).  The arithmetic is the FX32
production path of :class:`soilb200.B200MobileV2Solver`, so every patch ends
bit-identical to stepping it alone with that solver.
"""

from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np

from . import _lib
from .grid import choose_quantization
from .mobile_v2 import (MobileV2Config, MobileV2State, MobileV2Step, _device_index, build_step,
                        mobile_params)

_FIELDS = ("z_base", "b_eff", "mobile", "momentum_x", "momentum_y")


class B200PatchBatch:
    """Resident batch of terrain patches (FX32), stepped together.

    ``states`` are the patches' initial ``MobileV2State`` (each with its own
    shape); ``z_base`` optionally gives each patch's non-erodible base (default
    ``b_eff``).  Every patch gets its own height quantum from its initial
    support and mobile heights (``choose_quantization``).
    """

    def __init__(self, states: Sequence[MobileV2State], config: MobileV2Config | None = None, *,
                 z_base: Sequence[np.ndarray] | None = None, device=0) -> None:
        if not states:
            raise ValueError("[soilb200] a batch needs at least one patch")
        self.config = config or MobileV2Config()
        self.device = _device_index(device)
        self.shapes = [tuple(np.shape(s.h_m)) for s in states]
        self.quantization = []
        descs = (_lib.PatchDesc * len(states))()
        for i, s in enumerate(states):
            k, datum = choose_quantization(s.b_eff_m, mobile=s.h_m)
            self.quantization.append((k, datum))
            ny, nx = self.shapes[i]
            descs[i] = _lib.PatchDesc(ny, nx, float(self.config.dx_m), float(self.config.dy_m),
                                      int(k), 0, float(datum))
        lib = _lib.load()
        handle = C.c_void_p()
        rc = lib.sb_batch_create(self.device, len(states), descs, C.byref(handle))
        self._batch = handle
        if rc != _lib.SB_OK:
            msg = _lib.batch_last_error(handle) if handle.value else ""
            lib.sb_batch_destroy(handle)
            self._batch = None
            if rc == _lib.SB_ERR_BAD_ARG:
                raise ValueError(msg or "[soilb200] invalid patch description")
            _lib.check(None, rc, "batch create", batch=None)
        self._stats = (_lib.MobileStats * len(states))()
        for i, s in enumerate(states):
            self.upload(i, "b_eff", s.b_eff_m)
            self.upload(i, "z_base", s.b_eff_m if z_base is None else z_base[i])
            self.upload(i, "mobile", s.h_m)
            q = np.asarray(s.q_m2_s, dtype=np.float64)
            self.upload(i, "momentum_x", q[..., 0])
            self.upload(i, "momentum_y", q[..., 1])

    # --------------------------------------------------------------- fields
    @property
    def n_patches(self) -> int:
        return len(self.shapes)

    def _check(self, rc: int, what: str) -> None:
        _lib.check(None, rc, what, batch=self._batch)

    def upload(self, patch: int, name: str, values) -> None:
        if name not in _FIELDS:
            raise ValueError(f"[soilb200] {name!r} is not a patch field")
        arr = np.ascontiguousarray(values, dtype=np.float64)
        if arr.shape != self.shapes[patch]:
            raise ValueError(f"[soilb200] patch {patch} {name} shape {arr.shape} != "
                             f"{self.shapes[patch]}")
        self._check(_lib.load().sb_batch_upload(self._batch, int(patch), _lib.FIELD[name],
                                                arr.ctypes.data), "batch upload")

    def download(self, patch: int, name: str) -> np.ndarray:
        if name not in _FIELDS:
            raise ValueError(f"[soilb200] {name!r} is not a patch field")
        out = np.empty(self.shapes[patch], dtype=np.float64)
        self._check(_lib.load().sb_batch_download(self._batch, int(patch), _lib.FIELD[name],
                                                  out.ctypes.data), "batch download")
        return out

    def state(self, patch: int) -> MobileV2State:
        q = np.stack([self.download(patch, "momentum_x"), self.download(patch, "momentum_y")],
                     axis=-1)
        return MobileV2State(self.download(patch, "b_eff"), self.download(patch, "mobile"), q)

    # ---------------------------------------------------------- tile shapes
    @property
    def rows(self) -> list[int]:
        out = (C.c_int * self.n_patches)()
        self._check(_lib.load().sb_batch_get_rows(self._batch, out), "batch rows")
        return list(out)

    @rows.setter
    def rows(self, values: Sequence[int]) -> None:
        arr = (C.c_int * self.n_patches)(*[int(v) for v in values])
        self._check(_lib.load().sb_batch_set_rows(self._batch, arr), "batch rows")

    def autotune(self, dt_s: float, trials: int = 2) -> float:
        """Pick rows per warp strip for each group of equal-height patches by
        timing the candidates on the live state (put back after every trial).
        Returns the substep-loop milliseconds of one step with the choice."""
        best = C.c_double()
        self._check(_lib.load().sb_batch_autotune(self._batch, float(dt_s),
                                                  mobile_params(self.config), int(trials),
                                                  C.byref(best)), "batch autotune")
        return float(best.value)

    # ----------------------------------------------------------------- step
    def step_stats(self, dt_s: float) -> list[_lib.MobileStats]:
        """One physics step of every patch; returns the per-patch device records."""
        dt = float(dt_s)
        if not np.isfinite(dt) or dt <= 0.0:
            raise ValueError("dt must be finite/positive")
        self._check(_lib.load().sb_batch_step(self._batch, dt, mobile_params(self.config),
                                              self._stats), "batch step")
        return list(self._stats)

    def step(self, dt_s: float) -> list[MobileV2Step]:
        """One physics step of every patch, as the reference's step records
        (each patch's final state downloaded)."""
        stats = self.step_stats(dt_s)
        return [build_step(self.state(i), float(dt_s), st, self.config,
                           quantum=2.0 ** -self.quantization[i][0])
                for i, st in enumerate(stats)]

    def label(self, material, config=None) -> list:
        """Large-avalanche labelling of every patch's current state (yield +
        canonical union-find, as ``B200LargeAvalancheBridge.label`` on a
        single grid, without latches); returns one ``LabelStats`` per patch."""
        from .avalanche import B200LargeAvalancheBridge, LargeAvalancheTransitionConfig
        cfg = config or LargeAvalancheTransitionConfig()
        params = B200LargeAvalancheBridge.label_params(material, cfg, release=False)
        out = (_lib.LabelStats * self.n_patches)()
        self._check(_lib.load().sb_batch_label(self._batch, params, out), "batch label")
        return list(out)

    def labels(self, patch: int) -> np.ndarray:
        """Canonical labels of one patch after :meth:`label` (-1 = stable)."""
        ny, nx = self.shapes[patch]
        out = np.empty((ny, nx), dtype=np.int32)
        self._check(_lib.load().sb_batch_download_labels(self._batch, int(patch),
                                                          out.ctypes.data), "batch labels")
        return out

    def kernel_launches(self) -> int:
        return int(_lib.load().sb_batch_kernel_launch_count(self._batch))

    def stream_handle(self) -> int:
        return int(_lib.load().sb_batch_stream(self._batch) or 0)

    def close(self) -> None:
        if getattr(self, "_batch", None) is not None:
            _lib.load().sb_batch_destroy(self._batch)
            self._batch = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
