"""Device-resident terrain grid: one ``sb_ctx`` (GPU fields + graphs) per grid.

Role of the reference's ``DeviceBulkState`` field store
(``runtime/bulk_state_authority.py:493-619``): fields are addressed by the
reference's names (``z_base``, ``b_eff``, ``mobile``, ``momentum_x``,
``momentum_y``, ``frontier_reached`` ...) and live on the device; host arrays
only cross at explicit upload/download boundaries.
"""

from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib

PRECISIONS = {"fp64": _lib.SB_FP64, "fx32": _lib.SB_FX32}


def choose_quantization(*support_fields, mobile=None) -> tuple[int, float]:
    """Pick (height_exponent k, datum) for the 32-bit fixed-point precision.

    ``b_eff``/``z_base`` are stored as int32 multiples of 2**-k relative to the
    datum (mid-range of the supports); the largest k <= 30 is chosen that keeps
    4x headroom over the observed span, so typical terrains get a quantum of
    1-4 nm (the quantum only sets the resolution of stored heights).
    """
    lo, hi = math.inf, -math.inf
    for f in support_fields:
        if f is None:
            continue
        a = np.asarray(f, dtype=np.float64)
        if a.size:
            lo = min(lo, float(np.min(a)))
            hi = max(hi, float(np.max(a)))
    if not math.isfinite(lo):
        lo, hi = 0.0, 0.0
    datum = 0.5 * (lo + hi)
    span = max(hi - datum, 1.0e-6)
    if mobile is not None:
        m = np.asarray(mobile, dtype=np.float64)
        if m.size:
            span = max(span, float(np.max(np.abs(m))))
    k = int(math.floor(math.log2(2.0 ** 29 / span)))
    return int(min(30, max(12, k))), float(datum)


class DeviceGrid:
    """Owns one context.  ``shape = (ny, nx)`` row-major, as ``TerrainGrid``."""

    def __init__(self, shape, dx_m: float, dy_m: float, *, precision: str = "fx32",
                 tile_size: int = 64, device: int = 0, height_exponent: int = 28,
                 datum_m: float = 0.0) -> None:
        if precision not in PRECISIONS:
            raise ValueError(f"[soilb200] precision must be one of {sorted(PRECISIONS)}")
        lib = _lib.load()
        self.shape = (int(shape[0]), int(shape[1]))
        self.dx = float(dx_m)
        self.dy = float(dy_m)
        self.precision = precision
        self.tile_size = int(tile_size)
        self.height_exponent = int(height_exponent)
        self.datum = float(datum_m)
        desc = _lib.GridDesc(int(device), self.shape[0], self.shape[1], self.dx, self.dy,
                             self.tile_size, PRECISIONS[precision], self.height_exponent,
                             self.datum)
        ctx = C.c_void_p()
        rc = lib.sb_ctx_create(C.byref(desc), C.byref(ctx))
        self._ctx = ctx
        if rc != _lib.SB_OK:
            msg = _lib.last_error(ctx)
            lib.sb_ctx_destroy(ctx)
            self._ctx = None
            if rc == _lib.SB_ERR_BAD_ARG:
                raise ValueError(msg)
            raise _lib.B200BackendUnavailable(msg or "[soilb200] context creation failed")

    @property
    def ctx(self):
        if self._ctx is None:
            raise RuntimeError("[soilb200] grid context is closed")
        return self._ctx

    @property
    def quantum(self) -> float:
        return 2.0 ** (-self.height_exponent)

    @property
    def size(self) -> int:
        return self.shape[0] * self.shape[1]

    def close(self) -> None:
        if getattr(self, "_ctx", None) is not None:
            _lib.load().sb_ctx_destroy(self._ctx)
            self._ctx = None

    def __del__(self):  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:
            pass

    def upload(self, name: str, values) -> None:
        lib = _lib.load()
        if name not in _lib.FIELD:
            raise ValueError(f"[soilb200] unknown field {name!r}")
        if name in _lib.INT_FIELDS:
            arr = np.ascontiguousarray(values, dtype=np.int32)
            if arr.shape != self.shape:
                raise ValueError(f"[soilb200] {name} shape {arr.shape} != {self.shape}")
            _lib.check(self.ctx, lib.sb_upload_i32(self.ctx, _lib.FIELD[name], arr.ctypes.data),
                       "upload")
            return
        arr = np.ascontiguousarray(values, dtype=np.float64)
        if arr.shape != self.shape:
            raise ValueError(f"[soilb200] {name} shape {arr.shape} != {self.shape}")
        if not np.all(np.isfinite(arr)):
            raise ValueError(f"[soilb200] {name} must be finite")
        _lib.check(self.ctx, lib.sb_upload(self.ctx, _lib.FIELD[name], arr.ctypes.data), "upload")

    def upload_ptr(self, name: str, host_ptr: int) -> None:
        """Upload from a raw host pointer (e.g. pinned memory) of ny*nx float64."""
        lib = _lib.load()
        _lib.check(self.ctx, lib.sb_upload(self.ctx, _lib.FIELD[name], C.c_void_p(host_ptr)),
                   "upload")

    def download_ptr(self, name: str, host_ptr: int) -> None:
        lib = _lib.load()
        _lib.check(self.ctx, lib.sb_download(self.ctx, _lib.FIELD[name], C.c_void_p(host_ptr)),
                   "download")

    def download(self, name: str) -> np.ndarray:
        lib = _lib.load()
        if name not in _lib.FIELD:
            raise ValueError(f"[soilb200] unknown field {name!r}")
        if name in _lib.INT_FIELDS:
            out = np.empty(self.shape, dtype=np.int32)
            _lib.check(self.ctx, lib.sb_download_i32(self.ctx, _lib.FIELD[name], out.ctypes.data),
                       "download")
            return out
        out = np.empty(self.shape, dtype=np.float64)
        _lib.check(self.ctx, lib.sb_download(self.ctx, _lib.FIELD[name], out.ctypes.data),
                   "download")
        return out

    def synchronize(self) -> None:
        _lib.check(self.ctx, _lib.load().sb_synchronize(self.ctx), "synchronize")

    def stream_handle(self) -> int:
        """Integer cudaStream_t of this context (e.g. for torch.cuda.ExternalStream)."""
        return int(_lib.load().sb_stream(self.ctx) or 0)

    def kernel_launches(self) -> int:
        return int(_lib.load().sb_kernel_launch_count(self.ctx))
