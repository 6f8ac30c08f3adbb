"""C-ABI surface checks that need no GPU: the library loads and exports every
symbol declared in include/soilb200.h; host-side validation mirrors the
reference's ValueError behaviour."""

import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

import soilb200
from soilb200 import _lib

ROOT = Path(__file__).resolve().parents[1]


def _declared_symbols():
    text = (ROOT / "include" / "soilb200.h").read_text()
    # strip comments
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sb_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    declared = _declared_symbols()
    assert declared, "no declarations parsed"
    for name in declared:
        assert hasattr(lib, name), name
        assert name in _lib.exported_symbols(), f"{name} has no ctypes prototype"


def test_version_string():
    assert b"sm_100a" in _lib.load().sb_version()


def test_struct_layouts_match_compiled_library():
    lib = _lib.load()
    for name, struct in _lib.ABI_STRUCTS.items():
        assert lib.sb_sizeof(name.encode()) == ctypes.sizeof(struct), name
    assert lib.sb_sizeof(b"no_such_struct") == 0


def test_config_validation_matches_reference():
    with pytest.raises(ValueError, match="CFL must be <= 0.25"):
        soilb200.MobileV2Config(cfl=0.3)
    with pytest.raises(ValueError, match="finite/positive"):
        soilb200.MobileV2Config(dx_m=0.0)
    cfg = soilb200.MobileV2Config.unchecked(cfl=0.4)
    assert cfg.cfl == 0.4
    with pytest.raises(ValueError, match="shape mismatch"):
        soilb200.MobileV2State(np.zeros((3, 3)), np.zeros((3, 4)), np.zeros((3, 3, 2)))
    with pytest.raises(ValueError, match="nonnegative"):
        soilb200.MobileV2State(np.zeros((3, 3)), -np.ones((3, 3)), np.zeros((3, 3, 2)))


def test_quantization_choice_headroom():
    b = np.linspace(0.0, 2.0, 100).reshape(10, 10)
    k, datum = soilb200.choose_quantization(b, mobile=np.zeros((10, 10)))
    assert datum == pytest.approx(1.0)
    assert 2.0 ** (31 - k) >= 4.0 * 1.0  # 4x headroom over the 1 m half-span
    assert k <= 30


def test_missing_library_raises_backend_unavailable(monkeypatch, tmp_path):
    monkeypatch.setattr(_lib, "_LIB", None)
    monkeypatch.setenv("SOILB200_LIB", str(tmp_path / "absent.so"))
    with pytest.raises(soilb200.B200BackendUnavailable):
        _lib.load()
