"""Import shim: exposes the package directory
``iron-soil-physical-simulation-algorithom-for-isaac-sim_b200/`` (whose name is
not a Python identifier) under the import name ``soilb200``."""

import importlib.util as _ilu
import sys as _sys
from pathlib import Path as _Path

_PKG_DIR = _Path(__file__).resolve().parent / "iron-soil-physical-simulation-algorithom-for-isaac-sim_b200"
_spec = _ilu.spec_from_file_location(
    "soilb200", _PKG_DIR / "__init__.py", submodule_search_locations=[str(_PKG_DIR)])
_mod = _ilu.module_from_spec(_spec)
_sys.modules["soilb200"] = _mod
_spec.loader.exec_module(_mod)
