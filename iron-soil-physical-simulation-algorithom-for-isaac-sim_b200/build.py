"""Build recipe for ``libsoilb200.so`` (sm_100a), in-tree next to this file.

``python -m`` is not needed: ``build_library()`` is called by the repository's
``__graft_entry__.build()`` and by ``soilb200._lib`` only to report a missing
library (it never builds implicitly at import time).
"""

from __future__ import annotations

import os
import shutil
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
INCLUDE = HERE.parent / "include"
LIB_NAME = "libsoilb200.so"

# -fmad=false: every float/double operation is a separately rounded IEEE op,
# which the parity instantiation and the fixed-point CPU mirror rely on.
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17", "-fmad=false",
    "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC", "-shared",
]


def nvcc_path() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found; the soilb200 library needs the CUDA toolkit to build")
    return cand


def sources() -> list[Path]:
    return [CSRC / "soilb200.cu"]


def build_library(verbose: bool = False, extra_flags: list[str] | None = None) -> Path:
    out = HERE / LIB_NAME
    deps = list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
    if out.exists() and all(out.stat().st_mtime >= d.stat().st_mtime for d in deps):
        return out
    tmp = out.with_suffix(".so.tmp")
    cmd = [nvcc_path(), *NVCC_FLAGS, *(extra_flags or []), f"-I{INCLUDE}",
           *[str(s) for s in sources()], "-o", str(tmp)]
    if verbose:
        print(" ".join(cmd))
    env = dict(os.environ)
    subprocess.run(cmd, check=True, env=env)
    os.replace(tmp, out)
    return out


if __name__ == "__main__":
    print(build_library(verbose=True))
