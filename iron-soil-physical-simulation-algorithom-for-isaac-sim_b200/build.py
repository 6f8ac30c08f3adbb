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

# soilb200.cu: -fmad=false -- every float/double operation is a separately
# rounded IEEE op, which the FP64 parity instantiations and the fixed-point CPU
# mirror rely on.  sb_fv_fast.cu (the production FX32 substep kernel) is
# compiled with FMA contraction.  Each translation unit becomes an object file
# under _build/, then both are linked into the shared library.
COMMON_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC",
]
UNITS = {
    "soilb200.cu": ["-fmad=false"],
    "sb_fv_fast.cu": ["-fmad=true"],
}
NVCC_FLAGS = COMMON_FLAGS  # kept for callers that print the flags


def nvcc_path() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found; the soilb200 library needs the CUDA toolkit to build")
    return cand


def sources() -> list[Path]:
    return [CSRC / name for name in UNITS]


def build_library(verbose: bool = False, extra_flags: list[str] | None = None) -> Path:
    out = HERE / LIB_NAME
    deps = list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
    deps.append(Path(__file__))
    if out.exists() and all(out.stat().st_mtime >= d.stat().st_mtime for d in deps):
        return out
    objdir = HERE.parent / "_build"
    objdir.mkdir(exist_ok=True)
    nvcc = nvcc_path()
    env = dict(os.environ)
    objs = []
    for name, flags in UNITS.items():
        obj = objdir / (Path(name).stem + ".o")
        cmd = [nvcc, *COMMON_FLAGS, *flags, *(extra_flags or []), f"-I{INCLUDE}", "-c",
               str(CSRC / name), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True, env=env)
        objs.append(str(obj))
    tmp = out.with_suffix(".so.tmp")
    cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", *objs, "-o", str(tmp)]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True, env=env)
    os.replace(tmp, out)
    return out


if __name__ == "__main__":
    print(build_library(verbose=True))
