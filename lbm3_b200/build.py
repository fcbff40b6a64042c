"""Build the in-tree CUDA library ``lbm3_b200/_lib/liblbm3_b200.so`` for sm_100a.

Run ``python -m lbm3_b200.build`` (or call :func:`build`).  nvcc cross-compiles
for B200 without a GPU; the resulting shared library travels with the source
tree, so nothing is JIT-compiled at run time.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIB_DIR = PKG / "_lib"
LIB = LIB_DIR / "liblbm3_b200.so"
OBJ_DIR = PKG / "_build"

SOURCES = ["step.cu", "api.cu", "builder.cpp", "geometry.cpp", "energy_noalloc.cu"]
HEADERS = ["lattice.h", "cumulant.cuh", "step.cuh", "step_launch.h", "builder.h", "geometry.h", "mbbc.h",
           "mbbc_tables.h", "energy_noalloc.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
]


def _nvcc() -> str:
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    cand = Path(cuda) / "bin" / "nvcc"
    return str(cand) if cand.exists() else "nvcc"


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def build(verbose: bool = False, force: bool = False, extra_flags=None) -> Path:
    """Compile every CUDA/C++ source and link the shared library; returns its path."""
    LIB_DIR.mkdir(exist_ok=True)
    OBJ_DIR.mkdir(exist_ok=True)
    headers = [CSRC / h for h in HEADERS] + [PKG.parent / "include" / "lbm3_b200.h"]
    flags = NVCC_FLAGS + list(extra_flags or [])
    objs = []
    for src in SOURCES:
        s = CSRC / src
        o = OBJ_DIR / (src + ".o")
        objs.append(o)
        if force or _stale(o, [s, *headers, Path(__file__)]):
            cmd = [_nvcc(), *flags, "-c", str(s), "-o", str(o)]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    if force or _stale(LIB, objs):
        cmd = [_nvcc(), *ARCH, "-shared", *map(str, objs), "-o", str(LIB), "-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
