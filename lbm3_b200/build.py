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

# (source, object, extra defines): step.cu is compiled once per population
# storage type and kernel family (LBM3_STEP_PART) so the kernel sets build in
# parallel; the heaviest unit bounds the build time
STEP_STORAGES = [("f32", 0), ("f16", 1), ("bf16", 2), ("f64", 3)]
STEP_PARTS = [1, 2, 3, 4]
SOURCES = [
    # (each unit instantiates only its family, so helpers of the other
    # families are unreferenced there: diagnostic 177 is expected)
    *[("step.cu", f"step_{name}_p{part}.o",
       [f"-DLBM3_STEP_STORAGE={code}", f"-DLBM3_STEP_PART={part}", "-diag-suppress=177"])
      for part in STEP_PARTS for name, code in STEP_STORAGES],
    ("step_dispatch.cu", "step_dispatch.o", []),
    ("api.cu", "api.o", []),
    ("builder.cpp", "builder.o", []),
    ("geometry.cpp", "geometry.o", []),
    ("energy_noalloc.cu", "energy_noalloc.o", []),
]
HEADERS = ["lattice.h", "cumulant.cuh", "interface.cuh", "step.cuh", "step_launch.h", "builder.h", "geometry.h", "mbbc.h",
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
    objs, jobs = [], []
    for src, obj, defines in SOURCES:
        s = CSRC / src
        o = OBJ_DIR / obj
        objs.append(o)
        if force or _stale(o, [s, *headers, Path(__file__)]):
            jobs.append([_nvcc(), *flags, *defines, "-c", str(s), "-o", str(o)])
    if jobs:
        from concurrent.futures import ThreadPoolExecutor

        def run(cmd):
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)

        with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as pool:
            list(pool.map(run, jobs))
    if force or _stale(LIB, objs):
        cmd = [_nvcc(), *ARCH, "-shared", *map(str, objs), "-o", str(LIB), "-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
