"""Builds libsadcs_gpu.so (sm_100a) in-tree with nvcc.

``python -m sadcs_b200.build`` or ``sadcs_b200.build.build_library()``. The library is a single
translation unit (csrc/sadcs_gpu.cu includes the phase headers), so the __constant__ cover tables
need no relocatable device code.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PACKAGE = Path(__file__).resolve().parent
ROOT = PACKAGE.parent
CSRC = PACKAGE / "csrc"
LIBDIR = PACKAGE / "lib"
LIBRARY = LIBDIR / "libsadcs_gpu.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for candidate in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if candidate and Path(candidate).exists():
            return candidate
    raise FileNotFoundError("nvcc not found (set NVCC or install the CUDA toolkit)")


def _sources():
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cuh")) + [ROOT / "include" / "sadcs_gpu.h"]


def _stale(target: Path, sources) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(s.stat().st_mtime > t for s in sources)


def build_library(force: bool = False, verbose: bool = False) -> Path:
    """Compiles csrc/sadcs_gpu.cu into lib/libsadcs_gpu.so if it is missing or stale."""
    LIBDIR.mkdir(exist_ok=True)
    if not force and not _stale(LIBRARY, _sources()):
        return LIBRARY
    cmd = [nvcc(), *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
           "-o", str(LIBRARY) + ".tmp", str(CSRC / "sadcs_gpu.cu")]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(str(LIBRARY) + ".tmp", LIBRARY)
    return LIBRARY


if __name__ == "__main__":
    print(build_library(force="--force" in sys.argv, verbose=True))
