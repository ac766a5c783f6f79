"""Builds the runtime's shared library in-tree: neuroevolutionary-wordle_b200/libnwg.so.

Every CUDA source under csrc/ is compiled for sm_100a only (no other architecture, no JIT
fallback) into one shared library exporting the C ABI declared in include/nwg_capi.h.
"""
from __future__ import annotations

import os
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
CSRC = HERE / "csrc"
LIB = HERE / "libnwg.so"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-shared", "--expt-relaxed-constexpr"]


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def headers() -> list[Path]:
    return sorted(CSRC.glob("*.cuh")) + [ROOT / "include" / "nwg_capi.h"]


def stale() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    return any(p.stat().st_mtime > t for p in sources() + headers())


def build(force: bool = False, verbose_ptxas: bool = False) -> Path:
    if not force and not stale():
        return LIB
    cmd = [NVCC, *ARCH, *FLAGS, "-I", str(ROOT / "include"), *map(str, sources()), "-o", str(LIB)]
    if verbose_ptxas:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    import sys

    build(force=True, verbose_ptxas="-v" in sys.argv)
