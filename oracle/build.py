"""Build recipe for the oracle (test infrastructure only).

Outputs:
  oracle/_lib/libnwg_oracle.so  -- the CPU restatement (nwg_oracle.c), gcc
  oracle/_lib/libnwg_tape.so    -- GPU draw tapes for the oracle (nwg_tape.cu), nvcc sm_100a
  oracle/_ref/libref_host.so    -- the reference's host-callable code + episode loop harness
  oracle/_ref/libref_dev.so     -- the reference's device functions + harness kernels, sm_100a
  oracle/_ref/libref_ckpt.so    -- the reference's runtime (checkpoint format, capture, restore, resume), sm_100a
  oracle/_ref/shim_driver       -- tests/shim_driver.cu: a caller of the reference's slab_device API, linked
                                   against libnwg.so through include/nwg_slab_device_shim.hpp

The oracle/_ref libraries are compiled from the reference's own headers where they
lie (REFERENCE_ROOT/src); nothing is copied. They are only rebuilt when the reference
tree is present; elsewhere the prebuilt files are used as they are.
"""
from __future__ import annotations

import os
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB_DIR = HERE / "_lib"
REF_DIR = HERE / "_ref"
REFERENCE_ROOT = Path(os.environ.get("NWG_REFERENCE_ROOT", "/root/reference"))
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _run(cmd: list[str]) -> None:
    subprocess.run(cmd, check=True)


def _stale(target: Path, sources: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(s.stat().st_mtime > t for s in sources)


def build_oracle(force: bool = False) -> Path:
    LIB_DIR.mkdir(exist_ok=True)
    out = LIB_DIR / "libnwg_oracle.so"
    srcs = [HERE / "nwg_oracle.c", HERE / "nwg_oracle.h"]
    if force or _stale(out, srcs):
        _run(["gcc", "-O2", "-std=c11", "-Wall", "-Wextra", "-fPIC", "-shared", "-ffp-contract=off",
              str(HERE / "nwg_oracle.c"), "-o", str(out), "-lm"])
    return out


def build_tape(force: bool = False) -> Path:
    LIB_DIR.mkdir(exist_ok=True)
    out = LIB_DIR / "libnwg_tape.so"
    srcs = [HERE / "nwg_tape.cu"]
    if force or _stale(out, srcs):
        _run([NVCC, *ARCH, "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
              str(HERE / "nwg_tape.cu"), "-o", str(out)])
    return out


def reference_present() -> bool:
    return (REFERENCE_ROOT / "src" / "genetic_algorithm" / "device" / "slab_runtime.cu").exists()


def build_reference(force: bool = False) -> list[Path]:
    """Compile the reference's path from its own sources (skipped when they are absent)."""
    if not reference_present():
        return []
    REF_DIR.mkdir(exist_ok=True)
    inc = ["-I", str(REFERENCE_ROOT / "src")]
    host_out = REF_DIR / "libref_host.so"
    dev_out = REF_DIR / "libref_dev.so"
    if force or _stale(host_out, [HERE / "ref_host_harness.cu"]):
        # Host code only; -O3 without -march so the library runs on any x86-64 host.
        _run([NVCC, *ARCH, "-O3", "-std=c++20", *inc, "-Xcompiler", "-fPIC,-O3", "-shared",
              str(HERE / "ref_host_harness.cu"), "-o", str(host_out)])
    if force or _stale(dev_out, [HERE / "ref_dev_harness.cu"]):
        _run([NVCC, *ARCH, "-O3", "-std=c++20", *inc, "-Xcompiler", "-fPIC", "-shared",
              "-DNEUROEVOLUTION_PROJECT_SOURCE_DIR=\"/nonexistent\"",
              str(HERE / "ref_dev_harness.cu"), "-o", str(dev_out)])
    ckpt_out = REF_DIR / "libref_ckpt.so"
    if force or _stale(ckpt_out, [HERE / "ref_ckpt_harness.cu"]):
        _run([NVCC, *ARCH, "-O3", "-std=c++20", *inc, "-Xcompiler", "-fPIC", "-shared",
              "-DNEUROEVOLUTION_PROJECT_SOURCE_DIR=\"/nonexistent\"",
              str(HERE / "ref_ckpt_harness.cu"), "-o", str(ckpt_out)])
    return [host_out, dev_out, ckpt_out]


def build_shim_driver(force: bool = False) -> Path | None:
    """The compat-layer test program: the reference's API headers where they lie, the shim, libnwg.so."""
    if not reference_present():
        return None
    root = HERE.parent
    lib_dir = root / "neuroevolutionary-wordle_b200"
    out = REF_DIR / "shim_driver"
    srcs = [root / "tests" / "shim_driver.cu", root / "include" / "nwg_slab_device_shim.hpp",
            root / "include" / "nwg_capi.h"]
    if force or _stale(out, srcs):
        REF_DIR.mkdir(exist_ok=True)
        _run([NVCC, *ARCH, "-O2", "-std=c++20", "-I", str(REFERENCE_ROOT / "src"), "-I", str(root / "include"),
              str(root / "tests" / "shim_driver.cu"),
              str(REFERENCE_ROOT / "src" / "genetic_algorithm" / "genotype_slab" / "slab_allocator.cpp"),
              "-L", str(lib_dir), "-lnwg", "-Xlinker", "-rpath,$ORIGIN/../../neuroevolutionary-wordle_b200",
              "-o", str(out)])
    return out


def build_all(force: bool = False) -> None:
    build_oracle(force)
    build_tape(force)
    build_reference(force)
    build_shim_driver(force)


if __name__ == "__main__":
    build_all(force=True)
