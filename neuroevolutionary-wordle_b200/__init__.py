"""B200-native fitness evaluation and generation step for neuroevolutionary Wordle.

The runtime is libnwg.so (CUDA, sm_100a) behind the C ABI in include/nwg_capi.h; `capi` binds it
for Python callers (tests, benchmarks) and `workload` builds seeded synthetic inputs.
"""
from . import capi, workload  # noqa: F401
from .capi import NwgError, Runtime  # noqa: F401

__all__ = ["capi", "workload", "Runtime", "NwgError"]
