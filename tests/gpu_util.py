"""Helpers shared by the GPU parity tests (device buffers come from torch; kernels from libnwg.so)."""
from __future__ import annotations

import importlib

import numpy as np

from oracle import pyoracle as O

nwg = importlib.import_module("neuroevolutionary-wordle_b200")


def torch():
    import torch as t

    return t


def dev(array: np.ndarray):
    t = torch()
    return t.from_numpy(np.ascontiguousarray(array)).cuda()


def ptr(tensor) -> int:
    return tensor.data_ptr()


def stream_handle() -> int:
    return torch().cuda.current_stream().cuda_stream


def upload_catalog_everywhere(letters: np.ndarray) -> None:
    nwg.capi.upload_catalog(letters)
    ref = O.ref_dev()
    if ref is not None:
        arr = np.ascontiguousarray(letters, np.uint8)
        assert ref.refdev_upload_catalog(arr.ctypes.data_as(O._u8p), len(arr)) == 1


def slab_tensor(count: int, pitch: int):
    t = torch()
    return t.zeros(count * pitch, dtype=t.uint8, device="cuda")


def genome_halfs_at(slab_cpu: np.ndarray, index: int, pitch: int, action_count: int) -> np.ndarray:
    stride = nwg.capi.genome_stride_bytes(action_count)
    return slab_cpu[index * pitch:index * pitch + stride].view(np.uint16).copy()
