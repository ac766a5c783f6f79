"""The evaluation entry point that allocates no device memory, against the runtime's own evaluation.

Callers that cannot call cudaMalloc (graph capture, foreign allocators, fixed footprints) get
nwg_evaluate_noalloc, which keeps its working memory in a fixed array inside the library. This file is
collected last so that a run stopping at the first failure has already run every other test; it also
passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from tests import gpu_util as G
from tests import helpers as H

pytestmark = pytest.mark.gpu


def _bind():
    lib = G.nwg.capi.lib()
    fn = lib.nwg_evaluate_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t, C.c_size_t, C.c_size_t, C.c_void_p, C.c_size_t,
                   C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    return fn


def test_noalloc_evaluation_matches_runtime_on_two_calls_in_a_row():
    t = G.torch()
    action_count, population, columns, per_cell = 300, 16, 4, 7
    rng = np.random.default_rng(21)
    catalog = H.synthetic_words(rng, action_count)
    G.nwg.capi.upload_catalog(catalog)
    rt = G.nwg.Runtime(action_count, population, columns)
    rt.bootstrap(population, seed=606)
    offsets = np.arange(population + 1, dtype=np.uint32) * per_cell
    words = np.concatenate([rng.choice(action_count, per_cell, replace=False) for _ in range(population)])
    words = words.astype(np.uint32)
    rt.set_cell_words(offsets, words)
    counts = G.nwg.capi.word_counts(training=action_count, action_space=action_count)
    rt.evaluate(counts)
    expected = rt.current_generation()
    expected_stats = rt.stats()

    fn = _bind()
    slab, pitch = rt.device_slab()
    slots = G.dev(expected["slots"].astype(np.uint32))
    letters = G.dev(np.ascontiguousarray(catalog, np.uint8))
    d_offsets = G.dev(offsets)
    d_words = G.dev(words)
    for call in range(2):
        fitness = t.full((population,), -1.0, dtype=t.float32, device="cuda")
        counters = t.zeros(3, dtype=t.int64, device="cuda")
        status = fn(slab, pitch, slots.data_ptr(), population, columns, action_count, letters.data_ptr(),
                    len(catalog), d_offsets.data_ptr(), d_words.data_ptr(), fitness.data_ptr(),
                    counters.data_ptr(), G.stream_handle())
        assert status == 0, f"call {call}: status {status}"
        got = fitness.cpu().numpy()
        assert np.array_equal(got, expected["fitness"]), f"call {call}: fitness differs"
        c = counters.cpu().numpy()
        assert c[0] == expected_stats.game_steps and c[1] == expected_stats.encoded_turns
        assert c[2] == expected_stats.episodes


def test_noalloc_rejects_sizes_beyond_its_array():
    fn = _bind()
    t = G.torch()
    dummy = t.zeros(1024, dtype=t.uint8, device="cuda")
    p = dummy.data_ptr()
    status = fn(p, 301056 + 76 * 10 + 256 - ((301056 + 76 * 10) % 256), p, 4097, 1, 10, p, 10, p, p, p, 0,
                G.stream_handle())
    assert status == 18  # NWG_UNSUPPORTED: population above 4,096
