"""The evaluation entry point that allocates no device memory, against the runtime's own evaluation.

Some callers cannot call cudaMalloc: embedders whose device memory belongs to another allocator or pool, and
processes that keep a fixed device footprint after start-up. nwg_evaluate_noalloc serves them: the caller passes
every input and output as device buffers it owns, and the library keeps its working memory in one fixed array.
Its fitness must equal the runtime's (nwg_evaluate) bit for bit, on two calls in a row, because the array keeps
the previous call's contents. This file is collected last so that a run stopping at the first failure has
already run every other test; it also passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from tests import gpu_util as G
from tests import helpers as H

pytestmark = pytest.mark.gpu
MAX_POPULATION, MAX_CATALOG = 4096, 4739


def _bind():
    lib = G.nwg.capi.lib()
    fn = lib.nwg_evaluate_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t, C.c_size_t, C.c_size_t, C.c_void_p, C.c_size_t,
                   C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    return fn


def _compare_two_calls(action_count, catalog_count, population, columns, per_cell, seed, with_counters):
    """Runtime evaluation first, then two no-alloc calls in a row on the same genomes and word lists."""
    t = G.torch()
    rng = np.random.default_rng(seed)
    catalog = H.synthetic_words(rng, catalog_count)
    G.nwg.capi.upload_catalog(catalog)
    rt = G.nwg.Runtime(action_count, population, columns)
    rt.bootstrap(population, seed=seed)
    offsets = np.arange(population + 1, dtype=np.uint32) * per_cell
    words = np.concatenate([rng.choice(catalog_count, per_cell, replace=False) for _ in range(population)])
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
        counters = t.full((3,), -1, dtype=t.int64, device="cuda")
        status = fn(slab, pitch, slots.data_ptr(), population, columns, action_count, letters.data_ptr(),
                    len(catalog), d_offsets.data_ptr(), d_words.data_ptr(), fitness.data_ptr(),
                    counters.data_ptr() if with_counters else None, G.stream_handle())
        assert status == 0, f"call {call}: status {status}"
        got = fitness.cpu().numpy()
        assert np.array_equal(got.view(np.uint32), expected["fitness"].view(np.uint32)), f"call {call}: fitness"
        c = counters.cpu().numpy()
        if with_counters:
            assert c[0] == expected_stats.game_steps and c[1] == expected_stats.encoded_turns
            assert c[2] == expected_stats.episodes
        else:
            assert (c == -1).all()  # untouched
    rt.close()


@pytest.mark.parametrize("with_counters", [True, False], ids=["counters", "no-counters"])
@pytest.mark.parametrize("action_count,catalog_count", [(100, 300), (300, 300), (300, 500)])
def test_noalloc_evaluation_matches_runtime_on_two_calls_in_a_row(action_count, catalog_count, with_counters):
    """(100, 300) takes the tensor-tile scorer of at most 128 selectable actions; (300, 500) a catalog larger than
    the action space, with secrets beyond the selectable words."""
    _compare_two_calls(action_count, catalog_count, 16, 4, 7, 21 + action_count + catalog_count, with_counters)


def test_noalloc_at_its_documented_maximum():
    """4,096 individuals and a 4,739-word catalog, the largest sizes the fixed array holds."""
    _compare_two_calls(MAX_CATALOG, MAX_CATALOG, MAX_POPULATION, 64, 8, 4739, True)


def test_noalloc_rejects_sizes_beyond_its_array():
    fn = _bind()
    t = G.torch()
    dummy = t.zeros(1024, dtype=t.uint8, device="cuda")
    p = dummy.data_ptr()
    stride = G.nwg.capi.genome_stride_bytes(10)
    pitch = (stride + 255) // 256 * 256
    assert fn(p, pitch, p, MAX_POPULATION + 1, 1, 10, p, 10, p, p, p, None, G.stream_handle()) == 18
    assert fn(p, pitch, p, 16, 4, 10, p, MAX_CATALOG + 1, p, p, p, None, G.stream_handle()) == 18
    assert fn(p, pitch, p, 0, 4, 10, p, 10, p, p, p, None, G.stream_handle()) == 2  # no population


def test_noalloc_refuses_decreasing_offsets_on_the_device():
    """A decreasing pair of offsets would read as a huge word count; the cell is refused on the device before any
    of its words is read (every offset here stays inside the 24-word buffer), and the next call succeeds."""
    t = G.torch()
    action_count, population, columns = 150, 4, 2
    rng = np.random.default_rng(99)
    catalog = H.synthetic_words(rng, action_count)
    G.nwg.capi.upload_catalog(catalog)
    rt = G.nwg.Runtime(action_count, population, columns)
    rt.bootstrap(population, seed=5)
    slab, pitch = rt.device_slab()
    slots = G.dev(rt.current_generation()["slots"].astype(np.uint32))
    letters = G.dev(np.ascontiguousarray(catalog, np.uint8))
    words = G.dev(rng.choice(action_count, 24, replace=False).astype(np.uint32))
    fitness = t.zeros(population, dtype=t.float32, device="cuda")
    fn = _bind()
    bad = G.dev(np.array([0, 6, 3, 12, 24], np.uint32))
    assert fn(slab, pitch, slots.data_ptr(), population, columns, action_count, letters.data_ptr(), action_count,
              bad.data_ptr(), words.data_ptr(), fitness.data_ptr(), None, G.stream_handle()) == 5
    good = G.dev(np.array([0, 6, 12, 18, 24], np.uint32))
    assert fn(slab, pitch, slots.data_ptr(), population, columns, action_count, letters.data_ptr(), action_count,
              good.data_ptr(), words.data_ptr(), fitness.data_ptr(), None, G.stream_handle()) == 0
    assert (fitness.cpu().numpy() > 0).all()
    rt.close()
