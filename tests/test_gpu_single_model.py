"""Single-model inference on the B200 against the reference's single-model runtime.

Reference: TryCreateSingleModelDeviceRuntime / TrySelectNextGuessWithSingleModelDeviceRuntime
(inference/single_model_device_runtime.cu:89-183) and its test (tests/inference/single_model_device_runtime_test.cu:
the policy fixture over CABBY/CACAO/FUZZY picks CACAO with score 24.5; a zero genome with CRANE guessed picks SLATE
with score 0). Random genomes and grids are compared with the reference runtime itself (oracle/_ref/libref_ckpt.so),
one reference call per grid against one batched call here: index and score bit for bit.
"""
import numpy as np
import pytest

from oracle import pyoracle as O
from tests import gpu_util as G
from tests import helpers as H

pytestmark = pytest.mark.gpu
capi = G.nwg.capi


def _grids(rng, catalog, n):
    guesses = np.zeros((n, 6, 5), np.uint8)
    feedback = np.zeros((n, 6, 5), np.uint8)
    turns = np.zeros(n, np.uint8)
    for g in range(n):
        secret = catalog[rng.integers(len(catalog))]
        t = int(rng.integers(0, 6))
        k = 0
        for _ in range(t):
            word = catalog[rng.integers(len(catalog))]
            fb = O.feedback(word, secret)
            if np.all(fb == 0):
                continue  # a won turn ends the game
            guesses[g, k], feedback[g, k] = word, fb
            k += 1
        turns[g] = k
    return guesses, feedback, turns


def _reference(genome, catalog, guesses, feedback, turns):
    n = len(turns)
    status = np.zeros(n, np.int32)
    index = np.zeros(n, np.uint64)
    score = np.zeros(n, np.float32)
    g = np.ascontiguousarray(genome).view(np.uint8)
    assert O.ref_ckpt().refsm_select_many(g.ctypes.data, g.nbytes, catalog.ctypes.data, len(catalog),
                                          guesses.ctypes.data, feedback.ctypes.data, turns.ctypes.data, n,
                                          status.ctypes.data, index.ctypes.data, score.ctypes.data) == 1
    return status, index, score


def test_reference_test_cases():
    catalog = O.words_to_letters(["CABBY", "CACAO", "FUZZY"])
    g = H.empty_genome(3)
    H.policy_fixture(g)
    m = capi.SingleModel(g, catalog)
    guesses = np.zeros((1, 6, 5), np.uint8)
    feedback = np.zeros((1, 6, 5), np.uint8)
    guesses[0, 0] = O.word("ABCDE")
    feedback[0, 0] = O.feedback(O.word("ABCDE"), O.word("AEBDF"))
    index, score = m.select(guesses, feedback, np.array([1], np.uint8))
    assert index[0] == 1 and abs(score[0] - 24.5) <= 1e-6
    m.close()
    catalog = O.words_to_letters(["CRANE", "SLATE", "TRACE"])
    m = capi.SingleModel(H.empty_genome(3), catalog)
    guesses[0, 0] = catalog[0]
    feedback[0, 0] = O.feedback(catalog[0], catalog[2])
    index, score = m.select(guesses, feedback, np.array([1], np.uint8))
    assert index[0] == 1 and score[0] == 0.0
    m.close()


@pytest.mark.skipif(O.ref_ckpt() is None, reason="reference library not built")
@pytest.mark.parametrize("action_count,grids", [(3, 40), (100, 300), (1000, 300), (4739, 130)])
def test_selection_matches_reference_runtime(action_count, grids):
    rng = np.random.default_rng(action_count)
    catalog = H.synthetic_words(rng, action_count)
    genome = H.random_genome(rng, action_count)
    guesses, feedback, turns = _grids(rng, catalog, grids)
    if action_count == 3:
        turns = np.minimum(turns, 2).astype(np.uint8)  # keep an unguessed action
    m = capi.SingleModel(genome, catalog)
    index, score = m.select(guesses, feedback, turns)
    status, ref_index, ref_score = _reference(genome, catalog, guesses, feedback, turns)
    assert np.all(status == 0)
    assert np.array_equal(index, ref_index.astype(np.int64))
    assert np.array_equal(score.view(np.uint32), ref_score.view(np.uint32))
    m.close()


def test_invalid_grids_are_reported():
    rng = np.random.default_rng(3)
    catalog = H.synthetic_words(rng, 3)
    m = capi.SingleModel(H.random_genome(rng, 3), catalog)
    guesses = np.zeros((1, 6, 5), np.uint8)
    feedback = np.full((1, 6, 5), 2, np.uint8)
    guesses[0, :3] = catalog
    with pytest.raises(capi.NwgError) as e:
        m.select(guesses, feedback, np.array([3], np.uint8))  # every action already guessed
    assert e.value.status == 8
    with pytest.raises(capi.NwgError) as e:
        m.select(guesses, feedback, np.array([6], np.uint8))  # more than five turns
    assert e.value.status == 7
    won = feedback.copy()
    won[0, 0] = 0
    with pytest.raises(capi.NwgError) as e:
        m.select(guesses, won, np.array([1], np.uint8))
    assert e.value.status == 7
    with pytest.raises(capi.NwgError) as e:
        capi.SingleModel(H.random_genome(rng, 4), catalog)  # genome width differs from the catalog
    assert e.value.status == 2
    m.close()
