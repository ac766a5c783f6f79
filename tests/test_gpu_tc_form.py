"""The tensor-core scoring forms (BF16 / FP16 operands with exact FP32 re-scoring) against the plain form.

Both forms keep the FP32 trunk and re-score in FP32 every action chunk that an error bound cannot rule out,
so every guess, turn count, episode score, policy vector and fitness must equal the plain form's exactly.
"""
import numpy as np
import pytest

from tests import gpu_util as G
from tests import helpers as H

pytestmark = pytest.mark.gpu


def _trace(rt, counts, episodes):
    t = G.torch()
    p = rt.population
    choices = t.full((p, episodes, 6), -1, dtype=t.int32, device="cuda")
    turns = t.zeros((p, episodes), dtype=t.int32, device="cuda")
    scores = t.zeros((p, episodes), dtype=t.float32, device="cuda")
    policy = t.zeros((p, episodes, 6, 64), dtype=t.float32, device="cuda")
    rt.evaluate_traced(counts, episodes, choices.data_ptr(), turns.data_ptr(), scores.data_ptr(), policy.data_ptr())
    t.cuda.synchronize()
    gen = rt.current_generation()
    return (choices.cpu().numpy(), turns.cpu().numpy(), scores.cpu().numpy(), policy.cpu().numpy(),
            gen["fitness"].copy(), rt.stats())


@pytest.mark.parametrize("form", [1, 2])
@pytest.mark.parametrize("action_count,population,columns,sizes,generations", [
    (1000, 4, 2, [5, 9, 130, 7], 0),
    (100, 4, 2, [6, 6, 6, 6], 0),
    (4739, 4, 2, [12, 8, 10, 11], 0),
    (700, 16, 4, [7] * 16, 2),
])
def test_tensor_core_form_equals_plain_form(form, action_count, population, columns, sizes, generations):
    rng = np.random.default_rng(action_count + population + form)
    catalog = H.synthetic_words(rng, action_count)
    G.nwg.capi.upload_catalog(catalog)
    rt = G.nwg.Runtime(action_count, population, columns)
    rt.bootstrap(population, seed=31 + action_count)
    lists = [rng.choice(action_count, size=s, replace=False).astype(np.uint32) for s in sizes]
    offsets = np.zeros(population + 1, np.uint32)
    offsets[1:] = np.cumsum(sizes)
    rt.set_cell_words(offsets, np.concatenate(lists))
    counts = G.nwg.capi.word_counts(training=action_count, action_space=action_count)
    cfg = G.nwg.capi.assembly_config(radius=1, p=0.05, sigma=0.02)
    for g in range(generations):
        rt.advance(seed=500 + g, counts=counts, config=cfg)
    episodes = 3 * max(sizes)
    plain = _trace(rt, counts, episodes)
    rt.set_form(form)
    tc = _trace(rt, counts, episodes)
    for i in range(population):
        w3 = 3 * sizes[i]
        assert np.array_equal(tc[0][i, :w3], plain[0][i, :w3]), f"guesses differ for individual {i}"
        assert np.array_equal(tc[1][i, :w3], plain[1][i, :w3])
        assert np.array_equal(tc[2][i, :w3], plain[2][i, :w3])
        assert np.array_equal(tc[3][i, :w3], plain[3][i, :w3])
    assert np.array_equal(tc[4], plain[4])
    assert tc[5].game_steps == plain[5].game_steps
    if action_count > 128:
        assert tc[5].rescored_chunks > 0
    else:  # at <= 128 actions every form scores on the reference's tensor-tile path, in the plain kernel
        assert tc[5].rescored_chunks == 0
    rt.close()


def test_tensor_core_form_runs_a_generation():
    action_count, population, columns = 600, 9, 3
    rng = np.random.default_rng(77)
    catalog = H.synthetic_words(rng, action_count)
    G.nwg.capi.upload_catalog(catalog)
    results = []
    for form in (0, 1):
        rt = G.nwg.Runtime(action_count, population, columns)
        rt.set_form(form)
        rt.bootstrap(population, seed=9)
        offsets = np.arange(population + 1, dtype=np.uint32) * 5
        words = np.concatenate([np.arange(5 * i, 5 * i + 5) for i in range(population)]).astype(np.uint32)
        rt.set_cell_words(offsets, words)
        counts = G.nwg.capi.word_counts(training=action_count, action_space=action_count)
        for g in range(2):
            rt.advance(seed=100 + g, counts=counts, config=G.nwg.capi.assembly_config(radius=1, p=0.05))
        rt.evaluate(counts)
        gen = rt.current_generation()
        results.append((gen["fitness"].copy(), [rt.download_slot(int(s)) for s in gen["slots"]]))
        rt.close()
    assert np.array_equal(results[0][0], results[1][0])
    for a, b in zip(results[0][1], results[1][1]):
        assert np.array_equal(a, b)
