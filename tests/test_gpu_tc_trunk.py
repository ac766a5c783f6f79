"""The tensor-core trunk forms (encoder, trunk and scores on tcgen05, margin guard) against the plain form.

With a guard bound so large that every game step takes the exact FP32 path, every guess, turn count,
episode score, policy vector and fitness must equal the plain form's bit for bit. At the default guard
(tau = 1e-3) the FP16-operand form's guesses must agree on at least 99.9% of the comparable game steps
(steps whose game state is still identical in both runs); the BF16-operand form, which also rounds the
genome's FP16 weights and embeddings, needs tau = 1e-2 for that.
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


def _runtime(action_count, population, columns, sizes, generations, seed):
    rng = np.random.default_rng(seed)
    catalog = H.synthetic_words(rng, action_count)
    G.nwg.capi.upload_catalog(catalog)
    rt = G.nwg.Runtime(action_count, population, columns)
    rt.bootstrap(population, seed=31 + seed)
    lists = [rng.choice(action_count, size=s, replace=False).astype(np.uint32) for s in sizes]
    offsets = np.zeros(population + 1, np.uint32)
    offsets[1:] = np.cumsum(sizes)
    rt.set_cell_words(offsets, np.concatenate(lists))
    counts = G.nwg.capi.word_counts(training=action_count, action_space=action_count)
    cfg = G.nwg.capi.assembly_config(radius=1, p=0.05, sigma=0.02)
    for g in range(generations):
        rt.advance(seed=500 + g, counts=counts, config=cfg)
    return rt, counts


def agreement(a_choices, b_choices, sizes):
    """(identical decisions, comparable decisions): a step is comparable while every earlier choice agreed."""
    same = total = 0
    for i, s in enumerate(sizes):
        for e in range(3 * s):
            for step in range(6):
                x, y = a_choices[i, e, step], b_choices[i, e, step]
                if x < 0 and y < 0:
                    break
                total += 1
                if x != y:
                    break
                same += 1
    return same, total


@pytest.mark.parametrize("form", [3, 4])
@pytest.mark.parametrize("action_count,population,columns,sizes,generations", [
    (1000, 4, 2, [5, 9, 130, 7], 0),
    (100, 4, 2, [6, 6, 6, 6], 0),
    (4739, 4, 2, [12, 8, 10, 11], 0),
    (700, 16, 4, [7] * 16, 2),
])
def test_exact_path_equals_plain_form(form, action_count, population, columns, sizes, generations):
    rt, counts = _runtime(action_count, population, columns, sizes, generations, action_count + population + form)
    episodes = 3 * max(sizes)
    plain = _trace(rt, counts, episodes)
    rt.set_form(form)
    rt.set_margin_guard(1.0e30)
    tc = _trace(rt, counts, episodes)
    for i in range(population):
        w3 = 3 * sizes[i]
        assert np.array_equal(tc[0][i, :w3], plain[0][i, :w3]), f"guesses differ for individual {i}"
        assert np.array_equal(tc[1][i, :w3], plain[1][i, :w3])
        assert np.array_equal(tc[2][i, :w3], plain[2][i, :w3])
        assert np.array_equal(tc[3][i, :w3].view(np.uint32), plain[3][i, :w3].view(np.uint32))
    assert np.array_equal(tc[4], plain[4])
    assert tc[5].game_steps == plain[5].game_steps
    # at <= 128 actions every form scores on the reference's tensor-tile path, in the plain kernel
    assert tc[5].fallback_steps == (tc[5].game_steps if action_count > 128 else 0)
    rt.close()


@pytest.mark.parametrize("form,tau,floor", [(4, 1e-3, 0.999), (3, 1e-2, 0.999), (4, 0.0, 0.995), (3, 1e-3, 0.985)])
def test_guarded_guesses_agree_with_plain_form(form, tau, floor):
    sizes = [48] * 16
    rt, counts = _runtime(4739, 16, 4, sizes, 1, 7 + form)
    episodes = 3 * max(sizes)
    plain = _trace(rt, counts, episodes)
    rt.set_form(form)
    rt.set_margin_guard(tau)
    tc = _trace(rt, counts, episodes)
    same, total = agreement(tc[0], plain[0], sizes)
    assert total > 10000
    assert same / total >= floor, (same, total)
    st = tc[5]
    assert st.candidate_chunks > 0
    if tau > 0:
        assert 0 < st.fallback_steps < 0.2 * st.game_steps
    # the approximate policy stays close to the FP32 one on identical states (first step of every game)
    p_tc = tc[3][:, :, 0, :].reshape(-1, 64)
    p_fp = plain[3][:, :, 0, :].reshape(-1, 64)
    live = np.abs(p_fp).sum(1) > 0
    rel = np.abs(p_tc[live] - p_fp[live]).max() / np.abs(p_fp[live]).max()
    assert rel < (5e-2 if form == 3 else 1e-2), rel
    rt.close()


def test_trunk_form_runs_generations():
    action_count, population, columns = 600, 9, 3
    rng = np.random.default_rng(78)
    catalog = H.synthetic_words(rng, action_count)
    G.nwg.capi.upload_catalog(catalog)
    rt = G.nwg.Runtime(action_count, population, columns)
    rt.set_form(4)
    rt.bootstrap(population, seed=9)
    offsets = np.arange(population + 1, dtype=np.uint32) * 5
    words = np.concatenate([np.arange(5 * i, 5 * i + 5) for i in range(population)]).astype(np.uint32)
    rt.set_cell_words(offsets, words)
    counts = G.nwg.capi.word_counts(training=action_count, action_space=action_count)
    for g in range(3):
        rt.advance(seed=100 + g, counts=counts, config=G.nwg.capi.assembly_config(radius=1, p=0.05))
    rt.evaluate(counts)
    st = rt.stats()
    assert st.game_steps > 0 and st.episodes == 15 * population
    assert rt.status() == 0
    rt.close()


def test_margin_guard_rejects_bad_bounds():
    G.nwg.capi.upload_catalog(H.synthetic_words(np.random.default_rng(1), 64))
    rt = G.nwg.Runtime(64, 4, 2)
    for bad in (-1.0, float("nan"), float("inf")):
        with pytest.raises(Exception):
            rt.set_margin_guard(bad)
    rt.set_margin_guard(0.0)
    rt.close()
