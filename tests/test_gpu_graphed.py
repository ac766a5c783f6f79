"""Graphed generations (nwg_advance_graphed) against nwg_advance.

A graphed generation captures the same launches as nwg_advance into one CUDA graph, and its first generations
at each action width try different launch shapes (one or two persistent evaluation CTAs per SM, 4, 8 or 16
children per breeding CTA). The children and fitness must equal nwg_advance's bit for bit whatever the shapes,
with and without a widening generation (which runs ungraphed), on the default stream and on a caller's stream.
"""
import numpy as np
import pytest

from tests import gpu_util as G
from tests import helpers as H

pytestmark = pytest.mark.gpu


def _pair(action_count, population, columns, form, sizes, seed, stream=None):
    rng = np.random.default_rng(seed)
    catalog = H.synthetic_words(rng, action_count + 64)
    G.nwg.capi.upload_catalog(catalog)
    lists = [rng.choice(action_count, size=s, replace=False).astype(np.uint32) for s in sizes]
    offsets = np.zeros(population + 1, np.uint32)
    offsets[1:] = np.cumsum(sizes)
    words = np.concatenate(lists)
    rts = []
    for _ in range(2):
        rt = G.nwg.Runtime(action_count, population, columns, stream=stream)
        rt.bootstrap(population, seed=seed)
        rt.set_cell_words(offsets, words)
        rt.set_form(form)
        rts.append(rt)
    return rts, offsets, words


def _same_generation(a, b):
    ga, gb = a.current_generation(), b.current_generation()
    assert np.array_equal(ga["slots"], gb["slots"])
    assert np.array_equal(ga["fitness"], gb["fitness"])
    assert np.array_equal(ga["has_fitness"], gb["has_fitness"])
    for s in ga["slots"]:
        assert np.array_equal(a.download_slot(int(s)), b.download_slot(int(s)))


@pytest.mark.parametrize("form", [0, 4])
@pytest.mark.parametrize("use_stream", [False, True])
def test_graphed_generations_equal_direct(form, use_stream):
    side = G.torch().cuda.Stream() if use_stream else None  # a caller's stream (torch's default one is stream 0)
    stream = side.cuda_stream if use_stream else None
    population, columns, action_count = 16, 4, 700
    sizes = [5, 9, 6, 12, 7, 7, 5, 11, 6, 14, 8, 10, 5, 5, 9, 6]  # at least 5: the prefills never hit the secret
    (direct, graphed), _, _ = _pair(action_count, population, columns, form, sizes, 11 + form, stream)
    counts = G.nwg.capi.word_counts(training=action_count, action_space=action_count)
    cfg = G.nwg.capi.assembly_config(radius=1, p=0.05, sigma=0.02)
    for g in range(5):
        direct.advance(seed=300 + g, counts=counts, config=cfg)
        graphed.advance_graphed(seed=300 + g, counts=counts, config=cfg)
        _same_generation(direct, graphed)
        assert graphed.status() == 0
    info = graphed.graph_info()
    assert info.launches == 5 and info.instantiations >= 1 and info.instantiations + info.updates == 5
    tune = graphed.launch_tuning()
    assert tune.decided == 1 and tune.trials == 3
    assert tune.breed_warps in (4, 8, 16) and tune.eval_ctas > 0
    assert all(t > 0 for t in tune.breed_ms) and all(t > 0 for t in tune.eval_ms)
    direct.close()
    graphed.close()


def test_graphed_run_through_a_widening_generation():
    population, columns, action_count, injected = 16, 4, 300, 40
    sizes = [6] * population
    (direct, graphed), offsets, words = _pair(action_count, population, columns, 4, sizes, 5)
    counts = G.nwg.capi.word_counts(training=action_count, action_space=action_count)
    cfg = G.nwg.capi.assembly_config(radius=1, p=0.05, sigma=0.02)
    for g in range(6):
        pending = G.nwg.capi.PendingInjection(True, action_count, injected) if g == 2 else None
        direct.advance(seed=700 + g, counts=counts, config=cfg, pending=pending)
        graphed.advance_graphed(seed=700 + g, counts=counts, config=cfg, pending=pending)
        _same_generation(direct, graphed)
        if g == 2:
            # the byte budget fixed at creation holds fewer of the wider genomes: whole grid rows are dropped
            n = len(graphed.current_generation()["slots"])
            assert n == 12
            for rt in (direct, graphed):
                rt.set_cell_words(offsets[:n + 1], words[:offsets[n]])
            counts = G.nwg.capi.word_counts(training=action_count, action_space=action_count + injected)
    assert graphed.action_count == action_count + injected
    assert graphed.graph_info().launches == 5  # the widening generation ran ungraphed
    assert graphed.launch_tuning(width=action_count).trials == 2
    assert graphed.launch_tuning(width=action_count + injected).decided == 1
    direct.close()
    graphed.close()


def test_graphed_generation_rejects_a_bad_config_like_advance():
    population, columns, action_count = 16, 4, 300
    (direct, graphed), _, _ = _pair(action_count, population, columns, 4, [6] * population, 9)
    counts = G.nwg.capi.word_counts(training=action_count, action_space=action_count)
    bad = G.nwg.capi.assembly_config(radius=0)
    with pytest.raises(G.nwg.capi.NwgError) as e1:
        direct.advance(seed=1, counts=counts, config=bad)
    with pytest.raises(G.nwg.capi.NwgError) as e2:
        graphed.advance_graphed(seed=1, counts=counts, config=bad)
    assert str(e1.value).split(":")[-1] == str(e2.value).split(":")[-1]
    assert direct.status() == graphed.status() != 0
    # the runtime stays usable
    good = G.nwg.capi.assembly_config(radius=1)
    direct.advance(seed=2, counts=counts, config=good)
    graphed.advance_graphed(seed=2, counts=counts, config=good)
    _same_generation(direct, graphed)
    direct.close()
    graphed.close()
