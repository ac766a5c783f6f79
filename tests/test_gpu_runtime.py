"""The runtime behind the C ABI on the GPU: bootstrap -> evaluate -> advance, as the reference's
slab_runtime_test.cu exercises its runtime (bootstrap, evaluate ranges, one-generation advance,
locality of the cellular plan)."""
import numpy as np
import pytest

from oracle import pyoracle as O
from tests import gpu_util as G
from tests import helpers as H

pytestmark = pytest.mark.gpu


def _setup(action_count=180, population=16, columns=4, per_cell=6, seed=3):
    rng = np.random.default_rng(seed)
    catalog = H.synthetic_words(rng, action_count)
    G.upload_catalog_everywhere(catalog)
    rt = G.nwg.Runtime(action_count, population, columns)
    rt.bootstrap(population, seed=123)
    offsets = np.arange(population + 1, dtype=np.uint32) * per_cell
    words = np.concatenate([rng.choice(action_count, per_cell, replace=False) for _ in range(population)])
    rt.set_cell_words(offsets, words.astype(np.uint32))
    return rt, catalog, G.nwg.capi.word_counts(training=action_count, action_space=action_count)


def test_bootstrap_then_evaluate_gives_fitness_in_range():
    rt, _, counts = _setup()
    rt.evaluate(counts)
    gen = rt.current_generation()
    assert (gen["fitness"] > 0).all() and (gen["fitness"] <= 1.0).all()
    s = rt.summary()
    best, avg, bi = O.summarize(gen["fitness"])
    assert s.best_fitness == best and s.best_index == bi
    assert s.average_fitness == avg
    assert s.population_size == 16
    st = rt.stats()
    assert st.game_steps > 0
    assert abs(st.fitness_mean_fp64 - float(np.mean(gen["fitness"].astype(np.float64)))) < 1e-12


def test_advance_builds_local_plan_and_new_generation():
    rt, _, counts = _setup()
    cfg = G.nwg.capi.assembly_config(radius=1, p=0.05, sigma=0.02)
    rt.advance(seed=42, counts=counts, config=cfg)
    plan = rt.assembly_plan()
    rows, cols = 4, 4
    for child, (a, b) in enumerate(plan.astype(np.int64)):
        assert a != b
        for parent in (a, b):
            dr = min(abs(child // cols - parent // cols), rows - abs(child // cols - parent // cols))
            dc = min(abs(child % cols - parent % cols), cols - abs(child % cols - parent % cols))
            assert max(dr, dc) <= 1
    gen = rt.current_generation()
    assert gen["generation_index"] == 1
    assert not gen["has_fitness"].any()
    assert len(set(gen["slots"].tolist())) == 16
    rt.evaluate(counts)
    assert rt.current_generation()["has_fitness"].all()


def test_advance_is_deterministic():
    results = []
    for _ in range(2):
        rt, _, counts = _setup()
        cfg = G.nwg.capi.assembly_config(radius=1, p=0.05)
        for g in range(2):
            rt.advance(seed=1000 + g, counts=counts, config=cfg)
        rt.evaluate(counts)
        gen = rt.current_generation()
        images = [rt.download_slot(int(s)) for s in gen["slots"]]
        results.append((gen["fitness"].copy(), images))
        rt.close()
    assert np.array_equal(results[0][0], results[1][0])
    for a, b in zip(results[0][1], results[1][1]):
        assert np.array_equal(a, b)


def test_children_follow_parents_and_reference_breeding():
    """Each child image equals the reference's BreedAndMutateGenome of its planned parents."""
    if O.ref_dev() is None:
        pytest.skip("reference device library not built")
    t = G.torch()
    rt, _, counts = _setup(action_count=140, population=9, columns=3, per_cell=5)
    gen0 = rt.current_generation()
    parents = [rt.download_slot(int(s)) for s in gen0["slots"]]
    rt.advance(seed=77, counts=counts, config=G.nwg.capi.assembly_config(radius=1, p=0.05))
    plan = rt.assembly_plan()
    gen1 = rt.current_generation()
    stride = G.nwg.capi.genome_stride_bytes(140)
    pitch = ((stride + 255) // 256) * 256
    slab = np.zeros(9 * pitch, np.uint8)
    for i, img in enumerate(parents):
        slab[i * pitch:i * pitch + stride] = img
    parent_dev = G.dev(slab)
    out = G.slab_tensor(9, pitch)
    pairs = G.dev(plan.astype(np.uint32).reshape(-1))
    assert O.ref_dev().refdev_breed(parent_dev.data_ptr(), pitch, out.data_ptr(), pitch, pairs.data_ptr(), 9, 140,
                                    77, 0, 0.02, 0.01, 0.005, 0.05, 0.02, 0.0, G.stream_handle()) == 1
    t.cuda.synchronize()
    ref = out.cpu().numpy().reshape(9, pitch)[:, :stride]
    for c in range(9):
        assert np.array_equal(rt.download_slot(int(gen1["slots"][c])), ref[c])


def test_invalid_configs_are_rejected():
    rt, _, counts = _setup()
    with pytest.raises(G.nwg.NwgError) as err:
        rt.advance(seed=1, counts=counts, config=G.nwg.capi.assembly_config(radius=0))
    assert err.value.status == 10
    bad = G.nwg.capi.word_counts(training=181, action_space=180)
    with pytest.raises(G.nwg.NwgError) as err:
        rt.evaluate(bad)
    assert err.value.status == 5
    pending = G.nwg.capi.PendingInjection(True, 180, 10)  # words 180..189 are beyond the 180-word catalog
    with pytest.raises(G.nwg.NwgError) as err:
        rt.advance(seed=1, counts=counts, pending=pending)
    assert err.value.status == 15
