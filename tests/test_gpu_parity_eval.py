"""Fitness evaluation on the B200 against the reference's own device code and the CPU oracle.

The reference side is oracle/_ref/libref_dev.so: the reference's SelectNextGuessFromDynamicGenomeConcurrently,
TryInitializeEpisodeGrid and TryAppendGuess (its FP32 warp scorer, used for more than 128 actions),
compiled for sm_100a and run on the same genomes. Bar: identical guesses, turn counts and episode
scores, and policy vectors equal to the last bit (the zero-sign of an exactly-zero output is the only
freedom the reordered arithmetic has, and == treats +0 and -0 as equal), which is tighter than the
1e-5 relative tolerance the path is specified with.
"""
import numpy as np
import pytest

from oracle import pyoracle as O
from tests import gpu_util as G
from tests import helpers as H

pytestmark = pytest.mark.gpu
REL_TOL = 1e-5


def _run_reference(slab_ptr, pitch, population, columns, action_count, shards, episodes):
    t = G.torch()
    choices = t.full((population, episodes, 6), -1, dtype=t.int32, device="cuda")
    turns = t.zeros((population, episodes), dtype=t.int32, device="cuda")
    scores = t.zeros((population, episodes), dtype=t.float32, device="cuda")
    policy = t.zeros((population, episodes, 6, 64), dtype=t.float32, device="cuda")
    status = t.zeros(1, dtype=t.int32, device="cuda")
    arr = (O.ShardRecord * len(shards))(*shards)
    ok = O.ref_dev().refdev_evaluate(slab_ptr, pitch, population, columns, action_count, O.C.cast(arr, O.C.c_void_p),
                                     len(shards), episodes, scores.data_ptr(), turns.data_ptr(), choices.data_ptr(),
                                     policy.data_ptr(), status.data_ptr(), G.stream_handle())
    assert ok == 1
    t.cuda.synchronize()
    assert int(status.item()) == 0
    return choices.cpu().numpy(), turns.cpu().numpy(), scores.cpu().numpy(), policy.cpu().numpy()


def _run_ours(rt, counts, episodes):
    t = G.torch()
    p = rt.population
    choices = t.full((p, episodes, 6), -1, dtype=t.int32, device="cuda")
    turns = t.zeros((p, episodes), dtype=t.int32, device="cuda")
    scores = t.zeros((p, episodes), dtype=t.float32, device="cuda")
    policy = t.zeros((p, episodes, 6, 64), dtype=t.float32, device="cuda")
    rt.evaluate_traced(counts, episodes, choices.data_ptr(), turns.data_ptr(), scores.data_ptr(), policy.data_ptr())
    t.cuda.synchronize()
    return choices.cpu().numpy(), turns.cpu().numpy(), scores.cpu().numpy(), policy.cpu().numpy()


def _compare(ours, ref, episodes_per_individual):
    oc, ot, os_, op = ours
    rc, rt_, rs, rp = ref
    for i, w3 in enumerate(episodes_per_individual):
        assert np.array_equal(oc[i, :w3], rc[i, :w3]), f"guesses differ for individual {i}"
        assert np.array_equal(ot[i, :w3], rt_[i, :w3])
        assert np.array_equal(os_[i, :w3], rs[i, :w3])
        for e in range(w3):
            decisions = int((rc[i, e] >= 0).sum())
            a = op[i, e, :decisions]
            b = rp[i, e, :decisions]
            assert np.all(a == b), f"policy differs at individual {i} episode {e}"
            assert np.all(np.abs(a - b) <= REL_TOL * np.maximum(1.0, np.abs(b)))


@pytest.mark.skipif(O.ref_dev() is None, reason="reference device library not built")
@pytest.mark.parametrize("action_count,words,columns,population", [(160, 6, 2, 4), (300, 150, 2, 4),
                                                                   (1024, 9, 3, 9)])
def test_evaluation_matches_reference_device_code(action_count, words, columns, population):
    rng = np.random.default_rng(action_count + words)
    catalog = H.synthetic_words(rng, action_count)
    G.upload_catalog_everywhere(catalog)
    rt = G.nwg.Runtime(action_count, population, columns)
    rt.bootstrap(population, seed=1234 + words)
    counts = G.nwg.capi.word_counts(training=words, action_space=action_count)
    episodes = 3 * words
    ours = _run_ours(rt, counts, episodes)
    slab, pitch = rt.device_slab()
    ref = _run_reference(slab, pitch, population, columns, action_count, [O.ShardRecord(0, words, 0, 0, 0, 1)],
                         episodes)
    _compare(ours, ref, [episodes] * population)
    # fitness = episode-score sum normalised by 45 W (evaluation_ops.cuh:87-111)
    gen = rt.current_generation()
    for i in range(population):
        raw = np.float32(ref[2][i, :episodes].sum())
        assert gen["fitness"][i] == O.normalize_fitness(float(raw), words)
    assert gen["has_fitness"].all() and (gen["evaluation_counts"] == 1).all()


@pytest.mark.skipif(O.ref_dev() is None, reason="reference device library not built")
def test_spatial_shard_exposure_matches_reference():
    """Foundation shard plus radius-limited shards: cells see different word counts (slab_runtime_test.cu:533-575)."""
    action_count, columns, population = 200, 4, 16
    rng = np.random.default_rng(5)
    catalog = H.synthetic_words(rng, action_count)
    G.upload_catalog_everywhere(catalog)
    rt = G.nwg.Runtime(action_count, population, columns)
    rt.bootstrap(population, seed=77, generation_index=0)
    counts = G.nwg.capi.word_counts(training=12, action_space=action_count, initial=6, step=3, period=1,
                                    initial_radius=0, growth_period=2)
    shards = [O.ShardRecord(0, 6, 0, 0, 0, 1)]
    for local in range(2):
        cell = ((local + 1) * 11400714819323198485) % (1 << 64) % population
        shards.append(O.ShardRecord(6 + 3 * local, 3, cell // columns, cell % columns, 0, 0))
    per_cell = [len(O.cell_words_from_shards(shards, 4, 4, c)) for c in range(population)]
    assert sorted(set(per_cell)) == [6, 9]
    episodes = 3 * max(per_cell)
    ours = _run_ours(rt, counts, episodes)
    slab, pitch = rt.device_slab()
    ref = _run_reference(slab, pitch, population, columns, action_count, shards, episodes)
    _compare(ours, ref, [3 * w for w in per_cell])


def test_csr_lists_match_cpu_oracle():
    """Ragged explicit per-cell secret lists (no reference counterpart): checked against the CPU oracle."""
    action_count, columns, population = 200, 2, 4
    rng = np.random.default_rng(9)
    catalog = H.synthetic_words(rng, action_count)
    G.upload_catalog_everywhere(catalog)
    rt = G.nwg.Runtime(action_count, population, columns)
    rt.bootstrap(population, seed=4242)
    sizes = [5, 7, 131, 9]
    lists = [rng.choice(action_count, size=s, replace=False).astype(np.uint32) for s in sizes]
    offsets = np.zeros(population + 1, np.uint32)
    offsets[1:] = np.cumsum(sizes)
    rt.set_cell_words(offsets, np.concatenate(lists))
    counts = G.nwg.capi.word_counts(training=action_count, action_space=action_count)
    episodes = 3 * max(sizes)
    oc, ot, os_, op = _run_ours(rt, counts, episodes)
    gen = rt.current_generation()
    O.set_fma_mode(True)
    for i in range(population):
        genome = rt.download_slot(int(gen["slots"][i])).view(np.uint16)
        res = O.evaluate_individual(genome, action_count, catalog, lists[i], trace_policy=True)
        assert res["status"] == 0
        w3 = 3 * sizes[i]
        assert np.array_equal(ot[i, :w3], res["turns"])
        assert np.array_equal(os_[i, :w3], res["scores"])
        # oracle records every turn (prefilled ones too); ours records the policy's decisions
        for e in range(w3):
            pre = 0 if e % 3 == 0 else 2
            decided = res["guesses"][e][pre:res["turns"][e]]
            assert np.array_equal(oc[i, e, :len(decided)], decided)
            assert np.all(op[i, e, :len(decided)] == res["policy"][e, :len(decided)])
        assert gen["fitness"][i] == O.normalize_fitness(res["raw"], sizes[i])
    stats = rt.stats()
    assert stats.game_steps == sum(
        O.evaluate_individual(rt.download_slot(int(gen["slots"][i])).view(np.uint16), action_count, catalog,
                              lists[i])["steps"] for i in range(population))


@pytest.mark.skipif(O.ref_ckpt() is None, reason="reference runtime library not built")
@pytest.mark.parametrize("action_count,training,population,columns,forms", [
    (20, 20, 9, 3, (0, 1, 2, 3, 4)), (60, 60, 16, 4, (0, 2, 4)), (100, 40, 16, 4, (0, 3)),
    (127, 127, 9, 3, (0,)), (128, 64, 16, 4, (0, 1, 4)), (129, 129, 9, 3, (0, 1, 2)), (300, 30, 16, 4, (0, 2))])
def test_runtime_evaluation_matches_reference_runtime(action_count, training, population, columns, forms):
    """The reference's whole evaluation (TryEvaluateCurrentGenerationFitnessOnDevice) against ours, on both sides of
    its switch at 128 selectable actions (slab_runtime.cu:70, :1126-1140): FP16 tensor-tile scoring at or below it,
    FP32 warp scoring above it. Fitness bits, evaluation counts and the summary agree; at or below 128 actions every
    evaluation form takes the tensor-tile path."""
    import ctypes as C

    rng = np.random.default_rng(action_count * 7 + training)
    catalog = H.synthetic_words(rng, action_count)
    G.upload_catalog_everywhere(catalog)
    capi = G.nwg.capi
    counts = capi.word_counts(training=training, action_space=action_count)
    stride = capi.genome_stride_bytes(action_count)
    rc = capi.RuntimeConfig()
    rc.genotype_slab_byte_budget_bytes = 2 * population * stride
    rc.generation_byte_budget_bytes = population * stride
    rc.action_count, rc.population_size_ceiling, rc.grid_column_count = action_count, population, columns
    fit = np.zeros(population, np.float32)
    evals = np.zeros(population, np.uint32)
    has = np.zeros(population, np.uint8)
    summary = capi.FitnessSummary()
    assert O.ref_ckpt().refckpt_runtime_evaluate(C.addressof(rc), catalog.ctypes.data, len(catalog), population,
                                                 31 + action_count, 3, C.addressof(counts), None, fit.ctypes.data,
                                                 evals.ctypes.data, has.ctypes.data, C.addressof(summary)) == 1
    rt = G.nwg.Runtime(action_count, population, columns)
    rt.bootstrap(population, seed=31 + action_count, generation_index=3)
    for form in forms:
        rt.set_form(form)
        if form >= 3:
            rt.set_margin_guard(1.0e30)
        rt.evaluate(counts)
        gen = rt.current_generation()
        assert np.array_equal(gen["fitness"].view(np.uint32), fit.view(np.uint32)), f"form {form}"
        assert np.array_equal(gen["evaluation_counts"], evals) and np.array_equal(gen["has_fitness"], has)
        s = rt.summary()
        assert (s.best_fitness, s.average_fitness, s.best_index, s.generation_index, s.population_size) == (
            summary.best_fitness, summary.average_fitness, summary.best_index, summary.generation_index,
            summary.population_size)
    rt.close()


def test_evaluation_error_statuses():
    """Prefill that wins and then appends (W = 1) and an action space that runs out are reported, not trapped."""
    rng = np.random.default_rng(13)
    catalog = H.synthetic_words(rng, 8)
    G.upload_catalog_everywhere(catalog)
    rt = G.nwg.Runtime(8, 2, 2)
    rt.bootstrap(2, seed=5)
    rt.set_cell_words(np.array([0, 1, 2], np.uint32), np.array([3, 4], np.uint32))
    counts = G.nwg.capi.word_counts(training=8, action_space=8)
    with pytest.raises(G.nwg.NwgError) as err:
        rt.evaluate(counts)
    assert err.value.status == 6  # kGuessAppendFailed
    rt.set_cell_words(np.array([0, 5, 10], np.uint32), np.array([3, 4, 5, 6, 7, 3, 4, 5, 6, 7], np.uint32))
    counts1 = G.nwg.capi.word_counts(training=1, action_space=1)
    with pytest.raises(G.nwg.NwgError) as err:
        rt.evaluate(counts1)
    assert err.value.status == 8  # kActionSelectionFailed
    rt.evaluate(counts)  # the runtime stays usable
    assert rt.status() == 0
