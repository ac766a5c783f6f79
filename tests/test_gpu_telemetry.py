"""Shard-release statistics on the B200: fitness telemetry, convergence metrics and the release decision.

Reference: TryCollectGenerationFitnessTelemetry (cli/run_genetic_algorithm.cu:1080-1186),
TryCollectGeneticConvergenceTelemetry (:941-1054) with genetic_convergence.hpp:86-194, and
TryMaybeReleaseTrainingDataShard (:1199-1282). The GPU rows are compared bit for bit with the oracle's
restatement of the fitness row (on the downloaded fitness) and with the reference's own TryComputeMetrics (on the
sampled values gathered on the host from downloaded genomes, with the reference's own sample plan).
"""
import numpy as np
import pytest

from oracle import pyoracle as O
from tests import gpu_util as G
from tests import helpers as H

pytestmark = pytest.mark.gpu
capi = G.nwg.capi
POLICY_HALFS = 150528


def _runtime(action_count, population, columns, seed, per_cell=4):
    rng = np.random.default_rng(seed)
    catalog = H.synthetic_words(rng, action_count)
    G.upload_catalog_everywhere(catalog)
    rt = G.nwg.Runtime(action_count, population, columns)
    rt.bootstrap(population, seed=seed, generation_index=2)
    words = np.concatenate([rng.choice(action_count, per_cell, replace=False) for _ in range(population)])
    rt.set_cell_words(np.arange(population + 1, dtype=np.uint32) * per_cell, words.astype(np.uint32))
    return rt, catalog, capi.word_counts(training=action_count, action_space=action_count)


@pytest.mark.parametrize("action_count,population,columns", [(300, 300, 10), (4739, 4096, 64), (150, 8, 2)])
def test_fitness_telemetry_matches_oracle(action_count, population, columns):
    rt, _, counts = _runtime(action_count, population, columns, action_count + population)
    with pytest.raises(capi.NwgError) as e:  # before evaluation
        rt.fitness_telemetry(counts)
    assert e.value.status == 9
    rt.prepare(5, counts, config=capi.assembly_config(radius=1))
    gen = rt.current_generation()
    plan = rt.assembly_plan()
    row = rt.fitness_telemetry(counts, with_breeding=True)
    ref = O.fitness_telemetry(gen["fitness"], plan)
    for ours, key in ((row.fitness_min, "min"), (row.fitness_max, "max"), (row.fitness_mean, "mean"),
                      (row.fitness_median, "median"), (row.fitness_p90, "p90"), (row.fitness_p99, "p99"),
                      (row.fitness_stddev, "stddev")):
        assert np.float32(ours).view(np.uint32) == np.float32(ref[key]).view(np.uint32), key
    assert row.distinct_fitness_count == ref["distinct"]
    assert (row.generation, row.population_size, row.training_word_count) == (2, population, action_count)
    assert row.has_breeding_metrics
    assert (row.parent_childless_count, row.parent_one_child_count, row.parent_multiple_children_count) == (
        ref["childless"], ref["one_child"], ref["more"])
    rt.close()


@pytest.mark.skipif(O.ref_ckpt() is None, reason="reference library not built")
@pytest.mark.parametrize("action_count,population,columns,seed", [(300, 64, 8, 11), (4739, 4096, 64, 7),
                                                                  (200, 2, 2, 3)])
def test_convergence_telemetry_matches_reference(action_count, population, columns, seed):
    rt, _, counts = _runtime(action_count, population, columns, seed)
    rt.advance(9, counts, config=capi.assembly_config(radius=1, p=0.05, sigma=0.02))  # a bred generation
    row = rt.convergence_telemetry(seed)
    gen = rt.current_generation()
    trainable = POLICY_HALFS + 38 * action_count
    org, w, pairs = O.ref_convergence_plan(population, trainable, seed, int(gen["generation_index"]))
    assert (row.sample_organisms, row.sample_weights, row.pair_count) == (len(org), len(w), len(pairs))
    values = np.stack([rt.download_slot(int(gen["slots"][int(o)])).view(np.float16)[w.astype(np.int64)]
                       for o in org]).astype(np.float32)
    ref = O.ref_convergence_metrics(values, pairs)
    ours = np.array([row.centroid_distance_mean, row.centroid_distance_min, row.centroid_distance_max,
                     row.pairwise_distance_mean, row.pairwise_distance_min, row.pairwise_distance_max], np.float32)
    assert np.array_equal(ours.view(np.uint32), ref.view(np.uint32))
    assert row.generation == gen["generation_index"] and row.elapsed_ms > 0
    rt.close()


def test_release_decision_follows_the_reference_rules():
    action_count, catalog_count, population, columns = 200, 260, 16, 4
    rt, _, _ = _runtime(action_count, population, columns, 21)
    G.upload_catalog_everywhere(H.synthetic_words(np.random.default_rng(2), catalog_count))
    counts = capi.word_counts(training=action_count, action_space=action_count, initial=150, step=50, period=1)
    rt.evaluate(capi.word_counts(training=action_count, action_space=action_count))
    release_all = capi.ShardReleasePolicy(0, 0, 1.0e9, -1.0)
    history = capi.ShardReleaseHistory()
    with pytest.raises(capi.NwgError) as e:  # no foundation release record
        rt.maybe_release_training_shard(counts, release_all, catalog_count, 1, history)
    assert e.value.status == 5
    history.release_count = 1  # the foundation release at generation 0
    pending, nxt, f, c = rt.maybe_release_training_shard(counts, capi.ShardReleasePolicy(), catalog_count, 1, history)
    assert not pending.enabled and nxt == action_count and f.population_size == 0  # before the first new generation
    history.release_generations[0] = 2
    pending, nxt, f, c = rt.maybe_release_training_shard(counts, capi.ShardReleasePolicy(0, 0, 6.0, 2.0),
                                                         catalog_count, 1, history)
    assert not pending.enabled and f.population_size == population and c.sample_organisms == population  # p99 < 2
    pending, nxt, f, c = rt.maybe_release_training_shard(counts, release_all, catalog_count, 1, history)
    assert pending.enabled and (pending.first_catalog_word_index, pending.injection_count) == (action_count, 50)
    assert nxt == action_count + 50 and history.release_count == 2
    assert history.release_generations[1] == 3 and history.release_fitness_p99[1] == f.fitness_p99
    pending, nxt, f, c = rt.maybe_release_training_shard(counts, capi.ShardReleasePolicy(3, 0, 1.0e9, -1.0),
                                                         catalog_count, 1, history)
    assert not pending.enabled and history.release_count == 2  # within the minimum gap
    near_end = capi.word_counts(training=action_count, action_space=catalog_count - 10, initial=150, step=50,
                                period=1)
    history.release_generations[1] = 0
    history.release_count = 1
    pending, nxt, f, c = rt.maybe_release_training_shard(near_end, release_all, catalog_count, 1, history)
    assert pending.enabled and pending.injection_count == 10 and nxt == catalog_count  # the catalog's remainder
    rt.close()
