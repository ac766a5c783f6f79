"""Shard-release statistics on the host (no GPU): the convergence sample plan and the metric reductions.

Reference: MakeSamplePlan and TryComputeMetrics (genetic_algorithm/genetic_convergence.hpp:86-194), compiled from
its header into oracle/_ref/libref_ckpt.so; the fitness telemetry of cli/run_genetic_algorithm.cu:1100-1183, which
lives in the reference's CLI translation unit, is restated in oracle/pyoracle.py and checked here on hand-worked
cases. The library's plan (nwg_convergence_sample_plan, host code) equals the reference's draw for draw, and the
oracle's float32 restatement of the metrics equals the reference's bit for bit, so the GPU tests can use either.
"""
import importlib

import numpy as np
import pytest

from oracle import pyoracle as O

nwg = importlib.import_module("neuroevolutionary-wordle_b200")
needs_ref = pytest.mark.skipif(O.ref_ckpt() is None, reason="reference checkpoint library not built")


@needs_ref
@pytest.mark.parametrize("organisms,trainable,seed,generation", [
    (4096, 150528 + 38 * 4739, 0, 0), (4096, 150528 + 38 * 512, 12345, 17), (300, 9000, 7, 3),
    (256, 20000, 1, 1), (100, 5000, 2, 9), (1, 8192, 3, 0), (2, 10, 4, 2), (16384, 150528 + 38 * 1024, 99, 50)])
def test_sample_plan_matches_reference(organisms, trainable, seed, generation):
    org, w, pairs = nwg.capi.convergence_sample_plan(organisms, trainable, seed, generation)
    r_org, r_w, r_pairs = O.ref_convergence_plan(organisms, trainable, seed, generation)
    assert np.array_equal(org, r_org) and np.array_equal(w, r_w) and np.array_equal(pairs, r_pairs)
    assert len(set(org.tolist())) == len(org) == min(256, organisms)
    assert len(set(w.tolist())) == len(w) == min(8192, trainable)
    assert len(pairs) == (512 if len(org) >= 2 else 0)
    if len(pairs):
        assert np.all(pairs[:, 0] != pairs[:, 1]) and pairs.max() < len(org)


@needs_ref
@pytest.mark.parametrize("organisms,weights,pairs,scale", [(256, 8192, 512, 0.05), (7, 33, 40, 1.0),
                                                           (2, 5, 0, 3.0), (31, 100, 64, 1e-3)])
def test_metric_restatement_matches_reference(organisms, weights, pairs, scale):
    rng = np.random.default_rng(organisms * 31 + weights)
    values = (rng.standard_normal((organisms, weights)) * scale).astype(np.float16).astype(np.float32)
    first = rng.integers(0, organisms, pairs)
    second = (first + 1 + rng.integers(0, organisms - 1, pairs)) % organisms
    p = np.stack([first, second], 1)
    ours = O.convergence_metrics(values, p)
    ref = O.ref_convergence_metrics(values, p)
    assert np.array_equal(ours.view(np.uint32), ref.view(np.uint32))


@needs_ref
def test_metrics_of_identical_organisms_match_reference():
    values = np.tile(np.linspace(-1, 1, 50, dtype=np.float32), (6, 1))
    p = np.array([[0, 1], [2, 3]])
    ref = O.ref_convergence_metrics(values, p)
    assert np.array_equal(O.convergence_metrics(values, p).view(np.uint32), ref.view(np.uint32))
    assert np.array_equal(ref[3:], np.zeros(3, np.float32))  # the centroid (sum x 1/6) is not exactly x in float
    assert 0 < ref[0] < 1e-6


def test_fitness_telemetry_restatement_on_worked_cases():
    t = O.fitness_telemetry(np.array([0.5, 0.1, 0.3, 0.3], np.float32))
    assert (t["min"], t["max"], t["median"], t["distinct"]) == (np.float32(0.1), np.float32(0.5), np.float32(0.3), 3)
    assert t["p90"] == np.float32(0.5) and t["p99"] == np.float32(0.5)  # ceil(0.9 * 4) = 4 -> index 3
    assert t["mean"] == np.float32((0.1 + 0.3 + 0.3 + 0.5) / 4) or abs(t["mean"] - 0.3) < 1e-7
    odd = O.fitness_telemetry(np.arange(1, 101, dtype=np.float32) / 100, np.array([[0, 1], [0, 2], [5, 0]]))
    assert odd["median"] == np.float32(0.5) or odd["median"] == np.float32((np.float32(0.5) + np.float32(0.51)) * 0.5)
    assert odd["p90"] == np.float32(0.9) and odd["p99"] == np.float32(0.99)
    assert (odd["childless"], odd["one_child"], odd["more"]) == (96, 3, 1)
    one = O.fitness_telemetry(np.array([0.25], np.float32))
    assert one["stddev"] == 0 and one["median"] == np.float32(0.25) and one["distinct"] == 1
