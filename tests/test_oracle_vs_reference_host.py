"""Validates the oracle restatement against the reference's own host build (oracle/_ref/libref_host.so).

The reference host build rounds each multiply and add separately (no FMA contraction), so
the oracle is compared bit for bit in that mode; in its default mode the oracle follows the
reference's device arithmetic (fused multiply-add), which stays within 1e-5 of the host
result relative to the output's magnitude.
"""
import numpy as np
import pytest

from oracle import pyoracle as O
from tests import helpers as H

pytestmark = pytest.mark.skipif(O.ref_host() is None, reason="reference host library not built")


def random_grid(rng, catalog, turns):
    sol = catalog[rng.integers(len(catalog))]
    idx = rng.choice(len(catalog), size=turns, replace=False)
    guesses = catalog[idx]
    # a grid that is already won is not a valid decision state
    guesses = np.array([g for g in guesses if not np.array_equal(g, sol)])[:turns]
    return sol, guesses.reshape(-1, 5)


@pytest.fixture(autouse=True)
def _fma_default():
    yield
    O.set_fma_mode(True)


def test_policy_forward_bit_exact_against_reference_host():
    rng = np.random.default_rng(1)
    catalog = H.synthetic_words(rng, 64)
    O.set_fma_mode(False)
    for trial in range(6):
        g = H.random_genome(rng, 8)
        for turns in range(6):
            sol, guesses = random_grid(rng, catalog, turns)
            a = O.policy_forward(g, sol, guesses)
            b = O.ref_host_policy_forward(g, sol, guesses)
            assert a is not None and b is not None
            assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), (trial, turns)


def test_policy_forward_fma_within_tolerance():
    rng = np.random.default_rng(2)
    catalog = H.synthetic_words(rng, 64)
    for _ in range(4):
        g = H.random_genome(rng, 8)
        for turns in range(6):
            sol, guesses = random_grid(rng, catalog, turns)
            a = O.policy_forward(g, sol, guesses)
            b = O.ref_host_policy_forward(g, sol, guesses)
            scale = max(1.0, float(np.abs(b).max()))
            assert np.max(np.abs(a - b)) <= 1e-5 * scale


def test_policy_forward_rejects_finished_grid():
    rng = np.random.default_rng(3)
    catalog = H.synthetic_words(rng, 16)
    g = H.random_genome(rng, 4)
    sol = catalog[0]
    assert O.policy_forward(g, sol, sol.reshape(1, 5)) is None
    assert O.ref_host_policy_forward(g, sol, sol.reshape(1, 5)) is None


@pytest.mark.parametrize("action_count,w", [(48, 6), (40, 2), (130, 5)])
def test_episode_evaluation_matches_reference_host(action_count, w):
    rng = np.random.default_rng(action_count + w)
    catalog = H.synthetic_words(rng, action_count)
    O.set_fma_mode(False)
    genomes = np.stack([H.random_genome(rng, action_count) for _ in range(3)])
    cell_words = rng.choice(action_count, size=w, replace=False).astype(np.uint32)
    offsets = np.array([0, w], np.uint32)
    raw, steps, status = O.ref_host_evaluate(genomes, action_count, catalog, offsets, cell_words,
                                             np.zeros(3, np.uint32), threads=2)
    for i in range(3):
        res = O.evaluate_individual(genomes[i], action_count, catalog, cell_words)
        assert res["status"] == 0 and status[i] == 0
        assert res["raw"] == raw[i]
        assert res["steps"] == steps[i]


def test_cell_words_from_shards_covers_by_radius():
    # one global foundation shard plus a radius-0 shard centred on cell 7 of a 5x5 grid
    shards = [O.ShardRecord(0, 20, 0, 0, 0, 1), O.ShardRecord(20, 10, 1, 2, 0, 0)]
    center = O.cell_words_from_shards(shards, 5, 5, 7)
    other = O.cell_words_from_shards(shards, 5, 5, 8)
    assert center.tolist() == list(range(30))
    assert other.tolist() == list(range(20))
    shards[1].radius = 1
    assert len(O.cell_words_from_shards(shards, 5, 5, 8)) == 30
    assert len(O.cell_words_from_shards(shards, 5, 5, 9)) == 20
