"""Pins the CPU oracle to the known-answer vectors of the reference's own tests.

Sources of the vectors (reference project paths):
  tests/wordle/wordle_grid_test.cpp:107-125           feedback rules incl. duplicate letters
  tests/model/input_encoder/shared_encoder_fixture.hpp encoder golden output (5.5, 8.0, 1.25)
  tests/model/policy_model/policy_model_fixture.hpp    virgin (-1.5, 4.375, 4.0) and single-turn outputs
  tests/inference/dynamic_policy_test.cu:144-232       3-word catalog: best = index 1, repeat masking
"""
import numpy as np
import pytest

from oracle import pyoracle as O
from tests import helpers as H

FB = {"G": 0, "Y": 1, "-": 2}


def fb(s):
    return np.array([FB[c] for c in s], np.uint8)


@pytest.mark.parametrize("guess,solution,expected", [
    ("CRANE", "SOLAR", "-YY--"),
    ("EERIE", "STEEL", "YY---"),
    ("HELLO", "LEVEL", "-GYY-"),
    ("LEVEL", "HELLO", "YG--Y"),
    ("ABCDE", "AEBDF", "GY-GY"),
    ("SOLAR", "SOLAR", "GGGGG"),
])
def test_feedback_known_answers(guess, solution, expected):
    out = O.feedback(O.word(guess), O.word(solution))
    assert np.array_equal(out, fb(expected))


def test_feedback_rejects_invalid_letters():
    bad = np.array([0, 1, 2, 3, 26], np.uint8)
    assert O.feedback(bad, O.word("SOLAR")) is None


def test_encoder_golden_fixture():
    g = H.empty_genome(3)
    H.encoder_fixture(g)
    out = O.encode_turn(g, O.word("ABCDE"), fb("GY-GY"))
    assert out[:3].tolist() == [5.5, 8.0, 1.25]
    assert np.all(out[3:] == 0.0)


def test_policy_golden_fixture_virgin_and_single_turn():
    g = H.empty_genome(3)
    H.policy_fixture(g)
    virgin = O.policy_forward(g, O.word("AEBDF"), np.zeros((0, 5), np.uint8))
    assert virgin[:3].tolist() == [-1.5, 4.375, 4.0]
    one = O.policy_forward(g, O.word("AEBDF"), O.word("ABCDE").reshape(1, 5))
    t0, t1, t2 = 5.5, 8.0, 1.25
    h00 = -1.0 + t0 + 0.5 * t1
    h01 = -0.25 * t1 + 2.0 * t2
    h10 = 0.25 + 0.5 * h00 + 2.0 * h01
    h11 = -1.0 + 0.25 * h00
    assert one[:3].tolist() == [-2.0 + 2.0 * h10, 0.5 - 0.5 * h10 + 4.0 * h11, 1.0 + 3.0 * h11]


def test_dynamic_policy_three_word_catalog():
    catalog = O.words_to_letters(["CABBY", "CACAO", "FUZZY"])
    g = H.empty_genome(3)
    H.policy_fixture(g)
    policy = O.policy_forward(g, O.word("AEBDF"), O.word("ABCDE").reshape(1, 5))
    tails = g[H.POLICY_HALFS:].reshape(3, 38)
    scores = [O.score_action(policy, catalog[a], tails[a]) for a in range(3)]
    assert int(np.argmax(scores)) == 1
    # After CABBY is guessed the mask skips it and CACAO stays the choice.
    policy2 = O.policy_forward(g, O.word("AEBDF"), np.stack([O.word("ABCDE"), catalog[0]]))
    scores2 = [O.score_action(policy2, catalog[a], tails[a]) for a in range(3)]
    scores2[0] = -np.inf
    assert int(np.argmax(scores2)) == 1


def test_fitness_normalisation():
    assert O.normalize_fitness(0.0, 20) == pytest.approx(1.40129846e-45, rel=0, abs=0) or \
        O.normalize_fitness(0.0, 20) > 0.0
    assert O.normalize_fitness(45.0 * 20, 20) == 1.0
    assert O.normalize_fitness(450.0, 20) == np.float32(450.0) / np.float32(900.0)
    assert O.normalize_fitness(10.0, 0) > 0.0


def test_stride_matches_reference_layout():
    assert O.lib().nwo_genome_stride_bytes(512) == 339968
    assert O.lib().nwo_genome_stride_bytes(1024) == 378880
    assert O.lib().nwo_genome_stride_bytes(4739) == 661220
    assert O.lib().nwo_genome_stride_bytes(0) == 0
