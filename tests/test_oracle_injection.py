"""The oracle's hint grids and output-embedding injection, pinned to the reference's own tests.

Known answers: tests/wordle/hint_grid_test.cpp:138-229 (cyclic grid of SPARE uses its four rotations, AABCD only its
all-yellow rotations 2 and 3, the swap grid of LEVEL is ELVEL with feedback YYGGG, SPARE's group has swap
guesses PSARE and APSRE, AAAAA has no group). Injection properties: tests/genetic_algorithm/device/
slab_runtime_test.cu:670-690 (every injected row is finite, non-zero, with the median norm of the existing rows).
"""
import numpy as np
import pytest

from oracle import pyoracle as O
from tests import helpers as H


def word(s):
    return np.array([ord(c) - ord("A") for c in s], np.uint8)


def text(letters):
    return "".join(chr(ord("A") + int(x)) for x in letters)


FB = "GY-"


def test_cyclic_grid_of_an_isogram_uses_four_rotations():
    turns, guesses, fbs = O.hint_grid_group(word("SPARE"))
    assert turns == [4, 1, 1]
    assert [text(guesses[0][t]) for t in range(4)] == ["PARES", "ARESP", "RESPA", "ESPAR"]
    assert all("".join(FB[x] for x in fbs[0][t]) == "YYYYY" for t in range(4))


def test_cyclic_grid_skips_rotations_that_are_not_all_yellow():
    turns, guesses, fbs = O.hint_grid_group(word("AABCD"))
    assert turns[0] == 2
    assert [text(guesses[0][t]) for t in range(2)] == ["BCDAA", "CDAAB"]


def test_swap_grid_reads_three_green_two_yellow():
    turns, guesses, fbs = O.hint_grid_group(word("LEVEL"))
    assert text(guesses[1][0]) == "ELVEL"
    assert "".join(FB[x] for x in fbs[1][0]) == "YYGGG"


def test_group_has_two_distinct_swap_grids():
    turns, guesses, fbs = O.hint_grid_group(word("SPARE"))
    assert text(guesses[1][0]) == "PSARE" and text(guesses[2][0]) == "APSRE"
    for g in (1, 2):
        f = "".join(FB[x] for x in fbs[g][0])
        assert f.count("G") == 3 and f.count("Y") == 2


def test_monochrome_word_has_no_group():
    assert O.hint_grid_group(word("AAAAA")) is None


@pytest.mark.parametrize("parent,count", [(40, 3), (41, 5), (128, 1)])
def test_injected_rows_take_the_median_norm(parent, count):
    rng = np.random.default_rng(parent + count)
    catalog = H.synthetic_words(rng, parent + count)
    genome = H.random_genome(rng, parent + count)
    status, grown = O.inject_tails(genome, parent, catalog, parent, count)
    assert status == 0
    assert np.array_equal(grown[:O.genome_halfs(parent)], genome[:O.genome_halfs(parent)])
    target = O.median_tail_norm(genome, parent)
    rows = grown[O.genome_halfs(parent):].view(np.float16).astype(np.float32).reshape(count, 38)
    norms = np.sqrt((rows.astype(np.float64) ** 2).sum(1))
    assert np.all(np.isfinite(norms)) and np.all(norms > 0)
    np.testing.assert_allclose(norms, target, rtol=2e-3)


def test_injection_rejects_a_bad_range():
    rng = np.random.default_rng(3)
    catalog = H.synthetic_words(rng, 50)
    genome = H.random_genome(rng, 50)
    assert O.inject_tails(genome, 40, catalog, 41, 3)[0] == 2  # must start at the parent's action count
    assert O.inject_tails(genome, 40, catalog, 40, 20)[0] == 1  # beyond the catalog


def test_library_hint_group_availability_matches_oracle():
    """nwg_hint_groups_available (host code of the library) agrees with the oracle's hint-grid construction."""
    import importlib

    nwg = importlib.import_module("neuroevolutionary-wordle_b200")
    rng = np.random.default_rng(17)
    words = np.concatenate([rng.integers(0, 26, (3000, 5)), rng.integers(0, 3, (500, 5)),
                            np.array([[0, 0, 0, 0, 0], [1, 1, 1, 1, 2], [0, 1, 0, 1, 0], [2, 3, 4, 5, 6]])]).astype(np.uint8)
    got = nwg.capi.hint_groups_available(words)
    want = np.array([O.hint_grid_group(w) is not None for w in words])
    assert np.array_equal(got, want)
    assert not got[-4] and got[-1]  # a monochrome word has none; five distinct letters always do
