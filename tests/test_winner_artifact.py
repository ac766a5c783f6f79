"""Winner artefacts on the host (no GPU): the reference's genome + JSON metadata pair.

Reference: TryWriteWinnerArtifactToPaths and TryReadWinnerArtifact (model_artifact/winner_artifact.cpp:13-188,
:218-280; winner_artifact_reader.cpp:12-247) and their test (tests/model_artifact/winner_artifact_reader_test.cpp:
CRANE/SLATE/TRACE, a 512-byte payload of (7 b) mod 251, generation 12, index 4, slot 19, seed 99). Checked against
the reference's own writer and reader compiled from its sources (oracle/_ref/libref_ckpt.so): each reads what the
other writes, and given the reference file's timestamp this library writes the same bytes.
"""
import ctypes as C
import importlib

import numpy as np
import pytest

from oracle import pyoracle as O

nwg = importlib.import_module("neuroevolutionary-wordle_b200")
capi = nwg.capi
needs_ref = pytest.mark.skipif(O.ref_ckpt() is None, reason="reference checkpoint library not built")


def _letters(*words):
    return np.array([[ord(c) - ord("A") for c in w] for w in words], np.uint8)


def _reference_test_case():
    genome = (np.arange(512) * 7 % 251).astype(np.uint8)
    m = capi.WinnerMetadata()
    m.best_fitness, m.generation_index, m.best_index, m.best_slot_index = 0.25, 12, 4, 19
    m.action_count, m.genome_byte_count, m.seed = 3, 512, 99
    return genome, m, _letters("CRANE", "SLATE", "TRACE")


def _ref_read(binary, metadata):
    meta = np.zeros(7, np.uint64)
    genome = np.zeros(1 << 20, np.uint8)
    letters = np.zeros((capi.CATALOG_CAPACITY, 5), np.uint8)
    count = C.c_size_t()
    path = C.create_string_buffer(4096)
    ok = O.ref_ckpt().refart_read(str(binary).encode(), str(metadata).encode(), meta.ctypes.data, genome.ctypes.data,
                                  genome.nbytes, letters.ctypes.data, C.byref(count), path, len(path))
    if ok != 1:
        return None
    return dict(meta=meta, genome=genome[:int(meta[5])], words=letters[:count.value], path=path.value.decode())


def test_round_trip_of_the_reference_test_case(tmp_path):
    genome, m, words = _reference_test_case()
    b, j = tmp_path / "w.bin", tmp_path / "w.json"
    capi.write_winner_artifact(b, j, genome, m, words, "data/action-space-randomised.txt", "2026-01-02T03:04:05")
    got = capi.read_winner_artifact(b, j)
    g = got["metadata"]
    assert (g.best_fitness, g.generation_index, g.best_index, g.best_slot_index, g.action_count,
            g.genome_byte_count, g.seed) == (0.25, 12, 4, 19, 3, 512, 99)
    assert np.array_equal(got["genome"], genome) and np.array_equal(got["words"], words)
    assert got["action_space_path"] == "data/action-space-randomised.txt"
    assert got["timestamp"] == "2026-01-02T03:04:05"
    text = j.read_text()
    assert text.startswith('{\n  "format_version": 2,\n') and '"action_space_words": ["CRANE", "SLATE", "TRACE"]' in text
    assert not (tmp_path / "w.bin.tmp").exists() and not (tmp_path / "w.json.tmp").exists()


@needs_ref
@pytest.mark.parametrize("fitness,count,path", [(0.25, 3, "data/a.txt"), (0.0651852, 40, 'odd "quoted"\tpath'),
                                                (1.0, 4739, "")])
def test_reference_reads_ours_and_we_rewrite_the_reference_file(tmp_path, fitness, count, path):
    rng = np.random.default_rng(count)
    words = rng.integers(0, 26, (count, 5)).astype(np.uint8)
    genome = rng.integers(0, 256, 4096 + count).astype(np.uint8)
    m = capi.WinnerMetadata()
    m.best_fitness, m.generation_index, m.best_index, m.best_slot_index = fitness, 7, count - 1, 0xFFFFFFFF
    m.action_count, m.genome_byte_count, m.seed = count, genome.nbytes, 12345
    ours_b, ours_j = tmp_path / "o.bin", tmp_path / "o.json"
    capi.write_winner_artifact(ours_b, ours_j, genome, m, words, path)
    r = _ref_read(ours_b, ours_j)
    assert r is not None
    assert np.array_equal(r["genome"], genome) and np.array_equal(r["words"], words) and r["path"] == path
    assert np.float32(fitness).view(np.uint32) == np.uint32(r["meta"][0]) or abs(
        np.uint32(r["meta"][0]).view(np.float32) - fitness) <= 1e-6 * max(1.0, fitness)
    assert list(r["meta"][1:]) == [7, count - 1, 0xFFFFFFFF, count, genome.nbytes, 12345]

    ref_b, ref_j = tmp_path / "r.bin", tmp_path / "r.json"
    meta = np.array([np.float32(fitness).view(np.uint32), 7, count - 1, 0xFFFFFFFF, count, genome.nbytes, 12345],
                    np.uint64)
    assert O.ref_ckpt().refart_write(str(ref_b).encode(), str(ref_j).encode(), genome.ctypes.data, words.ctypes.data,
                                     count, meta.ctypes.data, path.encode()) == 1
    theirs = capi.read_winner_artifact(ref_b, ref_j)
    assert np.array_equal(theirs["genome"], genome) and np.array_equal(theirs["words"], words)
    again_b, again_j = tmp_path / "a.bin", tmp_path / "a.json"
    capi.write_winner_artifact(again_b, again_j, genome, m, words, path, theirs["timestamp"])
    assert again_j.read_bytes() == ref_j.read_bytes()
    assert again_b.read_bytes() == ref_b.read_bytes()


def test_bad_artifacts_are_refused(tmp_path):
    genome, m, words = _reference_test_case()
    b, j = tmp_path / "w.bin", tmp_path / "w.json"
    capi.write_winner_artifact(b, j, genome, m, words, "p", "t")
    good = j.read_text()
    for bad in (good.replace('"format_version": 2', '"format_version": 3'), good.replace('"CRANE"', '"crane"'),
                good.replace('"CRANE"', '"CRAN"'), good.replace('"action_count": 3', '"action_count": 4'),
                good.replace('"genome_byte_count": 512', '"genome_byte_count": 511'),
                good.replace('"seed"', '"sead"')):
        j.write_text(bad)
        with pytest.raises(capi.NwgError):
            capi.read_winner_artifact(b, j)
        if O.ref_ckpt() is not None:
            assert _ref_read(b, j) is None
    j.write_text(good)
    b.write_bytes(b"")
    with pytest.raises(capi.NwgError):
        capi.read_winner_artifact(b, j)
    with pytest.raises(capi.NwgError):  # more actions than catalog words
        m.action_count = 4
        capi.write_winner_artifact(b, j, genome, m, words, "p", "t")
