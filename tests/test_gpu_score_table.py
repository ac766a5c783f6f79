"""The 16-bit score table of the tensor-core forms against a numpy restatement.

Per individual: the header (max |e_ak| over the selectable actions, per column), the embedding rows (26 fixed
letter-count features from the catalog, -1 for an absent letter, then the genome's 38 tail values) rounded to
FP16 or BF16 in the K-major core-matrix layout with zero rows past the last action, and per 128-action tile the
column sums and sums of squares: each quarter of 32 actions summed in ascending order in float32 with every
operation rounded on its own, then the quarters added left to right. The scoring forms (1/2) read no moments and
their build skips them, so for those forms the header and the embedding tiles are compared.
"""
import numpy as np
import pytest

from oracle import pyoracle as O
from tests import gpu_util as G
from tests import helpers as H

pytestmark = pytest.mark.gpu

KIND = {1: "bf16", 2: "fp16", 3: "bf16", 4: "fp16"}


def _tile_offsets():
    r = np.arange(128)[:, None]
    k = np.arange(64)[None, :]
    return (r >> 3) * 1024 + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2


def _expected(genome: np.ndarray, catalog: np.ndarray, selectable: int, kind: str) -> bytes:
    tiles = (selectable + 127) // 128
    counts = np.zeros((selectable, 26), np.float32)
    for p in range(5):
        np.add.at(counts, (np.arange(selectable), catalog[:selectable, p].astype(np.int64)), 1.0)
    fixed = np.where(counts == 0, np.float32(-1.0), counts)
    start = O.genome_halfs(0)
    tail = genome.view(np.uint16)[start:start + 38 * selectable]
    tail = tail.view(np.float16).astype(np.float32).reshape(selectable, 38)
    e = np.zeros((tiles * 128, 64), np.float32)
    e[:selectable, :26] = fixed
    e[:selectable, 26:] = tail
    if kind == "fp16":
        bits = e.astype(np.float16).view(np.uint16)
    else:
        bits = (O.bf16_round(e).view(np.uint32) >> 16).astype(np.uint16)
    out = np.zeros(256 + tiles * 16384 + tiles * 64 * 8, np.uint8)
    out[:256] = np.abs(e[:selectable]).max(axis=0).astype(np.float32).view(np.uint8)
    off = (_tile_offsets() // 2).ravel()
    moments = np.zeros((tiles, 64, 2), np.float32)
    for t in range(tiles):
        tile = np.zeros(8192, np.uint16)
        tile[off] = bits[t * 128:(t + 1) * 128].ravel()
        out[256 + t * 16384:256 + (t + 1) * 16384] = tile.view(np.uint8)
        et = e[t * 128:(t + 1) * 128]
        parts = []
        for q in range(4):
            s = np.zeros(64, np.float32)
            sq = np.zeros(64, np.float32)
            for i in range(32):
                x = et[q * 32 + i]
                s = (s + x).astype(np.float32)
                sq = (sq + (x * x).astype(np.float32)).astype(np.float32)
            parts.append((s, sq))
        for j in (0, 1):
            moments[t, :, j] = ((parts[0][j] + parts[1][j]) + parts[2][j]) + parts[3][j]
    out[256 + tiles * 16384:] = moments.view(np.uint8).ravel()
    return out.tobytes()


@pytest.mark.parametrize("form", [2, 3])
@pytest.mark.parametrize("action_count,selectable", [(300, 300), (4739, 4739), (1000, 777)])
def test_score_table_matches_restatement(form, action_count, selectable):
    rng = np.random.default_rng(action_count + selectable + form)
    catalog = H.synthetic_words(rng, action_count)
    G.nwg.capi.upload_catalog(catalog)
    population = 4
    rt = G.nwg.Runtime(action_count, population, 2)
    rt.bootstrap(population, seed=action_count)
    words = np.concatenate([rng.choice(selectable, size=9, replace=False) for _ in range(population)])
    rt.set_cell_words(np.arange(population + 1, dtype=np.uint32) * 9, words.astype(np.uint32))
    rt.set_form(form)
    counts = G.nwg.capi.word_counts(training=selectable, action_space=selectable)
    rt.evaluate(counts)
    slots = rt.current_generation()["slots"]
    compared = 256 + (selectable + 127) // 128 * 16384 if form in (1, 2) else None
    for i in range(population):
        got = rt.score_table(i)
        want = _expected(rt.download_slot(int(slots[i])), catalog, selectable, KIND[form])
        assert got.tobytes()[:compared] == want[:compared], f"individual {i}"
    rt.close()
