"""The row-band split of one population on two gloo ranks (CPU): index arithmetic and both collectives.

Each rank holds one band of an 8 x 4 grid (radius-1 halo). With the fitness gathered from the bands, the
children's parent pairs drawn by the CPU oracle's selection (selection_ops.cuh:218-263 restated; the random draws
are synthetic per child, the same in both runs) equal the single-population plan; every parent a band's children
name lies in the band or its halo rows; and the halo exchange delivers exactly the neighbours' boundary rows
(genome stand-ins tagged with their global row and column), so every parent a child needs is found locally.
"""
import importlib
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent
ROWS, COLS, HALO, RADIUS = 8, 4, 1, 1
GENOME = 24  # bytes per stand-in genome: global row and column, then filler


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _fitness():
    rng = np.random.default_rng(17)
    return (rng.integers(0, 5, ROWS * COLS) / 7.0).astype(np.float32)  # many ties


def _draws(child):
    d = np.random.default_rng(1000 + child).integers(0, 2**32, 6, dtype=np.uint64).astype(np.uint32)
    for k in (2, 5):  # the two uniforms in (0, 1]
        d[k] = np.float32((child * 37 % 97 + k) / 103.0).view(np.uint32)
    return d


def _plan(fitness, children):
    from oracle import pyoracle as O

    weights = np.power(np.arange(32, dtype=np.float32), 0.5).astype(np.float32)
    has = np.ones(ROWS * COLS, np.uint8)
    return [O.select_parent_pair(fitness, has, ROWS, COLS, ROWS, c, RADIUS, _draws(c), weights) for c in children]


def _genome(row, col):
    g = np.zeros(GENOME, np.uint8)
    g[0], g[1] = row, col
    g[2:] = (row * COLS + col) % 251
    return g


def _rank(rank, world, port, out):
    import datetime

    import torch
    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    bands = importlib.import_module("neuroevolutionary-wordle_b200.bands")
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    layout = bands.band_layout(ROWS, COLS, world, rank, HALO)
    fitness = _fitness()
    local = torch.from_numpy(fitness[layout.first_cell:layout.first_cell + layout.cells].copy())
    gathered = torch.zeros(ROWS * COLS, dtype=torch.float32)
    bands.gather_bands(local, gathered)
    children = range(layout.first_cell, layout.first_cell + layout.cells)
    pairs = _plan(gathered.numpy(), children)

    # halo exchange of stand-in genomes: the band's rows, then its first and last halo rows sent to the neighbours
    own = {(layout.first_row + r, c): _genome(layout.first_row + r, c) for r in range(layout.rows)
           for c in range(COLS)}
    first = torch.from_numpy(np.concatenate([own[(layout.first_row + r, c)] for r in range(HALO) for c in range(COLS)]))
    last_row0 = layout.first_row + layout.rows - HALO
    last = torch.from_numpy(np.concatenate([own[(last_row0 + r, c)] for r in range(HALO) for c in range(COLS)]))
    above = torch.zeros(HALO * COLS * GENOME, dtype=torch.uint8)
    below = torch.zeros_like(above)
    bands.exchange_halo(layout, first, last, above, below)
    held = dict(own)
    for rows, buf in ((layout.above_rows(), above.numpy()), (layout.below_rows(), below.numpy())):
        for j, row in enumerate(rows):
            for c in range(COLS):
                held[(row, c)] = buf[(j * COLS + c) * GENOME:(j * COLS + c + 1) * GENOME].copy()
    out[rank] = {"pairs": pairs, "held": held, "parent_rows": layout.parent_rows(),
                 "above": layout.above_rows(), "below": layout.below_rows()}
    dist.destroy_process_group()


@pytest.mark.timeout(180)
def test_two_band_plan_and_halo_equal_the_whole_population():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(150)
        assert p.exitcode == 0
    sys.path.insert(0, str(ROOT))
    whole = _plan(_fitness(), range(ROWS * COLS))
    assert all(pair is not None for pair in whole)
    banded = out[0]["pairs"] + out[1]["pairs"]
    assert banded == whole  # the 2-band plan is the 1-band plan
    for rank in range(world):
        r = out[rank]
        assert r["above"] == [(rank * 4 - 1) % ROWS] and r["below"] == [(rank * 4 + 4) % ROWS]
        for first_parent, second_parent in r["pairs"]:
            for parent in (first_parent, second_parent):
                row, col = divmod(parent, COLS)
                assert row in r["parent_rows"]  # the halo covers every parent the band's children name
                assert np.array_equal(r["held"][(row, col)], _genome(row, col))  # and holds the right genome


def test_band_layout_rejects_bands_its_halo_cannot_cover():
    sys.path.insert(0, str(ROOT))
    bands = importlib.import_module("neuroevolutionary-wordle_b200.bands")
    layout = bands.band_layout(64, 64, 8, 3, 1)
    assert (layout.first_row, layout.rows, layout.previous, layout.next) == (24, 8, 2, 4)
    assert layout.above_rows() == [23] and layout.below_rows() == [32]
    assert bands.band_layout(64, 64, 8, 0, 2).above_rows() == [62, 63]
    with pytest.raises(ValueError):
        bands.band_layout(64, 64, 3, 0, 1)  # unequal bands
    with pytest.raises(ValueError):
        bands.band_layout(8, 4, 8, 0, 2)  # one-row bands cannot carry a two-row halo
    with pytest.raises(ValueError):
        bands.band_layout(4, 4, 2, 0, 2)  # band plus halos exceed the grid
