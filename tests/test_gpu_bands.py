"""The row-band split on one GPU: two bands of one population, driven in one process, against one runtime holding
the whole grid.

Each generation the bands evaluate their own rows, their fitness is concatenated (what the all-gather does across
ranks), each band selects its children over the whole grid (nwg_band_prepare), copies out its boundary rows and
installs its neighbour's (what the halo exchange does across ranks), then breeds (nwg_assemble_prepared). The
parent pairs, the children's images and the fitness must equal the whole runtime's bit for bit, generation after
generation: the children's random streams are their whole-grid indices.
"""
import importlib

import numpy as np
import pytest

from tests import gpu_util as G
from tests import helpers as H

pytestmark = pytest.mark.gpu
bands_mod = importlib.import_module("neuroevolutionary-wordle_b200.bands")


def _images(rt):
    gen = rt.current_generation()
    return [rt.download_slot(int(s)) for s in gen["slots"]]


@pytest.mark.parametrize("rows,cols,radius,halo,form", [(8, 4, 1, 1, 0), (8, 3, 2, 2, 0), (12, 4, 1, 1, 4)])
def test_two_bands_equal_the_whole_population(rows, cols, radius, halo, form):
    t = G.torch()
    action_count, per_cell = 160, 6
    rng = np.random.default_rng(rows * 10 + radius)
    catalog = H.synthetic_words(rng, action_count)
    G.nwg.capi.upload_catalog(catalog)
    population = rows * cols
    offsets = np.arange(population + 1, dtype=np.uint32) * per_cell
    words = np.concatenate([rng.choice(action_count, per_cell, replace=False) for _ in range(population)])
    words = words.astype(np.uint32)
    counts = G.nwg.capi.word_counts(training=action_count, action_space=action_count)
    cfg = G.nwg.capi.assembly_config(radius=radius, p=0.05, sigma=0.02)
    whole = G.nwg.Runtime(action_count, population, cols, stream=G.stream_handle())
    whole.set_form(form)
    whole.set_margin_guard(1e-3)
    whole.bootstrap(population, seed=9)
    whole.set_cell_words(offsets, words)
    parts = [bands_mod.BandRuntime(bands_mod.band_layout(rows, cols, 2, k, halo), action_count) for k in range(2)]
    for b in parts:
        b.rt.set_form(form)
        b.rt.set_margin_guard(1e-3)
        b.bootstrap(9)
        b.set_cell_words(offsets, words)
    assert all(np.array_equal(x, y) for x, y in zip(_images(whole), _images(parts[0].rt) + _images(parts[1].rt)))

    for generation in range(3):
        seed = 500 + generation
        whole.evaluate(counts)
        expected_fitness = whole.current_generation()["fitness"].copy()
        whole.advance(seed=seed, counts=counts, config=cfg)
        for b in parts:
            b.rt.evaluate(counts)
        fitness = t.cat([b.local_fitness()[0] for b in parts])
        has = t.cat([b.local_fitness()[1] for b in parts])
        assert np.array_equal(fitness.cpu().numpy().view(np.uint32), expected_fitness.view(np.uint32))
        for b in parts:
            b.fitness_all.copy_(fitness)
            b.has_all.copy_(has)
            b.rt.band_prepare(seed, cfg, b.fitness_all.data_ptr(), b.has_all.data_ptr())
            b.stage_halo()
        t.cuda.synchronize()
        for k, b in enumerate(parts):  # what the halo exchange delivers: the other band's boundary rows
            other = parts[1 - k]
            b.recv_above.copy_(other.send_last)
            b.recv_below.copy_(other.send_first)
        t.cuda.synchronize()
        for b in parts:
            b.install_halo()
            b.rt.assemble()
        plan = np.concatenate([b.rt.assembly_plan() for b in parts])
        assert np.array_equal(plan, whole.assembly_plan()), f"generation {generation}: parent pairs differ"
        got = _images(parts[0].rt) + _images(parts[1].rt)
        for c, (x, y) in enumerate(zip(_images(whole), got)):
            assert np.array_equal(x, y), f"generation {generation}: child {c} differs"
    for b in parts:
        b.close()
    whole.close()


def test_band_refuses_the_whole_grid_paths_and_a_missing_halo():
    action_count, rows, cols = 140, 8, 4
    rng = np.random.default_rng(2)
    G.nwg.capi.upload_catalog(H.synthetic_words(rng, action_count))
    band = bands_mod.BandRuntime(bands_mod.band_layout(rows, cols, 2, 1, 1), action_count)
    band.bootstrap(3)
    cells = band.layout.cells
    band.rt.set_cell_words(np.arange(cells + 1, dtype=np.uint32) * 5,
                           np.concatenate([rng.choice(action_count, 5, replace=False) for _ in range(cells)]))
    counts = G.nwg.capi.word_counts(training=action_count, action_space=action_count)
    with pytest.raises(G.nwg.NwgError) as err:
        band.rt.advance(seed=1, counts=counts)
    assert err.value.status == 18  # NWG_UNSUPPORTED: a band selects over the whole grid
    band.rt.evaluate(counts)
    fitness, has = band.local_fitness()
    band.fitness_all.fill_(0.5)
    band.has_all.fill_(1)
    band.rt.band_prepare(1, G.nwg.capi.assembly_config(radius=1), band.fitness_all.data_ptr(),
                         band.has_all.data_ptr())
    with pytest.raises(G.nwg.NwgError) as err:
        band.rt.assemble()
    assert err.value.status == 12  # NWG_INVALID_ASSEMBLY_PLAN: no halo installed for this generation
    with pytest.raises(G.nwg.NwgError) as err:
        band.rt.band_prepare(1, G.nwg.capi.assembly_config(radius=2), band.fitness_all.data_ptr(),
                             band.has_all.data_ptr())
    assert err.value.status == 10  # radius beyond the one-row halo
    band.close()
