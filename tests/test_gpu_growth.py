"""Action-space growth on the B200: widening the slab and injecting new output-embedding rows.

Reference: TryAdvanceGenerationOnDevice with a pending output-embedding injection (slab_runtime.cu:1464-1482):
the children of the widening generation are bred with the parents' action count into slots of the wider
stride, then every child gets one new tail row per released word (genotype_slab/device_runtime.cu:518-617,
device/injection_ops.cuh:22-64). Checked bit for bit against the reference's own device functions
(oracle/_ref/libref_dev.so: BreedAndMutateGenome then TryInjectExpandedOutputEmbeddingTailsConcurrently) and
against the CPU oracle; runtime semantics follow tests/genetic_algorithm/device/slab_runtime_test.cu:572-690
(population from the fixed generation byte budget, grown action count, injected norms at the median norm).
"""
import numpy as np
import pytest

from oracle import pyoracle as O
from tests import gpu_util as G
from tests import helpers as H

pytestmark = pytest.mark.gpu
needs_ref = pytest.mark.skipif(O.ref_dev() is None, reason="reference device library not built")


def _catalog(rng, count):
    """Distinct synthetic words that all have a hint-grid group (monochrome words have none)."""
    while True:
        words = H.synthetic_words(rng, count)
        if all(O.hint_grid_group(w) is not None for w in words):
            return words


def _upload(catalog):
    G.nwg.capi.upload_catalog(catalog)
    if O.ref_dev() is not None:
        flat = np.ascontiguousarray(catalog, np.uint8)
        assert O.ref_dev().refdev_upload_catalog(flat.ctypes.data_as(O._u8p), len(catalog)) == 1


@needs_ref
@pytest.mark.parametrize("parent,count", [(40, 3), (97, 9), (300, 130)])
def test_oracle_injection_matches_reference_device_code(parent, count):
    t = G.torch()
    rng = np.random.default_rng(parent * 7 + count)
    catalog = _catalog(rng, parent + count)
    _upload(catalog)
    genomes = [H.random_genome(rng, parent + count) for _ in range(3)]
    stride = G.nwg.capi.genome_stride_bytes(parent + count)
    pitch = ((stride + 255) // 256) * 256
    host = np.zeros((3, pitch), np.uint8)
    for i, g in enumerate(genomes):
        host[i, :g.nbytes] = g.view(np.uint8)
    dev = G.dev(host.reshape(-1))
    status = t.zeros(3, dtype=t.int32, device="cuda")
    assert O.ref_dev().refdev_inject(dev.data_ptr(), pitch, 3, parent, parent, count, status.data_ptr(),
                                     G.stream_handle()) == 1
    t.cuda.synchronize()
    assert status.cpu().numpy().tolist() == [0, 0, 0]
    out = dev.cpu().numpy().reshape(3, pitch)
    for i, g in enumerate(genomes):
        st, grown = O.inject_tails(g, parent, catalog, parent, count)
        assert st == 0
        assert np.array_equal(out[i, :stride], grown.view(np.uint8)[:stride]), f"genome {i}"


def _grown_runtime(action_count, injected, population, columns, seed, generations=0):
    rng = np.random.default_rng(seed)
    catalog = _catalog(rng, action_count + injected)
    _upload(catalog)
    rt = G.nwg.Runtime(action_count, population, columns)
    rt.bootstrap(population, seed=seed)
    sizes = [6] * population
    lists = [rng.choice(action_count, size=s, replace=False).astype(np.uint32) for s in sizes]
    offsets = np.zeros(population + 1, np.uint32)
    offsets[1:] = np.cumsum(sizes)
    rt.set_cell_words(offsets, np.concatenate(lists))
    counts = G.nwg.capi.word_counts(training=action_count, action_space=action_count)
    cfg = G.nwg.capi.assembly_config(radius=1, p=0.05, sigma=0.02)
    for g in range(generations):
        rt.advance(seed=100 + g, counts=counts, config=cfg)
    return rt, catalog, counts, cfg


@needs_ref
@pytest.mark.parametrize("action_count,injected,population,columns,generations", [
    (96, 5, 12, 4, 0), (500, 40, 16, 4, 1), (1024, 512, 8, 4, 0)])
def test_growth_children_match_reference(action_count, injected, population, columns, generations):
    t = G.torch()
    rt, catalog, counts, cfg = _grown_runtime(action_count, injected, population, columns, action_count + injected,
                                              generations)
    parents = rt.current_generation()
    old_stride = G.nwg.capi.genome_stride_bytes(action_count)
    parent_host = np.stack([rt.download_slot(int(s)) for s in parents["slots"]])
    gen_index = int(rt.info().current_generation_index)
    seed = 4242
    pending = G.nwg.capi.PendingInjection(True, action_count, injected)
    rt.advance(seed=seed, counts=counts, config=cfg, pending=pending)
    assert rt.action_count == action_count + injected
    plan = rt.assembly_plan()
    children = rt.current_generation()
    n_children = len(children["slots"])
    assert len(plan) == n_children
    new_stride = G.nwg.capi.genome_stride_bytes(action_count + injected)
    new_pitch = ((new_stride + 255) // 256) * 256
    ours = np.stack([rt.download_slot(int(s)) for s in children["slots"]])
    assert ours.shape[1] == new_stride
    # reference: BreedAndMutateGenome with the parents' action count into the wider slots, then injection
    parent_dev = G.dev(parent_host.reshape(-1))
    ref = G.slab_tensor(n_children, new_pitch)
    pairs = G.dev(plan.astype(np.uint32).reshape(-1))
    b, m = cfg.breeding, cfg.mutation
    assert O.ref_dev().refdev_breed(parent_dev.data_ptr(), old_stride, ref.data_ptr(), new_pitch, pairs.data_ptr(),
                                    n_children, action_count, seed, gen_index, b.crossover_temperature_level1,
                                    b.crossover_temperature_level2, b.crossover_temperature_level3,
                                    m.mutation_probability, m.mutation_sigma,
                                    m.output_tail_row_scale_mutation_probability, G.stream_handle()) == 1
    status = t.zeros(n_children, dtype=t.int32, device="cuda")
    assert O.ref_dev().refdev_inject(ref.data_ptr(), new_pitch, n_children, action_count, action_count, injected,
                                     status.data_ptr(), G.stream_handle()) == 1
    t.cuda.synchronize()
    assert (status.cpu().numpy() == 0).all()
    r = ref.cpu().numpy().reshape(n_children, new_pitch)[:, :new_stride]
    for c in range(n_children):
        assert np.array_equal(ours[c], r[c]), f"child {c} differs"
    # the grown generation (fewer cells when the budget shrank it) evaluates over the wider action space
    rng = np.random.default_rng(1)
    lists = [rng.choice(action_count, size=6, replace=False).astype(np.uint32) for _ in range(n_children)]
    rt.set_cell_words(np.arange(n_children + 1, dtype=np.uint32) * 6, np.concatenate(lists))
    grown = G.nwg.capi.word_counts(training=action_count, action_space=action_count + injected)
    rt.evaluate(grown)
    s = rt.summary()
    assert s.action_count == action_count + injected and s.population_size == n_children
    assert rt.status() == 0
    rt.close()


def test_growth_sizes_population_from_the_byte_budget_and_scales_rows_to_the_median():
    action_count, injected, population, columns = 60, 3, 18, 9
    rt, catalog, counts, cfg = _grown_runtime(action_count, injected, population, columns, 11)
    budget = population * G.nwg.capi.genome_stride_bytes(action_count)
    new_stride = G.nwg.capi.genome_stride_bytes(action_count + injected)
    expected = min(population, (min(budget // new_stride, population) // columns) * columns)
    assert expected < population  # the fixed budget drops one row at the wider stride
    rt.advance(seed=5, counts=counts, config=cfg,
               pending=G.nwg.capi.PendingInjection(True, action_count, injected))
    gen = rt.current_generation()
    assert len(gen["slots"]) == expected
    assert rt.info().action_count == action_count + injected
    for s in gen["slots"]:
        image = rt.download_slot(int(s)).view(np.uint16)
        target = O.median_tail_norm(image, action_count)
        rows = image[O.genome_halfs(action_count):].view(np.float16).astype(np.float64).reshape(injected, 38)
        norms = np.sqrt((rows ** 2).sum(1))
        assert np.all(norms > 0)
        np.testing.assert_allclose(norms, target, rtol=2e-3)
    rt.close()


def test_growth_rejects_bad_injections():
    action_count, population, columns = 40, 8, 4
    rt, catalog, counts, cfg = _grown_runtime(action_count, 4, population, columns, 13)
    with pytest.raises(G.nwg.capi.NwgError) as e:
        rt.advance(seed=1, counts=counts, config=cfg, pending=G.nwg.capi.PendingInjection(True, action_count + 1, 2))
    assert e.value.status == 10  # must start at the current action count (invalid assembly config)
    with pytest.raises(G.nwg.capi.NwgError) as e:
        rt.advance(seed=1, counts=counts, config=cfg, pending=G.nwg.capi.PendingInjection(True, action_count, 9))
    assert e.value.status == 15  # beyond the catalog
    rt.close()
