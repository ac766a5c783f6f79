"""Checkpoint capture, restore and resume on the B200, against the reference's own runtime.

Reference: TryCreatePrebreedingCheckpointOnDevice, TryRestorePrebreedingCheckpointToDevice and
TryResumeGenerationFromCheckpointOnDevice (genetic_algorithm/device/slab_runtime.cu:1707-1880), and the reference's
test of them (tests/genetic_algorithm/device/slab_runtime_test.cu:805-898: 20 actions, 18 slots, a generation of 9
at index 4, three injected words). The reference's runtime itself runs here (oracle/_ref/libref_ckpt.so) on the
same catalog, configuration and seeds. The two checkpoints agree field by field, slot numbers aside (the
reference's come from its free list). The children a resume assembles agree byte for byte for every pairing of
writer (ours, the reference's) and resumer (ours, the reference's), and equal the uninterrupted advance.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import pyoracle as O
from tests import gpu_util as G
from tests import helpers as H

pytestmark = pytest.mark.gpu
capi = G.nwg.capi
needs_ref = pytest.mark.skipif(O.ref_ckpt() is None, reason="reference checkpoint library not built")
RELEASED = 0xFFFFFFFF


def _catalog(rng, count):
    """Distinct synthetic words that all have a hint-grid group."""
    while True:
        words = H.synthetic_words(rng, count)
        if all(O.hint_grid_group(w) is not None for w in words):
            return words


def _children(rt):
    gen = rt.current_generation()
    return gen, np.stack([rt.download_slot(int(s)) for s in gen["slots"]])


def _reference_resume(path, catalog):
    size = 64 * capi.genome_stride_bytes(int(catalog.shape[0]))
    out = np.zeros(size, np.uint8)
    count, stride = C.c_size_t(), C.c_size_t()
    ok = O.ref_ckpt().refckpt_runtime_resume(str(path).encode(), catalog.ctypes.data, len(catalog), out.ctypes.data,
                                             size, C.byref(count), C.byref(stride))
    assert ok == 1
    return out[:count.value * stride.value].reshape(count.value, stride.value)


CASES = {
    # the reference's own checkpoint test: zero temperatures and mutation, three injected words
    "reference_test": dict(actions=20, injected=3, slots=18, population=9, columns=3, boot_seed=173, boot_index=4,
                           seed=29, cfg=dict(radius=2, l1=0.0, l2=0.0, l3=0.0, p=0.0, sigma=0.0)),
    "no_injection": dict(actions=60, injected=0, slots=32, population=16, columns=4, boot_seed=7, boot_index=0,
                         seed=1234, cfg=dict(radius=1, p=0.05, sigma=0.02, row_scale=0.1)),
    "injection_mutating": dict(actions=40, injected=5, slots=24, population=12, columns=4, boot_seed=99,
                               boot_index=2, seed=77, cfg=dict(radius=1, p=0.01, sigma=0.03)),
}


@needs_ref
@pytest.mark.parametrize("name", list(CASES))
def test_checkpoint_matches_reference_and_every_resume_agrees(tmp_path, name):
    k = CASES[name]
    a, n_inj, pop, cols = k["actions"], k["injected"], k["population"], k["columns"]
    rng = np.random.default_rng(len(name))
    catalog = _catalog(rng, a + n_inj)
    G.upload_catalog_everywhere(catalog)
    counts = capi.word_counts(training=a, action_space=a)
    cfg = capi.assembly_config(**k["cfg"])
    pending = capi.PendingInjection(n_inj > 0, a if n_inj else 0, n_inj)

    # ours: capture at the boundary, write
    rt = G.nwg.Runtime(a, pop, cols, slab_generations=k["slots"] / pop)
    rt.bootstrap(pop, seed=k["boot_seed"], generation_index=k["boot_index"])
    ck = rt.checkpoint(k["seed"], counts, config=cfg, pending=pending, catalog=catalog)
    ours_path, ref_path = tmp_path / "ours.bin", tmp_path / "ref.bin"
    ck.write(ours_path)

    # the reference's runtime on the same inputs
    stride = capi.genome_stride_bytes(a)
    rc = capi.RuntimeConfig()
    rc.genotype_slab_byte_budget_bytes = k["slots"] * stride
    rc.generation_byte_budget_bytes = pop * stride
    rc.action_count, rc.population_size_ceiling, rc.grid_column_count = a, pop, cols
    assert O.ref_ckpt().refckpt_runtime_capture(C.addressof(rc), catalog.ctypes.data, len(catalog), pop,
                                                k["boot_seed"], k["boot_index"], k["seed"], C.addressof(counts),
                                                C.addressof(cfg),
                                                C.addressof(pending), None, 1, str(ref_path).encode()) == 1
    ref = capi.Checkpoint.read(ref_path)

    # field by field (the reference's slot numbers come from its free list; released parents coincide)
    r, o = ref.record, ck.record
    for field in ("schema_version", "genome_layout_version", "resume_phase", "training_data_identity_hash",
                  "generation_seed", "generation_index"):
        assert getattr(r, field) == getattr(o, field), field
    for field in ("runtime_word_counts", "training_shard_release_history", "assembly_config",
                  "pending_output_embedding_injection", "runtime_config", "slab_layout", "current_grid_shape",
                  "next_grid_shape", "epicenter_grid_shape"):
        assert bytes(getattr(r, field)) == bytes(getattr(o, field)), field
    assert np.array_equal(ref.fitness.view(np.uint32), ck.fitness.view(np.uint32))
    assert np.array_equal(ref.evaluation_counts, ck.evaluation_counts)
    assert np.array_equal(ref.has_fitness, ck.has_fitness)
    assert np.array_equal(ref.parent_pairs, ck.parent_pairs)
    assert np.array_equal(ref.slot_indices == RELEASED, ck.slot_indices == RELEASED)
    assert np.array_equal(ref.live_organisms, ck.live_organisms)
    assert np.array_equal(ref.live_genomes, ck.live_genomes)
    # the reference test's expectations
    assert o.generation_index == k["boot_index"] and len(ck.slot_indices) == pop
    assert 0 < len(ck.live_organisms) <= pop and o.training_data_identity_hash != 0
    if name == "reference_test":
        assert len(ck.parent_pairs) == 6

    # every resume: uninterrupted, ours from either file, the reference's from either file
    rt.assemble()
    gen, uninterrupted = _children(rt)
    assert gen["generation_index"] == k["boot_index"] + 1 and len(gen["slots"]) == len(ck.parent_pairs)
    for path in (ours_path, ref_path):
        restored = capi.Checkpoint.read(path).restore()
        if (ck.slot_indices == RELEASED).any():  # a boundary with released parents is not evaluable
            with pytest.raises(capi.NwgError) as e:
                restored.evaluate(counts)
            assert e.value.status == 4
        restored.resume()
        g2, resumed = _children(restored)
        assert g2["generation_index"] == gen["generation_index"]
        assert np.array_equal(resumed, uninterrupted), f"ours from {path.name}"
        restored.evaluate(capi.word_counts(training=a, action_space=a + n_inj))
        assert restored.current_generation()["has_fitness"].all()
        restored.close()
        assert np.array_equal(_reference_resume(path, catalog), uninterrupted), f"reference from {path.name}"
    rt.close()


def test_restore_rejects_bad_checkpoints(tmp_path):
    rng = np.random.default_rng(5)
    catalog = _catalog(rng, 30)
    G.upload_catalog_everywhere(catalog)
    rt = G.nwg.Runtime(30, 8, 4)
    rt.bootstrap(8, seed=3)
    ck = rt.checkpoint(11, capi.word_counts(training=30, action_space=30), config=capi.assembly_config(radius=1))
    rt.close()
    for edit in (lambda c: setattr(c.record, "resume_phase", 2),
                 lambda c: setattr(c.record.slab_layout, "slot_count", c.record.slab_layout.slot_count + 1),
                 lambda c: c.parent_pairs.__setitem__((0, 0), 99),
                 lambda c: c.slot_indices.__setitem__(int(c.live_organisms[0]), RELEASED),
                 lambda c: setattr(c.record.pending_output_embedding_injection, "enabled", True)):
        bad = capi.Checkpoint(capi.CheckpointRecord.from_buffer_copy(ck.record), ck.slot_indices.copy(),
                              ck.fitness, ck.evaluation_counts, ck.has_fitness, ck.parent_pairs.copy(),
                              ck.live_organisms, ck.live_genomes)
        edit(bad)
        bad.seal()
        with pytest.raises(capi.NwgError) as e:
            bad.restore()
        assert e.value.status == 19
    stale = capi.Checkpoint(capi.CheckpointRecord.from_buffer_copy(ck.record), ck.slot_indices, ck.fitness.copy(),
                            ck.evaluation_counts, ck.has_fitness, ck.parent_pairs, ck.live_organisms, ck.live_genomes)
    stale.fitness[0] += 1.0
    with pytest.raises(capi.NwgError) as e:
        stale.restore()
    assert e.value.status == 19
    good = ck.restore()
    good.resume()
    with pytest.raises(capi.NwgError) as e:  # nothing prepared any more
        good.resume()
    assert e.value.status == 12
    good.close()


def test_persist_winner_writes_the_best_individual(tmp_path):
    """TryPersistWinningGenome (cli/run_genetic_algorithm.cu:1519-1532): the summary's best slot image and metadata."""
    rng = np.random.default_rng(8)
    catalog = _catalog(rng, 200)
    G.upload_catalog_everywhere(catalog)
    rt = G.nwg.Runtime(200, 8, 4)
    rt.bootstrap(8, seed=21, generation_index=5)
    rt.evaluate(capi.word_counts(training=50, action_space=200))
    s = rt.summary()
    b, j = tmp_path / "win.bin", tmp_path / "win.json"
    rt.persist_winner(b, j, seed=77, catalog=catalog, action_space_path="words.txt")
    got = capi.read_winner_artifact(b, j)
    m = got["metadata"]
    assert np.array_equal(got["genome"], rt.download_slot(s.best_slot_index))
    assert (m.generation_index, m.best_index, m.best_slot_index, m.action_count, m.seed) == (
        5, s.best_index, s.best_slot_index, 200, 77)
    assert abs(m.best_fitness - s.best_fitness) <= 1e-6 and np.array_equal(got["words"], catalog)
    if O.ref_ckpt() is not None:
        meta = np.zeros(7, np.uint64)
        genome = np.zeros(m.genome_byte_count, np.uint8)
        letters = np.zeros((capi.CATALOG_CAPACITY, 5), np.uint8)
        count = C.c_size_t()
        path = C.create_string_buffer(256)
        assert O.ref_ckpt().refart_read(str(b).encode(), str(j).encode(), meta.ctypes.data, genome.ctypes.data,
                                        genome.nbytes, letters.ctypes.data, C.byref(count), path, len(path)) == 1
        assert np.array_equal(genome, got["genome"]) and count.value == 200
    rt.close()
