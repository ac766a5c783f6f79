"""Runtime checkpoint files on the host (no GPU): the reference's byte format, checksum and identity hash.

Reference: RuntimeCheckpoint and its file (genetic_algorithm/device/slab_runtime.hpp:86-117,
slab_runtime.cu:1182-1248 checksum, :1283-1297 identity hash, :1934-2073 writer and reader). Checked against the
reference's own code compiled from its sources (oracle/_ref/libref_ckpt.so): a file written here re-writes byte
for byte through the reference's reader and writer (whose reader also checks the checksum), and a file the
reference writes, with non-zero padding in its padded records, reads here and re-writes byte for byte.
"""
import importlib

import numpy as np
import pytest

from oracle import pyoracle as O

nwg = importlib.import_module("neuroevolutionary-wordle_b200")
capi = nwg.capi
needs_ref = pytest.mark.skipif(O.ref_ckpt() is None, reason="reference checkpoint library not built")


def _synthetic(seed, individuals=12, children=8, action_count=7, releases=3, injection=False):
    """A checkpoint of seeded content built through the Python API (no runtime)."""
    rng = np.random.default_rng(seed)
    stride = capi.genome_stride_bytes(action_count)
    rec = capi.CheckpointRecord()
    rec.schema_version, rec.genome_layout_version, rec.resume_phase = 3, 1, 1
    rec.training_data_identity_hash = int(rng.integers(1, 2**63))
    rec.generation_seed = int(rng.integers(0, 2**32))
    rec.runtime_word_counts = capi.word_counts(training=action_count, action_space=action_count)
    h = rec.training_shard_release_history
    h.release_count = releases
    for i in range(releases):
        h.release_generations[i] = int(rng.integers(0, 1000))
        h.release_fitness_p99[i] = float(rng.random())
    rec.assembly_config = capi.assembly_config(radius=2, p=0.01, sigma=0.03)
    if injection:
        rec.pending_output_embedding_injection = capi.PendingInjection(True, action_count - 2, 2)
    rec.slab_layout.action_count = action_count
    rec.slab_layout.slot_stride_bytes = stride
    rec.slab_layout.slot_count = 2 * individuals
    rec.slab_layout.slab_bytes = 2 * individuals * stride
    rc = rec.runtime_config
    rc.genotype_slab_byte_budget_bytes = rec.slab_layout.slab_bytes
    rc.generation_byte_budget_bytes = individuals * stride
    rc.action_count = action_count
    rc.population_size_ceiling = individuals
    rc.grid_column_count = 4
    for shape, n in ((rec.current_grid_shape, individuals), (rec.next_grid_shape, children),
                     (rec.epicenter_grid_shape, individuals)):
        shape.row_count, shape.column_count, shape.cell_count = n // 4, 4, n
    rec.generation_index = int(rng.integers(0, 50))
    live = rng.random(individuals) < 0.75
    slots = np.where(live, np.arange(individuals), 0xFFFFFFFF).astype(np.uint32)
    organisms = np.flatnonzero(live).astype(np.uint32)
    live_index = organisms[rng.integers(0, len(organisms), size=2 * children)]
    ck = capi.Checkpoint(rec, slots, rng.random(individuals).astype(np.float32),
                         rng.integers(0, 40, individuals).astype(np.uint32),
                         rng.integers(0, 2, individuals).astype(np.uint8), live_index.reshape(-1, 2), organisms,
                         rng.integers(0, 256, (len(organisms), stride)).astype(np.uint8))
    ck.seal()
    return ck


def test_record_sizes_match_the_reference_lp64_layout():
    import ctypes as C

    assert C.sizeof(capi.AssemblyConfig) == 40
    assert C.sizeof(capi.PendingInjection) == 24
    assert C.sizeof(capi.RuntimeWordCounts) == 56
    assert C.sizeof(capi.RuntimeConfig) == 48
    assert C.sizeof(capi.SlabLayout) == 32
    assert C.sizeof(capi.GridShape) == 24
    if O.ref_ckpt() is not None:
        out = (C.c_size_t * 8)()
        O.ref_ckpt().refckpt_layouts(out)
        assert list(out) == [56, C.sizeof(capi.ShardReleaseHistory), 40, 24, 48, 32, 24, 5]


@pytest.mark.parametrize("seed,injection", [(1, False), (2, True), (3, False)])
def test_write_then_read_round_trips(tmp_path, seed, injection):
    ck = _synthetic(seed, injection=injection)
    path = tmp_path / "ck.bin"
    ck.write(path)
    back = capi.Checkpoint.read(path)
    assert back.record.checksum == ck.record.checksum == back.checksum()
    assert bytes(back.record)[:64] == bytes(ck.record)[:64]
    for name in ("slot_indices", "fitness", "evaluation_counts", "has_fitness", "parent_pairs", "live_organisms",
                 "live_genomes"):
        assert np.array_equal(getattr(back, name), getattr(ck, name)), name
    assert back.record.pending_output_embedding_injection.enabled == injection


@needs_ref
@pytest.mark.parametrize("seed,individuals,children,action_count,releases,injection", [
    (4, 12, 8, 7, 3, False), (5, 16, 16, 40, 0, True), (6, 8, 4, 1, 11, False)])
def test_reference_rewrites_our_file_byte_for_byte(tmp_path, seed, individuals, children, action_count, releases,
                                                    injection):
    ck = _synthetic(seed, individuals, children, action_count, releases, injection)
    ours, theirs = tmp_path / "ours.bin", tmp_path / "theirs.bin"
    ck.write(ours)
    assert O.ref_ckpt().refckpt_roundtrip(str(ours).encode(), str(theirs).encode()) == 1  # reader checks the sum
    assert ours.read_bytes() == theirs.read_bytes()


@needs_ref
@pytest.mark.parametrize("seed,individuals,children,action_count,releases,injection", [
    (7, 12, 8, 20, 2, 1), (8, 16, 12, 3, 0, 0), (9, 4, 4, 100, 5, 1)])
def test_we_rewrite_the_reference_file_byte_for_byte(tmp_path, seed, individuals, children, action_count, releases,
                                                     injection):
    theirs, ours = tmp_path / "theirs.bin", tmp_path / "ours.bin"
    assert O.ref_ckpt().refckpt_write_synthetic(str(theirs).encode(), seed, individuals, children, action_count,
                                                releases, injection) == 1
    ck = capi.Checkpoint.read(theirs)
    # the reference filled its padded records' padding with 0xA5; the bytes are carried as stored
    assert bytes(ck.record.assembly_config)[12:16] == b"\xa5" * 4
    assert ck.record.pending_output_embedding_injection.enabled == bool(injection)
    assert len(ck.slot_indices) == individuals and len(ck.parent_pairs) == children
    ck.write(ours)
    assert ours.read_bytes() == theirs.read_bytes()


def test_corruption_is_rejected(tmp_path):
    ck = _synthetic(10)
    path = tmp_path / "ck.bin"
    ck.write(path)
    data = bytearray(path.read_bytes())
    for offset in (0, 9, 40, len(data) // 2, len(data) - 1):
        bad = bytearray(data)
        bad[offset] ^= 0x01
        p = tmp_path / f"bad{offset}.bin"
        p.write_bytes(bytes(bad))
        with pytest.raises(capi.NwgError) as e:
            capi.Checkpoint.read(p)
        assert e.value.status == 19
        if O.ref_ckpt() is not None:
            assert O.ref_ckpt().refckpt_roundtrip(str(p).encode(), str(tmp_path / "x.bin").encode()) == 0
    truncated = tmp_path / "short.bin"
    truncated.write_bytes(bytes(data[:-5]))
    with pytest.raises(capi.NwgError):
        capi.Checkpoint.read(truncated)
    with pytest.raises(capi.NwgError):
        capi.Checkpoint.read(tmp_path / "missing.bin")


def test_stale_checksum_is_refused_on_write(tmp_path):
    ck = _synthetic(11)
    ck.fitness[0] += 1.0
    with pytest.raises(capi.NwgError) as e:
        ck.write(tmp_path / "ck.bin")
    assert e.value.status == 19
    assert not (tmp_path / "ck.bin").exists() and not (tmp_path / "ck.bin.tmp").exists()
    ck.seal()
    ck.write(tmp_path / "ck.bin")


def test_checksum_covers_every_field():
    ck = _synthetic(12, injection=True)
    base = ck.checksum()
    edits = [
        lambda c: setattr(c.record, "generation_seed", c.record.generation_seed ^ 1),
        lambda c: setattr(c.record, "training_data_identity_hash", c.record.training_data_identity_hash ^ 1),
        lambda c: setattr(c.record.runtime_word_counts, "shard_initial_radius", 3),
        lambda c: setattr(c.record.training_shard_release_history, "release_count", 2),
        lambda c: setattr(c.record.assembly_config.mutation, "mutation_sigma", 0.5),
        lambda c: setattr(c.record.pending_output_embedding_injection, "injection_count", 5),
        lambda c: setattr(c.record.runtime_config, "grid_column_count", 2),
        lambda c: setattr(c.record.slab_layout, "slot_count", 99),
        lambda c: setattr(c.record.next_grid_shape, "row_count", 9),
        lambda c: setattr(c.record, "generation_index", c.record.generation_index + 1),
        lambda c: c.evaluation_counts.__setitem__(3, c.evaluation_counts[3] + 1),
        lambda c: c.has_fitness.__setitem__(1, 1 - c.has_fitness[1]),
        lambda c: c.parent_pairs.__setitem__((0, 1), c.parent_pairs[0, 1] ^ 1),
        lambda c: c.live_genomes.__setitem__((0, -1), c.live_genomes[0, -1] ^ 1),
    ]
    for i, edit in enumerate(edits):
        c = _synthetic(12, injection=True)
        edit(c)
        assert c.checksum() != base, i


@needs_ref
@pytest.mark.parametrize("with_history,with_catalog", [(False, False), (True, False), (False, True), (True, True)])
def test_identity_hash_matches_reference(with_history, with_catalog):
    import ctypes as C

    rng = np.random.default_rng(13)
    counts = capi.word_counts(training=30, action_space=40, initial=20, step=5, period=3)
    history = None
    if with_history:
        history = capi.ShardReleaseHistory()
        history.release_count = 4
        for i in range(4):
            history.release_generations[i] = 10 * i
            history.release_fitness_p99[i] = 0.25 * i
    catalog = rng.integers(0, 26, (57, 5)).astype(np.uint8) if with_catalog else None
    ours = capi.identity_hash(counts, history, catalog)
    theirs = O.ref_ckpt().refckpt_identity_hash(C.addressof(counts), C.addressof(history) if history else None,
                                                catalog.ctypes.data if catalog is not None else None,
                                                0 if catalog is None else len(catalog))
    assert ours == theirs
