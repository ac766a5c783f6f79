"""Selection, breeding/mutation and bootstrap on the B200, bit for bit against the reference's device code.

Reference side: oracle/_ref/libref_dev.so (TrySelectCellularParentPairDevice, BreedAndMutateGenome,
InitializeRandomGenome compiled for sm_100a from the reference's headers). CPU side: the oracle's
restatement of the same control flow, fed by draw tapes recorded from the toolkit generator.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import pyoracle as O
from tests import gpu_util as G
from tests import helpers as H

pytestmark = pytest.mark.gpu
needs_ref = pytest.mark.skipif(O.ref_dev() is None, reason="reference device library not built")


def _fitness_with_ties(rng, n):
    return (rng.integers(0, 6, n) / 7.0).astype(np.float32)


@needs_ref
@pytest.mark.parametrize("rows,cols,next_rows,radius,exponent", [
    (8, 8, 8, 1, 0.5), (8, 8, 8, 2, 0.5), (6, 5, 4, 2, 1.3), (7, 7, 7, 3, 0.5), (2, 3, 2, 1, 0.0)])
def test_selection_matches_reference(rows, cols, next_rows, radius, exponent):
    t = G.torch()
    rng = np.random.default_rng(rows * 100 + radius)
    n = rows * cols
    children = next_rows * cols
    fitness = G.dev(_fitness_with_ties(rng, n))
    has = G.dev(np.ones(n, np.uint8))
    ours = t.zeros(2 * children, dtype=t.int32, device="cuda")
    ref = t.zeros(2 * children, dtype=t.int32, device="cuda")
    ok = t.zeros(children, dtype=t.int32, device="cuda")
    seed = 0x5EED ^ 0xA341316C
    for generation in (0, 3):
        cfg = G.nwg.capi.ParentSelectionConfig(radius, exponent)
        status = G.nwg.capi.lib().nwg_select_parents_device(fitness.data_ptr(), has.data_ptr(), n, cols, children,
                                                              generation, C.byref(cfg), seed, ours.data_ptr(),
                                                              G.stream_handle())
        assert status == 0
        assert O.ref_dev().refdev_select(fitness.data_ptr(), has.data_ptr(), n, children, cols, generation, radius,
                                         exponent, seed, ref.data_ptr(), ok.data_ptr(), G.stream_handle()) == 1
        t.cuda.synchronize()
        assert bool(ok.all())
        assert t.equal(ours, ref)
        pairs = ours.cpu().numpy().reshape(-1, 2)
        assert (pairs[:, 0] != pairs[:, 1]).all()


def test_selection_matches_cpu_oracle_with_recorded_draws():
    t = G.torch()
    rows, cols, radius, exponent, generation = 6, 6, 1, 0.5, 2
    rng = np.random.default_rng(3)
    n = rows * cols
    f_host = _fitness_with_ties(rng, n)
    fitness = G.dev(f_host)
    has = G.dev(np.ones(n, np.uint8))
    ours = t.zeros(2 * n, dtype=t.int32, device="cuda")
    seed = 1234
    cfg = G.nwg.capi.ParentSelectionConfig(radius, exponent)
    assert G.nwg.capi.lib().nwg_select_parents_device(fitness.data_ptr(), has.data_ptr(), n, cols, n, generation,
                                                        C.byref(cfg), seed, ours.data_ptr(), G.stream_handle()) == 0
    draws = t.zeros(6 * n, dtype=t.int32, device="cuda")
    weights = t.zeros(32, dtype=t.float32, device="cuda")
    assert O.tape_lib().tape_selection_draws(seed, generation, n, draws.data_ptr()) == 1
    assert O.tape_lib().tape_pow_table(exponent, 32, weights.data_ptr()) == 1
    d = draws.cpu().numpy().view(np.uint32).reshape(n, 6)
    w = weights.cpu().numpy()
    got = ours.cpu().numpy().reshape(-1, 2)
    for c in range(n):
        pair = O.select_parent_pair(f_host, np.ones(n, np.uint8), rows, cols, rows, c, radius, d[c], w)
        assert pair == tuple(got[c])


BREED_CASES = {
    "defaults": dict(l1=0.02, l2=0.01, l3=0.005, p=1e-4, sigma=0.02, row_scale=0.0),
    "baseline_rate": dict(l1=0.02, l2=0.01, l3=0.005, p=0.05, sigma=0.02, row_scale=0.0),
    "all_flips": dict(l1=1.0, l2=1.0, l3=1.0, p=0.3, sigma=0.5, row_scale=0.0),
    "half_flips": dict(l1=0.5, l2=0.5, l3=0.5, p=0.01, sigma=0.1, row_scale=0.5),
    "every_value": dict(l1=0.0, l2=0.0, l3=0.0, p=1.0, sigma=0.02, row_scale=0.0),
    "no_sigma": dict(l1=0.3, l2=0.3, l3=0.3, p=0.2, sigma=0.0, row_scale=1.0),
    "no_mutation": dict(l1=0.1, l2=0.1, l3=1.0, p=0.0, sigma=0.02, row_scale=0.0),
    # the window-parallel walk at its extremes: almost every position a hit (fresh pairs straddling nearly every
    # window edge), and hits so rare that most 4,096-position steps have none
    "dense_hits": dict(l1=0.02, l2=0.01, l3=0.005, p=0.9, sigma=0.02, row_scale=0.0),
    "sparse_hits": dict(l1=0.02, l2=0.01, l3=0.005, p=2e-6, sigma=0.02, row_scale=0.0),
}


def _parents(rng, count, action_count, pitch):
    slab = np.zeros(count * pitch, np.uint8)
    for i in range(count):
        g = H.random_genome(rng, action_count)
        slab[i * pitch:i * pitch + g.nbytes] = g.view(np.uint8)
    return slab


@needs_ref
@pytest.mark.parametrize("case", sorted(BREED_CASES))
@pytest.mark.parametrize("action_count", [37, 512])
def test_breeding_matches_reference(case, action_count):
    t = G.torch()
    cfg = BREED_CASES[case]
    rng = np.random.default_rng(len(case) * 1000 + action_count)
    parents = 6
    children = 12
    stride = G.nwg.capi.genome_stride_bytes(action_count)
    pitch = ((stride + 255) // 256) * 256
    parent_slab = G.dev(_parents(rng, parents, action_count, pitch))
    slots = G.dev(np.arange(parents, dtype=np.uint32))
    pairs_host = np.stack([rng.integers(0, parents, children), rng.integers(0, parents, children)], 1)
    pairs_host[:, 1] = np.where(pairs_host[:, 0] == pairs_host[:, 1], (pairs_host[:, 1] + 1) % parents,
                                pairs_host[:, 1])
    pairs = G.dev(pairs_host.astype(np.uint32).reshape(-1))
    ours = G.slab_tensor(children, pitch)
    ref = G.slab_tensor(children, pitch)
    seed, generation = 987654321, 5
    b = G.nwg.capi.BreedingConfig(cfg["l1"], cfg["l2"], cfg["l3"])
    m = G.nwg.capi.MutationConfig(cfg["p"], cfg["sigma"], cfg["row_scale"])
    assert G.nwg.capi.lib().nwg_breed_device(parent_slab.data_ptr(), pitch, slots.data_ptr(), ours.data_ptr(), pitch,
                                               pairs.data_ptr(), children, action_count, seed, generation, C.byref(b),
                                               C.byref(m), G.stream_handle()) == 0
    assert O.ref_dev().refdev_breed(parent_slab.data_ptr(), pitch, ref.data_ptr(), pitch, pairs.data_ptr(), children,
                                    action_count, seed, generation, cfg["l1"], cfg["l2"], cfg["l3"], cfg["p"],
                                    cfg["sigma"], cfg["row_scale"], G.stream_handle()) == 1
    t.cuda.synchronize()
    a = ours.cpu().numpy().reshape(children, pitch)[:, :stride]
    r = ref.cpu().numpy().reshape(children, pitch)[:, :stride]
    for c in range(children):
        assert np.array_equal(a[c], r[c]), f"child {c} differs ({case})"


@pytest.mark.parametrize("case", ["baseline_rate", "all_flips", "half_flips", "every_value", "no_sigma"])
def test_breeding_matches_cpu_oracle_with_recorded_draws(case):
    t = G.torch()
    cfg = BREED_CASES[case]
    action_count = 24
    rng = np.random.default_rng(17)
    stride = G.nwg.capi.genome_stride_bytes(action_count)
    pitch = ((stride + 255) // 256) * 256
    host = _parents(rng, 2, action_count, pitch)
    parent_slab = G.dev(host)
    slots = G.dev(np.arange(2, dtype=np.uint32))
    pairs = G.dev(np.array([0, 1, 1, 0], np.uint32))
    ours = G.slab_tensor(2, pitch)
    seed, generation = 31337, 2
    b = G.nwg.capi.BreedingConfig(cfg["l1"], cfg["l2"], cfg["l3"])
    m = G.nwg.capi.MutationConfig(cfg["p"], cfg["sigma"], cfg["row_scale"])
    assert G.nwg.capi.lib().nwg_breed_device(parent_slab.data_ptr(), pitch, slots.data_ptr(), ours.data_ptr(), pitch,
                                               pairs.data_ptr(), 2, action_count, seed, generation, C.byref(b),
                                               C.byref(m), G.stream_handle()) == 0
    t.cuda.synchronize()
    out = ours.cpu().numpy().reshape(2, pitch)[:, :stride]
    length = 400000
    raw = t.zeros(length, dtype=t.int32, device="cuda")
    uni = t.zeros(length, dtype=t.float32, device="cuda")
    nrm = t.zeros(2 * length, dtype=t.float32, device="cuda")
    p0 = host[:stride].view(np.uint16)
    p1 = host[pitch:pitch + stride].view(np.uint16)
    O.set_fma_mode(True)
    for child, (first, second) in enumerate([(p0, p1), (p1, p0)]):
        subsequence = (child + generation * 4099) & 0xFFFFFFFF
        assert O.tape_lib().tape_positions(seed, subsequence, length, raw.data_ptr(), uni.data_ptr(),
                                           nrm.data_ptr()) == 1
        tape = dict(raw=raw.cpu().numpy().view(np.uint32), uniform=uni.cpu().numpy(), normal_pair=nrm.cpu().numpy())
        expected = O.breed_and_mutate(first, second, action_count, tape, cfg)
        assert expected is not None
        assert np.array_equal(out[child].view(np.uint16), expected), f"child {child} ({case})"


@needs_ref
@pytest.mark.parametrize("action_count,population,generation", [(100, 3, 0), (4739, 2, 4)])
def test_bootstrap_matches_reference(action_count, population, generation):
    t = G.torch()
    stride = G.nwg.capi.genome_stride_bytes(action_count)
    pitch = ((stride + 255) // 256) * 256
    ours = G.slab_tensor(population, pitch)
    ref = G.slab_tensor(population, pitch)
    seed = 2024
    assert G.nwg.capi.lib().nwg_bootstrap_device(ours.data_ptr(), pitch, population, generation, seed, action_count,
                                                   G.stream_handle()) == 0
    assert O.ref_dev().refdev_bootstrap(ref.data_ptr(), pitch, population, generation, seed, action_count,
                                        G.stream_handle()) == 1
    t.cuda.synchronize()
    assert t.equal(ours, ref)


def test_bootstrap_matches_cpu_oracle_with_recorded_normals():
    t = G.torch()
    action_count, population, generation, seed = 50, 2, 1, 77
    stride = G.nwg.capi.genome_stride_bytes(action_count)
    pitch = ((stride + 255) // 256) * 256
    ours = G.slab_tensor(population, pitch)
    assert G.nwg.capi.lib().nwg_bootstrap_device(ours.data_ptr(), pitch, population, generation, seed, action_count,
                                                   G.stream_handle()) == 0
    t.cuda.synchronize()
    per = O.bootstrap_normals_per_thread(action_count)
    normals = t.zeros(256 * per, dtype=t.float32, device="cuda")
    host = ours.cpu().numpy()
    for organism in range(population):
        first = (generation * population + organism) * 256
        assert O.tape_lib().tape_normal_streams(seed, first, 256, per, normals.data_ptr()) == 1
        expected = O.bootstrap_genome(action_count, normals.cpu().numpy(), per)
        got = host[organism * pitch:organism * pitch + stride].view(np.uint16)
        assert np.array_equal(got, expected)
