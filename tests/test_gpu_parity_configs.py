"""The benchmark workloads themselves against the reference's own device code, bit for bit.

Reference side: oracle/_ref/libref_dev.so, whose refdev_evaluate_csr runs the reference's
SelectNextGuessFromDynamicGenomeConcurrently, TryAppendGuess and ScoreCompletedEpisode warp per episode
(slab_runtime.cu:452-549) over explicit per-individual word lists (only the word lookup of
evaluation_ops.cuh:203-237 is restated), and refdev_select / refdev_breed / refdev_bootstrap, the reference's
TrySelectCellularParentPairDevice, BreedAndMutateGenome and InitializeRandomGenome.

- The small configuration in full: 64 individuals on an 8x8 grid, 512 active words, 64 secrets per cell from a
  256-word subset, all 192 episodes of every individual, then one generation (radius-1 rank selection, exponent
  0.5, mutation p = 0.05, sigma = 0.02). Genomes from the reference's bootstrap (seed 0) or drawn from
  N(0, 0.05) under seed 0 and stored in FP16.
- A sample of the full configuration: 16 evolved individuals of the 4,096-individual, 4,739-word population
  with their own 256-secret cell lists (768 games each).

Bar: identical guesses, turn counts and episode scores, policy vectors equal to the last bit (tighter than the
1e-5 relative tolerance the path is specified with), fitness bits, parent pairs and child images.
"""
import numpy as np
import pytest

from oracle import pyoracle as O
from tests import gpu_util as G

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(O.ref_dev() is None, reason="reference device library not built")]
REL_TOL = 1e-5
PLANNING_SEED_MIX = 0xA341316C  # slab_runtime.cu:1443


def _trace_ours(rt, counts, episodes, policy=True):
    t = G.torch()
    p = len(rt.current_generation()["slots"])
    choices = t.full((p, episodes, 6), -1, dtype=t.int32, device="cuda")
    turns = t.zeros((p, episodes), dtype=t.int32, device="cuda")
    scores = t.zeros((p, episodes), dtype=t.float32, device="cuda")
    pol = t.zeros((p, episodes, 6, 64), dtype=t.float32, device="cuda") if policy else None
    rt.evaluate_traced(counts, episodes, choices.data_ptr(), turns.data_ptr(), scores.data_ptr(),
                       pol.data_ptr() if policy else 0)
    t.cuda.synchronize()
    return (choices.cpu().numpy(), turns.cpu().numpy(), scores.cpu().numpy(),
            pol.cpu().numpy() if policy else None)


def _trace_reference(slab_ptr, pitch, slots, offsets, words, action_count, episodes):
    t = G.torch()
    p = len(slots)
    choices = t.full((p, episodes, 6), -1, dtype=t.int32, device="cuda")
    turns = t.zeros((p, episodes), dtype=t.int32, device="cuda")
    scores = t.zeros((p, episodes), dtype=t.float32, device="cuda")
    pol = t.zeros((p, episodes, 6, 64), dtype=t.float32, device="cuda")
    status = t.zeros(1, dtype=t.int32, device="cuda")
    d_slots = G.dev(np.asarray(slots, np.uint32))
    d_off = G.dev(np.asarray(offsets, np.uint32))
    d_words = G.dev(np.asarray(words, np.uint32))
    assert O.ref_dev().refdev_evaluate_csr(slab_ptr, pitch, d_slots.data_ptr(), p, action_count, d_off.data_ptr(),
                                           d_words.data_ptr(), episodes, scores.data_ptr(), turns.data_ptr(),
                                           choices.data_ptr(), pol.data_ptr(), status.data_ptr(),
                                           G.stream_handle()) == 1
    t.cuda.synchronize()
    assert int(status.item()) == 0
    return choices.cpu().numpy(), turns.cpu().numpy(), scores.cpu().numpy(), pol.cpu().numpy()


def _assert_same_games(ours, ref, label):
    oc, ot, os_, op = ours
    rc, rt_, rs, rp = ref
    assert np.array_equal(oc, rc), f"{label}: guesses differ"
    assert np.array_equal(ot, rt_), f"{label}: turn counts differ"
    assert np.array_equal(os_, rs), f"{label}: episode scores differ"
    decided = rc >= 0
    assert np.all(op[decided] == rp[decided]), f"{label}: policy vectors differ"
    assert np.all(np.abs(op[decided] - rp[decided]) <= REL_TOL * np.maximum(1.0, np.abs(rp[decided])))


def _reference_fitness(scores, words_per_cell):
    raw = scores.astype(np.float64).sum(axis=1)  # integers below 2^24: every order sums exactly
    return np.array([O.normalize_fitness(float(r), int(w)) for r, w in zip(raw, words_per_cell)], np.float32)


def _normal005_images(population, action_count, seed):
    rng = np.random.default_rng(seed)
    halfs = O.genome_halfs(action_count)
    return (rng.standard_normal((population, halfs)) * 0.05).astype(np.float16).view(np.uint16)


@pytest.mark.parametrize("init", ["bootstrap", "normal005"])
def test_small_configuration_generation_matches_reference(init):
    t = G.torch()
    wl = G.nwg.workload.SMALL
    assert (wl.population, wl.columns, wl.action_count, wl.secret_subset, wl.secrets_per_cell) == (64, 8, 512, 256,
                                                                                                  64)
    catalog = wl.catalog()
    offsets, words = wl.cell_lists()
    G.upload_catalog_everywhere(catalog)
    capi = G.nwg.capi
    stride = capi.genome_stride_bytes(wl.action_count)
    rt = G.nwg.Runtime(wl.action_count, wl.population, wl.columns)
    rt.bootstrap(wl.population, seed=0)
    slab, pitch = rt.device_slab()
    slots = rt.current_generation()["slots"]
    if init == "bootstrap":
        ref = G.slab_tensor(wl.population, pitch)
        assert O.ref_dev().refdev_bootstrap(ref.data_ptr(), pitch, wl.population, 0, 0, wl.action_count,
                                            G.stream_handle()) == 1
        t.cuda.synchronize()
        ref_images = ref.cpu().numpy().reshape(wl.population, pitch)[:, :stride]
        for i, s in enumerate(slots):
            assert np.array_equal(rt.download_slot(int(s)), ref_images[i]), f"bootstrap image {i}"
    else:
        for i, img in enumerate(_normal005_images(wl.population, wl.action_count, 0)):
            rt.upload_slot(int(slots[i]), img)
    rt.set_cell_words(offsets, words)
    counts = capi.word_counts(training=wl.action_count, action_space=wl.action_count)
    episodes = 3 * wl.secrets_per_cell
    ref = _trace_reference(slab, pitch, slots, offsets, words, wl.action_count, episodes)
    ref_fitness = _reference_fitness(ref[2], np.diff(offsets))
    for form in (capi.FORM_FP32, capi.FORM_TC_TRUNK_FP16):
        rt.set_form(form)
        if form != capi.FORM_FP32:
            rt.set_margin_guard(1.0e30)  # every step through the exact path
        _assert_same_games(_trace_ours(rt, counts, episodes), ref, f"{init}, form {form}")
        gen = rt.current_generation()
        assert np.array_equal(gen["fitness"].view(np.uint32), ref_fitness.view(np.uint32)), f"form {form}: fitness"

    # one generation: the reference's plan on the reference's fitness, the reference's children of those parents
    parents = np.zeros(wl.population * pitch, np.uint8)
    for i, s in enumerate(slots):
        parents[i * pitch:i * pitch + stride] = rt.download_slot(int(s))
    rt.set_form(capi.FORM_FP32)
    seed = 1000
    cfg = capi.assembly_config(radius=wl.radius, p=wl.mutation_probability, sigma=wl.mutation_sigma)
    rt.advance(seed=seed, counts=counts, config=cfg)
    plan = rt.assembly_plan()
    ref_pairs = t.zeros(2 * wl.population, dtype=t.int32, device="cuda")
    ok = t.zeros(wl.population, dtype=t.int32, device="cuda")
    assert O.ref_dev().refdev_select(G.dev(ref_fitness).data_ptr(), G.dev(np.ones(wl.population, np.uint8)).data_ptr(),
                                     wl.population, wl.population, wl.columns, 0, wl.radius, 0.5,
                                     seed ^ PLANNING_SEED_MIX, ref_pairs.data_ptr(), ok.data_ptr(),
                                     G.stream_handle()) == 1
    t.cuda.synchronize()
    assert bool(ok.all())
    assert np.array_equal(plan.astype(np.int64), ref_pairs.cpu().numpy().reshape(-1, 2).astype(np.int64))
    children = G.slab_tensor(wl.population, pitch)
    assert O.ref_dev().refdev_breed(G.dev(parents).data_ptr(), pitch, children.data_ptr(), pitch,
                                    G.dev(plan.astype(np.uint32).reshape(-1)).data_ptr(), wl.population,
                                    wl.action_count, seed, 0, 0.02, 0.01, 0.005, wl.mutation_probability,
                                    wl.mutation_sigma, 0.0, G.stream_handle()) == 1
    t.cuda.synchronize()
    ref_children = children.cpu().numpy().reshape(wl.population, pitch)[:, :stride]
    gen1 = rt.current_generation()
    assert gen1["generation_index"] == 1
    for c, s in enumerate(gen1["slots"]):
        assert np.array_equal(rt.download_slot(int(s)), ref_children[c]), f"child {c}"
    rt.close()


def test_full_configuration_sample_matches_reference():
    """16 individuals of the 4,096 x 4,739 population after two generations (FP16 trunk form, guard 1e-3) play
    their 768 games in the plain form and in the trunk form with the exact path forced, against the reference."""
    wl = G.nwg.workload.FULL
    catalog = wl.catalog()
    offsets, words = wl.cell_lists()
    G.upload_catalog_everywhere(catalog)
    capi = G.nwg.capi
    counts = capi.word_counts(training=wl.action_count, action_space=wl.action_count)
    cfg = capi.assembly_config(radius=wl.radius, p=wl.mutation_probability, sigma=wl.mutation_sigma)
    rt = G.nwg.Runtime(wl.action_count, wl.population, wl.columns)
    rt.set_cell_words(offsets, words)
    rt.set_form(capi.FORM_TC_TRUNK_FP16)
    rt.set_margin_guard(1e-3)
    rt.bootstrap(wl.population, seed=0)
    for g in range(2):
        rt.advance(seed=1000 + g, counts=counts, config=cfg)
    rt.set_form(capi.FORM_FP32)
    rt.evaluate(counts)
    full = rt.current_generation()
    rng = np.random.default_rng(4739)
    chosen = np.sort(rng.choice(wl.population, 16, replace=False))
    images = [rt.download_slot(int(full["slots"][i])) for i in chosen]
    rt.close()

    sub_off = np.zeros(17, np.uint32)
    sub_words = []
    for k, i in enumerate(chosen):
        sub_words.append(words[offsets[i]:offsets[i + 1]])
        sub_off[k + 1] = sub_off[k] + offsets[i + 1] - offsets[i]
    sub_words = np.concatenate(sub_words).astype(np.uint32)
    sample = G.nwg.Runtime(wl.action_count, 16, 4)
    sample.bootstrap(16, seed=1)
    slots = sample.current_generation()["slots"]
    for k, img in enumerate(images):
        sample.upload_slot(int(slots[k]), img)
    sample.set_cell_words(sub_off, sub_words)
    slab, pitch = sample.device_slab()
    episodes = 3 * wl.secrets_per_cell
    ref = _trace_reference(slab, pitch, slots, sub_off, sub_words, wl.action_count, episodes)
    ref_fitness = _reference_fitness(ref[2], np.diff(sub_off))
    # the full-population evaluation (plain form) gave these individuals the reference's fitness
    assert np.array_equal(full["fitness"][chosen].view(np.uint32), ref_fitness.view(np.uint32))
    for form in (capi.FORM_FP32, capi.FORM_TC_TRUNK_FP16):
        sample.set_form(form)
        if form != capi.FORM_FP32:
            sample.set_margin_guard(1.0e30)
        _assert_same_games(_trace_ours(sample, counts, episodes), ref, f"form {form}")
        gen = sample.current_generation()
        assert np.array_equal(gen["fitness"].view(np.uint32), ref_fitness.view(np.uint32)), f"form {form}: fitness"
    sample.close()
