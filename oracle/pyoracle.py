"""ctypes front end for the oracle libraries (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference legs use
this module. It loads
  _lib/libnwg_oracle.so  (CPU restatement),
  _lib/libnwg_tape.so    (GPU draw tapes),
  _ref/libref_host.so    (reference host code, CPU),
  _ref/libref_dev.so     (reference device code, GPU).
"""
from __future__ import annotations

import ctypes as C
from functools import lru_cache
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
POLICY_HALFS = 150528
TAIL_DIM = 38

_u8p = C.POINTER(C.c_uint8)
_u16p = C.POINTER(C.c_uint16)
_u32p = C.POINTER(C.c_uint32)
_i32p = C.POINTER(C.c_int32)
_f32p = C.POINTER(C.c_float)
_u64p = C.POINTER(C.c_uint64)
_sz = C.c_size_t


def _ptr(a: np.ndarray | None, t):
    if a is None:
        return C.cast(None, t)
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(t)


def genome_halfs(action_count: int) -> int:
    return POLICY_HALFS + TAIL_DIM * action_count


def stride_bytes(action_count: int) -> int:
    return 2 * genome_halfs(action_count) if action_count else 0


class ShardRecord(C.Structure):
    """TrainingDataShardRuntime (training_folder/training_data.hpp:35-42), 48 bytes."""

    _fields_ = [
        ("first_catalog_word_index", C.c_uint64),
        ("word_count", C.c_uint64),
        ("center_row", C.c_uint64),
        ("center_column", C.c_uint64),
        ("radius", C.c_uint64),
        ("global_from_outset", C.c_uint8),
    ]


assert C.sizeof(ShardRecord) == 48


class DrawTape(C.Structure):
    _fields_ = [
        ("raw", _u32p),
        ("uniform", _f32p),
        ("normal_pair", _f32p),
        ("length", _sz),
        ("position", _sz),
        ("has_cached_normal", C.c_int),
        ("cached_normal", C.c_float),
        ("overflow", C.c_int),
    ]


class BreedConfig(C.Structure):
    _fields_ = [
        ("crossover_l1", C.c_float),
        ("crossover_l2", C.c_float),
        ("crossover_l3", C.c_float),
        ("mutation_probability", C.c_float),
        ("mutation_sigma", C.c_float),
        ("row_scale_probability", C.c_float),
    ]


@lru_cache(None)
def lib() -> C.CDLL:
    path = HERE / "_lib" / "libnwg_oracle.so"
    if not path.exists():
        from oracle import build

        build.build_oracle()
    L = C.CDLL(str(path))
    L.nwo_genome_stride_bytes.restype = _sz
    L.nwo_genome_stride_bytes.argtypes = [_sz]
    L.nwo_set_fma_mode.argtypes = [C.c_int]
    L.nwo_feedback.argtypes = [_u8p, _u8p, _u8p]
    L.nwo_encode_turn.argtypes = [_u16p, _u8p, _u8p, _f32p]
    L.nwo_policy_forward.argtypes = [_u16p, _sz, _u8p, _u8p, C.c_int, _f32p]
    L.nwo_score_action.restype = C.c_float
    L.nwo_score_action.argtypes = [_f32p, _u8p, _u16p]
    L.nwo_evaluate_individual.argtypes = [_u16p, _sz, _u8p, _sz, _u32p, _sz, _f32p, _u64p, _f32p, _i32p, _i32p,
                                          _f32p]
    L.nwo_normalize_fitness.restype = C.c_float
    L.nwo_normalize_fitness.argtypes = [C.c_float, _sz]
    L.nwo_cell_words_from_shards.restype = _sz
    L.nwo_cell_words_from_shards.argtypes = [C.POINTER(ShardRecord), _sz, _sz, _sz, _sz, _u32p, _sz]
    L.nwo_select_parent_pair.argtypes = [_f32p, _u8p, _sz, _sz, _sz, _sz, _sz, _u32p, _f32p, _sz, _u32p, _u32p]
    L.nwo_breed_and_mutate.argtypes = [_u16p, _u16p, _sz, _u16p, C.POINTER(DrawTape), C.POINTER(BreedConfig)]
    L.nwo_bootstrap_genome.argtypes = [_u16p, _sz, _f32p, _sz]
    L.nwo_bootstrap_normals_per_thread.restype = _sz
    L.nwo_bootstrap_normals_per_thread.argtypes = [_sz, _sz]
    L.nwo_summarize.argtypes = [_f32p, _sz, _f32p, _f32p, C.POINTER(_sz)]
    L.nwo_hint_grid_group.argtypes = [_u8p, C.POINTER(_sz), _u8p, _u8p]
    L.nwo_median_tail_norm.restype = C.c_float
    L.nwo_median_tail_norm.argtypes = [_u16p, _sz]
    L.nwo_inject_tails.argtypes = [_u16p, _sz, _u8p, _sz, _sz, _sz]
    return L


def set_fma_mode(on: bool) -> None:
    lib().nwo_set_fma_mode(1 if on else 0)


def word(s: str) -> np.ndarray:
    return np.frombuffer(s.upper().encode(), dtype=np.uint8) - ord("A")


def words_to_letters(words: list[str]) -> np.ndarray:
    return np.ascontiguousarray(np.stack([word(w) for w in words]).astype(np.uint8))


def feedback(guess: np.ndarray, solution: np.ndarray) -> np.ndarray | None:
    out = np.zeros(5, np.uint8)
    ok = lib().nwo_feedback(_ptr(np.ascontiguousarray(guess, np.uint8), _u8p),
                            _ptr(np.ascontiguousarray(solution, np.uint8), _u8p), _ptr(out, _u8p))
    return out if ok else None


def encode_turn(genome: np.ndarray, guess: np.ndarray, fb: np.ndarray) -> np.ndarray:
    out = np.zeros(64, np.float32)
    lib().nwo_encode_turn(_ptr(genome, _u16p), _ptr(np.ascontiguousarray(guess, np.uint8), _u8p),
                          _ptr(np.ascontiguousarray(fb, np.uint8), _u8p), _ptr(out, _f32p))
    return out


def policy_forward(genome: np.ndarray, solution: np.ndarray, guesses: np.ndarray) -> np.ndarray | None:
    """Policy vector for the grid with `solution` after `guesses` (rows of 5 letters)."""
    guesses = np.ascontiguousarray(np.asarray(guesses, np.uint8).reshape(-1, 5))
    fbs = np.zeros_like(guesses)
    finished = 0
    for t in range(len(guesses)):
        fbs[t] = feedback(guesses[t], solution)
        if np.array_equal(guesses[t], solution):
            finished = 1
    if len(guesses) >= 6:
        finished = 1
    out = np.zeros(64, np.float32)
    ok = lib().nwo_policy_forward(_ptr(genome, _u16p), len(guesses), _ptr(guesses, _u8p), _ptr(fbs, _u8p), finished,
                                  _ptr(out, _f32p))
    return out if ok else None


def score_action(policy: np.ndarray, w: np.ndarray, tail_row: np.ndarray) -> float:
    return lib().nwo_score_action(_ptr(np.ascontiguousarray(policy, np.float32), _f32p),
                                  _ptr(np.ascontiguousarray(w, np.uint8), _u8p),
                                  _ptr(np.ascontiguousarray(tail_row, np.uint16), _u16p))


def evaluate_individual(genome: np.ndarray, action_count: int, catalog: np.ndarray, cell_words: np.ndarray,
                        trace_policy: bool = False) -> dict:
    w = len(cell_words)
    scores = np.zeros(3 * w, np.float32)
    turns = np.zeros(3 * w, np.int32)
    guesses = np.zeros(3 * w * 6, np.int32)
    policy = np.zeros(3 * w * 6 * 64, np.float32) if trace_policy else None
    raw = C.c_float()
    steps = C.c_uint64()
    cw = np.ascontiguousarray(cell_words, np.uint32)
    status = lib().nwo_evaluate_individual(_ptr(genome, _u16p), action_count, _ptr(catalog, _u8p), len(catalog),
                                           _ptr(cw, _u32p), w, C.byref(raw), C.byref(steps), _ptr(scores, _f32p),
                                           _ptr(turns, _i32p), _ptr(guesses, _i32p), _ptr(policy, _f32p))
    return dict(status=status, raw=raw.value, steps=steps.value, scores=scores, turns=turns,
                guesses=guesses.reshape(3 * w, 6), policy=None if policy is None else policy.reshape(3 * w, 6, 64))


def normalize_fitness(raw: float, w: int) -> float:
    return lib().nwo_normalize_fitness(raw, w)


def cell_words_from_shards(shards: list[ShardRecord], rows: int, cols: int, cell: int, capacity: int = 8192):
    arr = (ShardRecord * len(shards))(*shards)
    out = np.zeros(capacity, np.uint32)
    n = lib().nwo_cell_words_from_shards(arr, len(shards), rows, cols, cell, _ptr(out, _u32p), capacity)
    return out[:n].copy()


def select_parent_pair(fitness, has, rows, cols, next_rows, child, radius, draws, weights):
    p1 = C.c_uint32()
    p2 = C.c_uint32()
    ok = lib().nwo_select_parent_pair(_ptr(np.ascontiguousarray(fitness, np.float32), _f32p),
                                      _ptr(np.ascontiguousarray(has, np.uint8), _u8p), rows, cols, next_rows, child,
                                      radius, _ptr(np.ascontiguousarray(draws, np.uint32), _u32p),
                                      _ptr(np.ascontiguousarray(weights, np.float32), _f32p), len(weights) - 1,
                                      C.byref(p1), C.byref(p2))
    return (p1.value, p2.value) if ok else None


def breed_and_mutate(p1: np.ndarray, p2: np.ndarray, action_count: int, tape: dict, cfg: dict) -> np.ndarray | None:
    child = np.zeros(genome_halfs(action_count), np.uint16)
    t = DrawTape(_ptr(tape["raw"], _u32p), _ptr(tape["uniform"], _f32p), _ptr(tape["normal_pair"], _f32p),
                 len(tape["raw"]), 0, 0, 0.0, 0)
    c = BreedConfig(cfg["l1"], cfg["l2"], cfg["l3"], cfg["p"], cfg["sigma"], cfg.get("row_scale", 0.0))
    ok = lib().nwo_breed_and_mutate(_ptr(p1, _u16p), _ptr(p2, _u16p), action_count, _ptr(child, _u16p),
                                    C.byref(t), C.byref(c))
    return child if ok else None


def bootstrap_normals_per_thread(action_count: int) -> int:
    return max(lib().nwo_bootstrap_normals_per_thread(action_count, t) for t in range(256))


def bootstrap_genome(action_count: int, normals: np.ndarray, per_thread: int) -> np.ndarray:
    g = np.zeros(genome_halfs(action_count), np.uint16)
    lib().nwo_bootstrap_genome(_ptr(g, _u16p), action_count, _ptr(np.ascontiguousarray(normals, np.float32), _f32p),
                               per_thread)
    return g


def hint_grid_group(word: np.ndarray):
    """(turn counts[3], guesses[3][4][5], feedbacks[3][4][5]) of a word's hint grids, or None."""
    turns = (_sz * 3)()
    guesses = np.zeros((3, 4, 5), np.uint8)
    fbs = np.zeros((3, 4, 5), np.uint8)
    w = np.ascontiguousarray(np.asarray(word, np.uint8))
    ok = lib().nwo_hint_grid_group(_ptr(w, _u8p), turns, _ptr(guesses, _u8p), _ptr(fbs, _u8p))
    return (list(turns), guesses, fbs) if ok else None


def median_tail_norm(genome: np.ndarray, rows: int) -> float:
    return float(lib().nwo_median_tail_norm(_ptr(np.ascontiguousarray(genome, np.uint16), _u16p), rows))


def inject_tails(genome: np.ndarray, parent_action_count: int, catalog: np.ndarray, first: int, count: int):
    """(status, genome with rows parent_action_count .. + count injected); genome needs room for the rows."""
    g = np.array(genome, np.uint16, copy=True)
    cat = np.ascontiguousarray(np.asarray(catalog, np.uint8))
    st = lib().nwo_inject_tails(_ptr(g, _u16p), parent_action_count, _ptr(cat, _u8p), len(cat), first, count)
    return st, g


def summarize(fitness: np.ndarray):
    best = C.c_float()
    avg = C.c_float()
    bi = _sz()
    f = np.ascontiguousarray(fitness, np.float32)
    lib().nwo_summarize(_ptr(f, _f32p), len(f), C.byref(best), C.byref(avg), C.byref(bi))
    return best.value, avg.value, bi.value


# ---------------- reference host library (oracle/_ref/libref_host.so) ----------------

@lru_cache(None)
def ref_host() -> C.CDLL | None:
    path = HERE / "_ref" / "libref_host.so"
    if not path.exists():
        return None
    L = C.CDLL(str(path))
    L.refhost_feedback.argtypes = [_u8p, _u8p, _u8p]
    L.refhost_policy_forward.argtypes = [_u8p, _u8p, _sz, _u8p, _f32p]
    L.refhost_score_action.restype = C.c_float
    L.refhost_score_action.argtypes = [_f32p, _u8p, _u8p]
    L.refhost_genome_stride_bytes.restype = _sz
    L.refhost_genome_stride_bytes.argtypes = [_sz]
    L.refhost_evaluate_population.argtypes = [_u8p, _sz, _sz, _sz, _u8p, _u32p, _u32p, _u32p, C.c_int, _f32p, _u64p,
                                              C.POINTER(C.c_int)]
    return L


@lru_cache(None)
def ref_ckpt() -> C.CDLL | None:
    """The reference's runtime-checkpoint code (oracle/ref_ckpt_harness.cu), or None when not built."""
    path = HERE / "_ref" / "libref_ckpt.so"
    if not path.exists():
        return None
    L = C.CDLL(str(path))
    L.refckpt_roundtrip.argtypes = [C.c_char_p, C.c_char_p]
    L.refckpt_write_synthetic.argtypes = [C.c_char_p, C.c_uint32, _sz, _sz, _sz, _sz, C.c_int]
    L.refckpt_identity_hash.restype = C.c_uint64
    L.refckpt_identity_hash.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, _sz]
    L.refckpt_layouts.argtypes = [C.POINTER(_sz)]
    L.refckpt_runtime_capture.argtypes = [C.c_void_p, C.c_void_p, _sz, _sz, C.c_uint32, _sz, C.c_uint32, C.c_void_p,
                                          C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_char_p]
    L.refckpt_runtime_evaluate.argtypes = [C.c_void_p, C.c_void_p, _sz, _sz, C.c_uint32, _sz, C.c_void_p, C.c_void_p,
                                           C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.refckpt_time_evaluation.argtypes = [C.c_void_p, C.c_void_p, _sz, _sz, C.c_uint32, _sz, C.c_void_p, _sz,
                                          C.c_void_p, C.c_void_p]
    L.refart_write.argtypes = [C.c_char_p, C.c_char_p, C.c_void_p, C.c_void_p, _sz, C.c_void_p, C.c_char_p]
    L.refart_read.argtypes = [C.c_char_p, C.c_char_p, C.c_void_p, C.c_void_p, _sz, C.c_void_p, C.POINTER(_sz),
                              C.c_char_p, _sz]
    L.refconv_plan.argtypes = [_sz, _sz, C.c_uint32, _sz, C.c_void_p, C.POINTER(_sz), C.c_void_p, C.POINTER(_sz),
                               C.c_void_p, C.POINTER(_sz)]
    L.refconv_metrics.argtypes = [C.c_void_p, _sz, _sz, C.c_void_p, _sz, C.c_void_p]
    L.refsm_select_many.argtypes = [C.c_void_p, _sz, C.c_void_p, _sz, C.c_void_p, C.c_void_p, C.c_void_p, _sz,
                                    C.c_void_p, C.c_void_p, C.c_void_p]
    L.refckpt_runtime_resume.argtypes = [C.c_char_p, C.c_void_p, _sz, C.c_void_p, _sz, C.POINTER(_sz),
                                         C.POINTER(_sz)]
    return L


def ref_host_policy_forward(genome: np.ndarray, solution: np.ndarray, guesses: np.ndarray) -> np.ndarray | None:
    guesses = np.ascontiguousarray(np.asarray(guesses, np.uint8).reshape(-1, 5))
    out = np.zeros(64, np.float32)
    ok = ref_host().refhost_policy_forward(_ptr(genome.view(np.uint8), _u8p),
                                           _ptr(np.ascontiguousarray(solution, np.uint8), _u8p), len(guesses),
                                           _ptr(guesses, _u8p), _ptr(out, _f32p))
    return out if ok else None


def ref_host_evaluate(genomes: np.ndarray, action_count: int, catalog: np.ndarray, cell_offsets: np.ndarray,
                      cell_words: np.ndarray, cells: np.ndarray, threads: int):
    """genomes: (n, halfs) uint16; returns (raw fitness, steps, status) per individual."""
    n = genomes.shape[0]
    raw = np.zeros(n, np.float32)
    steps = np.zeros(n, np.uint64)
    status = np.zeros(n, np.int32)
    g = np.ascontiguousarray(genomes)
    ref_host().refhost_evaluate_population(
        _ptr(g.view(np.uint8).reshape(-1), _u8p), g.shape[1] * 2, n, action_count, _ptr(catalog, _u8p),
        _ptr(np.ascontiguousarray(cell_offsets, np.uint32), _u32p),
        _ptr(np.ascontiguousarray(cell_words, np.uint32), _u32p), _ptr(np.ascontiguousarray(cells, np.uint32), _u32p),
        threads, _ptr(raw, _f32p), _ptr(steps, _u64p), status.ctypes.data_as(C.POINTER(C.c_int)))
    return raw, steps, status


# ---------------- GPU-side libraries (tapes and reference device code) ----------------

@lru_cache(None)
def tape_lib() -> C.CDLL:
    L = C.CDLL(str(HERE / "_lib" / "libnwg_tape.so"))
    L.tape_positions.argtypes = [C.c_uint32, C.c_ulonglong, _sz, C.c_void_p, C.c_void_p, C.c_void_p]
    L.tape_normal_streams.argtypes = [C.c_uint32, C.c_ulonglong, _sz, _sz, C.c_void_p]
    L.tape_selection_draws.argtypes = [C.c_uint32, _sz, _sz, C.c_void_p]
    L.tape_pow_table.argtypes = [C.c_float, _sz, C.c_void_p]
    return L


@lru_cache(None)
def ref_dev() -> C.CDLL | None:
    path = HERE / "_ref" / "libref_dev.so"
    if not path.exists():
        return None
    L = C.CDLL(str(path))
    L.refdev_upload_catalog.argtypes = [_u8p, _sz]
    L.refdev_evaluate.argtypes = [C.c_void_p, _sz, _sz, _sz, _sz, C.c_void_p, _sz, _sz, C.c_void_p, C.c_void_p,
                                  C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.refdev_evaluate_csr.argtypes = [C.c_void_p, _sz, C.c_void_p, _sz, _sz, C.c_void_p, C.c_void_p, _sz,
                                      C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.refdev_select.argtypes = [C.c_void_p, C.c_void_p, _sz, _sz, _sz, _sz, _sz, C.c_float, C.c_uint32, C.c_void_p,
                                C.c_void_p, C.c_void_p]
    L.refdev_breed.argtypes = [C.c_void_p, _sz, C.c_void_p, _sz, C.c_void_p, _sz, _sz, C.c_uint32, _sz, C.c_float,
                               C.c_float, C.c_float, C.c_float, C.c_float, C.c_float, C.c_void_p]
    L.refdev_bootstrap.argtypes = [C.c_void_p, _sz, _sz, _sz, C.c_uint32, _sz, C.c_void_p]
    L.refdev_inject.argtypes = [C.c_void_p, _sz, _sz, _sz, _sz, _sz, C.c_void_p, C.c_void_p]
    return L


# ---- shard-release statistics (test infrastructure: restatements of the reference's host reductions) ----

def fitness_telemetry(fitness: np.ndarray, pairs: np.ndarray | None = None) -> dict:
    """cli/run_genetic_algorithm.cu:1100-1183: sort, sequential double sums, nearest-rank percentiles, distinct
    count; with pairs, children per parent classified 0 / 1 / more."""
    import math

    v = np.sort(np.asarray(fitness, np.float32))
    n = len(v)
    total = 0.0
    for x in v:
        total += float(x)
    mean = total / n
    squares = 0.0
    for x in v:
        d = float(x) - mean
        squares += d * d
    mid = n // 2
    median = v[mid] if n % 2 else np.float32(np.float32(v[mid - 1] + v[mid]) * np.float32(0.5))

    def rank(p):
        r = math.ceil((p / 100.0) * n)
        i = 0 if r == 0 else r - 1
        return v[i if i < n else n - 1]

    out = dict(min=v[0], max=v[-1], mean=np.float32(mean), median=np.float32(median), p90=rank(90.0), p99=rank(99.0),
               stddev=np.float32(math.sqrt(squares / n)), distinct=int(1 + np.count_nonzero(v[1:] != v[:-1])))
    if pairs is not None:
        per = np.bincount(np.asarray(pairs, np.int64).reshape(-1), minlength=n)
        out.update(childless=int(np.sum(per == 0)), one_child=int(np.sum(per == 1)), more=int(np.sum(per > 1)))
    return out


def convergence_metrics(values: np.ndarray, pairs: np.ndarray) -> np.ndarray:
    """genetic_convergence.hpp:121-194 in its loop order with float32 rounding per operation: centroid mean, min,
    max, then pairwise mean, min, max."""
    values = np.asarray(values, np.float32)
    organisms, weights = values.shape
    centroid = np.zeros(weights, np.float32)
    for o in range(organisms):
        centroid = centroid + values[o]
    inverse = np.float32(1.0) / np.float32(organisms)
    centroid = centroid * inverse

    def distances(a, b):
        squared = np.zeros(a.shape[0], np.float32)
        for w in range(weights):
            d = a[:, w] - b[:, w]
            squared = squared + d * d
        return np.sqrt(squared)

    def summary(d, mean_of):
        total = np.float32(0.0)
        for x in d:
            total = np.float32(total + x)
        return [mean_of(total), np.float32(d.min()), np.float32(max(np.float32(0.0), d.max()))]

    out = summary(distances(values, np.broadcast_to(centroid, values.shape)), lambda t: np.float32(t * inverse))
    pairs = np.asarray(pairs, np.int64).reshape(-1, 2)
    if len(pairs) == 0:
        out += [np.float32(0.0), np.float32(0.0), np.float32(0.0)]
    else:
        out += summary(distances(values[pairs[:, 0]], values[pairs[:, 1]]),
                       lambda t: np.float32(t / np.float32(len(pairs))))
    return np.array(out, np.float32)


def ref_convergence_plan(organisms: int, trainable: int, seed: int, generation: int):
    """MakeSamplePlan of the reference (oracle/_ref/libref_ckpt.so)."""
    L = ref_ckpt()
    o = np.zeros(256, np.uint64)
    w = np.zeros(8192, np.uint64)
    p = np.zeros((512, 2), np.uint64)
    n_o, n_w, n_p = _sz(), _sz(), _sz()
    assert L.refconv_plan(organisms, trainable, seed, generation, o.ctypes.data, C.byref(n_o), w.ctypes.data,
                          C.byref(n_w), p.ctypes.data, C.byref(n_p)) == 1
    return o[:n_o.value], w[:n_w.value], p[:n_p.value]


def ref_convergence_metrics(values: np.ndarray, pairs: np.ndarray) -> np.ndarray:
    """TryComputeMetrics of the reference (oracle/_ref/libref_ckpt.so)."""
    values = np.ascontiguousarray(values, np.float32)
    p = np.ascontiguousarray(np.asarray(pairs, np.uint64).reshape(-1, 2))
    out = np.zeros(6, np.float32)
    assert ref_ckpt().refconv_metrics(values.ctypes.data, values.shape[0], values.shape[1], p.ctypes.data, len(p),
                                      out.ctypes.data) == 1
    return out


# ---- the surrogate network (test infrastructure: an FP64 restatement of csrc/surrogate_mlp.cu) ----

MLP_SHAPES = (("W1", (512, 8192)), ("b1", (512,)), ("W2", (128, 512)), ("b2", (128,)), ("w3", (128,)), ("b3", (1,)))


def mlp_unflatten(flat: np.ndarray) -> dict:
    out, off = {}, 0
    for name, shape in MLP_SHAPES:
        n = int(np.prod(shape))
        out[name] = np.asarray(flat[off:off + n], np.float64).reshape(shape)
        off += n
    return out


def bf16_round(a: np.ndarray) -> np.ndarray:
    """Round-to-nearest-even of float32 values to BF16, returned as float32."""
    bits = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    bits = (bits + 0x7FFF + ((bits >> 16) & 1)) >> 16 << 16
    return bits.astype(np.uint32).view(np.float32)


def _gelu(x):
    from scipy.special import erf

    return 0.5 * x * (1.0 + erf(x / np.sqrt(2.0)))


def _gelu_grad(x):
    from scipy.special import erf

    return 0.5 * (1.0 + erf(x / np.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / np.sqrt(2.0 * np.pi)


def mlp_forward(flat: np.ndarray, x: np.ndarray, bf16_w1: bool = True) -> tuple[np.ndarray, dict]:
    """y = b3 + w3 . gelu(b2 + W2 gelu(b1 + W1 x)) in FP64; W1 rounded to BF16 as the device products use it."""
    p = mlp_unflatten(flat)
    w1 = bf16_round(p["W1"].astype(np.float32)).astype(np.float64) if bf16_w1 else p["W1"]
    x = np.asarray(x, np.float64)
    z1 = x @ w1.T + p["b1"]
    a1 = _gelu(z1)
    z2 = a1 @ p["W2"].T + p["b2"]
    a2 = _gelu(z2)
    y = a2 @ p["w3"] + p["b3"][0]
    return y, dict(x=x, z1=z1, a1=a1, z2=z2, a2=a2)


def mlp_gradients(flat: np.ndarray, x: np.ndarray, t: np.ndarray, bf16: bool = True) -> tuple[np.ndarray, float]:
    """Gradients of mean((y - t)^2) in FP64, flat in the parameter order. With bf16 the first layer's weight
    gradient uses BF16-rounded dZ1, as the device's tensor-core product does."""
    p = mlp_unflatten(flat)
    y, c = mlp_forward(flat, x, bf16)
    n = len(t)
    dy = 2.0 * (y - np.asarray(t, np.float64)) / n
    dz2 = np.outer(dy, p["w3"]) * _gelu_grad(c["z2"])
    dz1 = (dz2 @ p["W2"]) * _gelu_grad(c["z1"])
    dz1_w = bf16_round(dz1.astype(np.float32)).astype(np.float64) if bf16 else dz1
    grads = [dz1_w.T @ c["x"], dz1.sum(0), dz2.T @ c["a1"], dz2.sum(0), dy @ c["a2"], np.array([dy.sum()])]
    return np.concatenate([g.reshape(-1) for g in grads]), float(np.mean((y - t) ** 2))
