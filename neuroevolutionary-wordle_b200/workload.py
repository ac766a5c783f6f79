"""Seeded synthetic workloads with the shapes of the benchmark configurations.

No dataset ships with this package: catalog words are distinct synthetic 5-letter A-Z strings drawn
from an English-like unigram letter distribution, secrets are a seeded subset of them, and each cell
of the toroidal grid gets its own list of secrets (CSR form), either of fixed size or of log-uniform
size.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

# Relative letter frequencies of English text, A..Z (percent).
ENGLISH_UNIGRAM = np.array([8.2, 1.5, 2.8, 4.3, 12.7, 2.2, 2.0, 6.1, 7.0, 0.15, 0.77, 4.0, 2.4, 6.7, 7.5, 1.9, 0.095,
                            6.0, 6.3, 9.1, 2.8, 0.98, 2.4, 0.15, 2.0, 0.074])


def synthetic_words(count: int, seed: int) -> np.ndarray:
    """`count` distinct words as (count, 5) letter indices."""
    rng = np.random.default_rng(seed)
    p = ENGLISH_UNIGRAM / ENGLISH_UNIGRAM.sum()
    seen: set[bytes] = set()
    out = np.zeros((count, 5), np.uint8)
    n = 0
    while n < count:
        batch = rng.choice(26, size=(2 * (count - n) + 16, 5), p=p).astype(np.uint8)
        for w in batch:
            key = w.tobytes()
            if key in seen:
                continue
            seen.add(key)
            out[n] = w
            n += 1
            if n == count:
                break
    return out


def secret_subset(word_count: int, subset_size: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed + 1)
    return rng.permutation(word_count)[:subset_size].astype(np.uint32)


def fixed_cell_lists(cells: int, per_cell: int, subset: np.ndarray, seed: int):
    """Each cell draws `per_cell` distinct secrets uniformly from `subset` (CSR offsets, words)."""
    rng = np.random.default_rng(seed + 2)
    words = np.concatenate([rng.choice(subset, size=per_cell, replace=False) for _ in range(cells)])
    offsets = np.arange(cells + 1, dtype=np.uint32) * per_cell
    return offsets.astype(np.uint32), words.astype(np.uint32)


def loguniform_cell_lists(cells: int, low: int, high: int, subset: np.ndarray, seed: int):
    """Per-cell list sizes floor(exp(U[ln low, ln high])), secrets drawn without replacement."""
    rng = np.random.default_rng(seed + 3)
    sizes = np.floor(np.exp(rng.uniform(np.log(low), np.log(high), size=cells))).astype(np.int64)
    sizes = np.clip(sizes, low, min(high, len(subset)))
    words = np.concatenate([rng.choice(subset, size=int(s), replace=False) for s in sizes])
    offsets = np.zeros(cells + 1, np.uint32)
    offsets[1:] = np.cumsum(sizes)
    return offsets, words.astype(np.uint32)


@dataclass(frozen=True)
class Workload:
    name: str
    population: int
    columns: int
    action_count: int
    secret_subset: int
    secrets_per_cell: int
    mutation_probability: float = 0.05
    mutation_sigma: float = 0.02
    radius: int = 1
    seed: int = 0

    def catalog(self) -> np.ndarray:
        return synthetic_words(self.action_count, self.seed)

    def cell_lists(self):
        subset = secret_subset(self.action_count, self.secret_subset, self.seed)
        return fixed_cell_lists(self.population, self.secrets_per_cell, subset, self.seed)


# P=64 on 8x8, 512 words, 64 secrets per cell from a 256-word subset.
SMALL = Workload("p64_a512_s64", 64, 8, 512, 256, 64)
# P=4096 on 64x64, 4,739 words, 256 secrets per cell from a 2,315-word subset.
FULL = Workload("p4096_a4739_s256", 4096, 64, 4739, 2315, 256)
# The same per-individual work on 1,024 individuals (32x32): seven children per SM, slabs of 680 MB each.
QUARTER = Workload("p1024_a4739_s256", 1024, 32, 4739, 2315, 256)
# The same per-individual work on 256 individuals (16x16): a profiling case whose slab (170 MB) still exceeds L2.
MEDIUM = Workload("p256_a4739_s256", 256, 16, 4739, 2315, 256)
