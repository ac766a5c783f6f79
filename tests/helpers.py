"""Shared builders for the tests: genome images, fixtures and synthetic catalogs."""
from __future__ import annotations

import numpy as np

POLICY_HALFS = 150528
TAIL_DIM = 38

# Genome image offsets in halfs (parameter structs in declaration order).
ENC_W1, ENC_B1, ENC_W2, ENC_B2 = 0, 18560, 18688, 26880
TR_W1, TR_B1, TR_W2, TR_B2, TR_W3, TR_B3 = 26944, 109120, 109376, 142144, 142272, 150464
LAYERS = [  # (weight offset, bias offset, inputs, outputs)
    (ENC_W1, ENC_B1, 145, 128),
    (ENC_W2, ENC_B2, 128, 64),
    (TR_W1, TR_B1, 321, 256),
    (TR_W2, TR_B2, 256, 128),
    (TR_W3, TR_B3, 128, 64),
]


def h(value: float) -> int:
    return int(np.array(value, np.float16).view(np.uint16))


def empty_genome(action_count: int) -> np.ndarray:
    return np.zeros(POLICY_HALFS + TAIL_DIM * action_count, np.uint16)


def random_genome(rng: np.random.Generator, action_count: int, scale: float = 1.0) -> np.ndarray:
    """He-normal weights, small random biases and N(0, 0.05) tails, stored in fp16."""
    g = empty_genome(action_count)
    for w_off, b_off, n_in, n_out in LAYERS:
        w = rng.normal(0.0, scale * np.sqrt(2.0 / n_in), n_in * n_out).astype(np.float16)
        g[w_off:w_off + n_in * n_out] = w.view(np.uint16)
        b = rng.normal(0.0, 0.05, n_out).astype(np.float16)
        g[b_off:b_off + n_out] = b.view(np.uint16)
    tail = rng.normal(0.0, 0.05, TAIL_DIM * action_count).astype(np.float16)
    g[POLICY_HALFS:] = tail.view(np.uint16)
    return g


def set_w(g, w_off, n_in, o, i, value):
    g[w_off + o * n_in + i] = h(value)


def encoder_fixture(g: np.ndarray) -> None:
    """tests/model/input_encoder/shared_encoder_fixture.hpp: sparse hand-set encoder weights."""
    letter = lambda p, l: p * 26 + l  # noqa: E731
    tile = lambda p, f: 130 + p * 3 + f  # noqa: E731
    for o, b in enumerate([-2.0, 1.0, -1.0]):
        g[ENC_B1 + o] = h(b)
    set_w(g, ENC_W1, 145, 0, letter(0, 0), 1.5)
    set_w(g, ENC_W1, 145, 0, letter(1, 1), 0.5)
    set_w(g, ENC_W1, 145, 0, tile(0, 0), 4.0)
    set_w(g, ENC_W1, 145, 1, letter(2, 2), 2.0)
    set_w(g, ENC_W1, 145, 1, tile(2, 2), -5.0)
    set_w(g, ENC_W1, 145, 1, tile(4, 1), 0.5)
    set_w(g, ENC_W1, 145, 2, letter(3, 3), 1.0)
    set_w(g, ENC_W1, 145, 2, letter(4, 4), 2.0)
    set_w(g, ENC_W1, 145, 2, tile(1, 1), 0.25)
    set_w(g, ENC_W1, 145, 2, tile(3, 0), 0.75)
    for o, b in enumerate([0.5, -2.0, 1.25]):
        g[ENC_B2 + o] = h(b)
    set_w(g, ENC_W2, 128, 0, 0, 2.0)
    set_w(g, ENC_W2, 128, 0, 2, -1.0)
    set_w(g, ENC_W2, 128, 1, 0, -0.5)
    set_w(g, ENC_W2, 128, 1, 2, 4.0)
    set_w(g, ENC_W2, 128, 2, 1, 7.0)


def policy_fixture(g: np.ndarray) -> None:
    """tests/model/policy_model/policy_model_fixture.hpp: encoder fixture + sparse trunk."""
    encoder_fixture(g)
    g[TR_B1 + 0] = h(-1.0)
    set_w(g, TR_W1, 321, 0, 1, 1.0)
    set_w(g, TR_W1, 321, 0, 2, 0.5)
    g[TR_B1 + 1] = h(0.0)
    set_w(g, TR_W1, 321, 1, 2, -0.25)
    set_w(g, TR_W1, 321, 1, 3, 2.0)
    g[TR_B1 + 2] = h(-1.5)
    set_w(g, TR_W1, 321, 2, 0, 2.0)
    g[TR_B2 + 0] = h(0.25)
    set_w(g, TR_W2, 256, 0, 0, 0.5)
    set_w(g, TR_W2, 256, 0, 1, 2.0)
    g[TR_B2 + 1] = h(-1.0)
    set_w(g, TR_W2, 256, 1, 0, 0.25)
    set_w(g, TR_W2, 256, 1, 2, 4.0)
    g[TR_B3 + 0] = h(-2.0)
    set_w(g, TR_W3, 128, 0, 0, 2.0)
    g[TR_B3 + 1] = h(0.5)
    set_w(g, TR_W3, 128, 1, 0, -0.5)
    set_w(g, TR_W3, 128, 1, 1, 4.0)
    g[TR_B3 + 2] = h(1.0)
    set_w(g, TR_W3, 128, 2, 1, 3.0)


def synthetic_words(rng: np.random.Generator, count: int) -> np.ndarray:
    """`count` distinct 5-letter words (letter indices 0..25), English-like unigram letter frequencies."""
    freq = np.array([8.2, 1.5, 2.8, 4.3, 12.7, 2.2, 2.0, 6.1, 7.0, 0.15, 0.77, 4.0, 2.4, 6.7, 7.5, 1.9, 0.095, 6.0,
                     6.3, 9.1, 2.8, 0.98, 2.4, 0.15, 2.0, 0.074])
    freq = freq / freq.sum()
    seen = set()
    out = []
    while len(out) < count:
        w = tuple(rng.choice(26, 5, p=freq).tolist())
        if w in seen:
            continue
        seen.add(w)
        out.append(w)
    return np.array(out, np.uint8)
