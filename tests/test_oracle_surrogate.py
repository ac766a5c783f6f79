"""The surrogate network's CPU oracle (no GPU): its analytic gradient against central finite differences, in FP64.

The oracle (oracle/pyoracle.py: mlp_forward, mlp_gradients) restates csrc/surrogate_mlp.cu's network
(8,192 -> 512 -> 128 -> 1, GELU, loss mean((y - t)^2)); the GPU tests check the device's gradients against it.
"""
import numpy as np

from oracle import pyoracle as O


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    sizes = [int(np.prod(s)) for _, s in O.MLP_SHAPES]
    flat = np.concatenate([rng.standard_normal(n) * (0.05 if n > 1000 else 0.3) for n in sizes])
    x = rng.standard_normal((4, 8192)) * 0.5
    t = rng.standard_normal(4)
    grads, _ = O.mlp_gradients(flat, x, t, bf16=False)
    offsets = np.cumsum([0] + sizes)
    picks = [offsets[0] + 5 * 8192 + 17, offsets[0] + 300 * 8192 + 8000, offsets[1] + 3, offsets[2] + 100 * 512 + 7,
             offsets[3] + 64, offsets[4] + 127, offsets[5]]
    h = 1e-6
    for i in picks:
        up, down = flat.copy(), flat.copy()
        up[i] += h
        down[i] -= h
        yu, _ = O.mlp_forward(up, x, bf16_w1=False)
        yd, _ = O.mlp_forward(down, x, bf16_w1=False)
        numeric = (np.mean((yu - t) ** 2) - np.mean((yd - t) ** 2)) / (2 * h)
        assert abs(numeric - grads[i]) <= 1e-6 + 1e-5 * abs(numeric), (i, numeric, grads[i])


def test_bf16_rounding_is_round_to_nearest_even():
    v = np.array([1.0, 1.00390625, 1.005859375, -3.0e-3, 65504.0, 1.0 + 2 ** -8], np.float32)
    r = O.bf16_round(v)
    assert r[0] == 1.0 and r[1] == 1.0  # halfway between 1 and 1 + 2^-7 rounds to even (1)
    assert r[2] == np.float32(1.0078125)
    assert np.all(np.abs(r - v) <= np.abs(v) * 2 ** -8)
