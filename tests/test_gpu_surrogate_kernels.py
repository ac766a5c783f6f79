"""The surrogate's device kernels on the B200: the tcgen05 BF16 product, the behavioural descriptors, the network's
gradients against the FP64 CPU oracle, and learning.

The descriptors are the plain form's FP32 policy vectors (bit-exact with the CPU oracle's device-arithmetic mode) on
128 probe states of 0..4 turns, scaled and rounded to BF16: compared bit for bit. The product is checked against an
FP64 product of the same BF16 values (FP32 accumulation bound). The gradients are checked against
oracle/pyoracle.py's FP64 restatement, itself pinned by finite differences (tests/test_oracle_surrogate.py).
"""
import numpy as np
import pytest

from oracle import pyoracle as O
from tests import gpu_util as G
from tests import helpers as H

pytestmark = pytest.mark.gpu
capi = G.nwg.capi


def _bf16(t, a):
    return t.from_numpy(np.ascontiguousarray(a, np.float32)).to(t.bfloat16).cuda()


@pytest.mark.parametrize("m,n,k", [(128, 256, 64), (256, 512, 1024), (512, 8192, 1024), (1024, 512, 8192)])
def test_gemm_matches_fp64_product(m, n, k):
    t = G.torch()
    rng = np.random.default_rng(m + n + k)
    a = _bf16(t, rng.uniform(-1, 1, (m, k)))
    b = _bf16(t, rng.uniform(-1, 1, (n, k)))
    c = t.zeros((m, n), dtype=t.float32, device="cuda")
    capi.bf16_gemm_nt(a.data_ptr(), k, b.data_ptr(), k, c.data_ptr(), n, m, n, k, G.stream_handle())
    t.cuda.synchronize()
    ad = a.float().cpu().numpy().astype(np.float64)
    bd = b.float().cpu().numpy().astype(np.float64)
    ref = ad @ bd.T
    bound = (np.abs(ad) @ np.abs(bd).T) * (k * 2.0 ** -24) + 1e-30
    assert np.all(np.abs(c.cpu().numpy() - ref) <= bound)


def test_gemm_rejects_unsupported_shapes():
    t = G.torch()
    a = t.zeros((128, 64), dtype=t.bfloat16, device="cuda")
    c = t.zeros((128, 256), dtype=t.float32, device="cuda")
    with pytest.raises(capi.NwgError) as e:
        capi.bf16_gemm_nt(a.data_ptr(), 64, a.data_ptr(), 64, c.data_ptr(), 256, 128, 128, 64)
    assert e.value.status == 18


def _probes(rng, catalog, seed):
    letters = np.zeros((128, 4, 5), np.uint8)
    feedback = np.zeros((128, 4, 5), np.uint8)
    turns = np.zeros(128, np.uint8)
    secrets = np.zeros((128, 5), np.uint8)
    for p in range(128):
        secret = catalog[rng.integers(len(catalog))]
        secrets[p] = secret
        k = 0
        for _ in range(int(rng.integers(0, 5))):
            w = catalog[rng.integers(len(catalog))]
            fb = O.feedback(w, secret)
            if np.all(fb == 0):
                continue
            letters[p, k], feedback[p, k] = w, fb
            k += 1
        turns[p] = k
    return letters, feedback, turns, secrets


def test_descriptors_are_the_policy_vectors_in_bf16():
    t = G.torch()
    rng = np.random.default_rng(17)
    action_count = 300
    catalog = H.synthetic_words(rng, action_count)
    G.upload_catalog_everywhere(catalog)
    rt = G.nwg.Runtime(action_count, 4, 2)
    rt.bootstrap(4, seed=5)
    slab, pitch = rt.device_slab()
    gen = rt.current_generation()
    slots = G.dev(gen["slots"].astype(np.uint32))
    letters, feedback, turns, secrets = _probes(rng, catalog, 3)
    assert set(turns.tolist()) >= {0, 1, 2, 3, 4}
    out = t.zeros((4, 8192), dtype=t.bfloat16, device="cuda")
    scale = 0.75
    capi.descriptors(slab, pitch, slots.data_ptr(), 4, letters, feedback, turns, scale, out.data_ptr(),
                     G.stream_handle())
    got = out.view(t.int16).cpu().numpy().view(np.uint16).reshape(4, 128, 64)
    O.set_fma_mode(True)
    for i in range(4):
        genome = rt.download_slot(int(gen["slots"][i])).view(np.uint16)
        for p in range(128):
            policy = O.policy_forward(genome, secrets[p], letters[p, :turns[p]])
            want = (O.bf16_round(policy.astype(np.float32) * np.float32(scale)).view(np.uint32) >> 16).astype(np.uint16)
            assert np.array_equal(got[i, p], want), (i, p, int(turns[p]))
    rt.close()


def test_mlp_gradients_match_the_oracle():
    t = G.torch()
    rng = np.random.default_rng(5)
    rows = 128
    net = capi.Mlp(rows, seed=3)
    flat = net.parameters()
    x = O.bf16_round(rng.standard_normal((rows, 8192)).astype(np.float32) * 0.5)
    targets = rng.standard_normal(rows).astype(np.float32)
    xd = _bf16(t, x)
    td = t.from_numpy(targets).cuda()
    grads, loss = net.gradients(xd.data_ptr(), td.data_ptr(), rows)
    ref, ref_loss = O.mlp_gradients(flat.astype(np.float64), x.astype(np.float64), targets.astype(np.float64))
    assert abs(loss - ref_loss) <= 1e-4 * max(1.0, ref_loss)
    sizes = [int(np.prod(s)) for _, s in O.MLP_SHAPES]
    off = np.cumsum([0] + sizes)
    for k, (name, _) in enumerate(O.MLP_SHAPES):
        g, r = grads[off[k]:off[k + 1]].astype(np.float64), ref[off[k]:off[k + 1]]
        err = np.linalg.norm(g - r) / max(np.linalg.norm(r), 1e-30)
        # w3 and b3 sum (y - t) over the batch, with cancellation: their relative error follows the terms' size
        assert err <= {"W1": 2e-3, "w3": 1e-3, "b3": 2e-3}.get(name, 1e-4), (name, err)
    y = t.zeros(rows, dtype=t.float32, device="cuda")
    net.forward(xd.data_ptr(), rows, y.data_ptr())
    t.cuda.synchronize()
    ref_y, _ = O.mlp_forward(flat.astype(np.float64), x.astype(np.float64))
    assert np.allclose(y.cpu().numpy(), ref_y, rtol=1e-4, atol=1e-5)
    net.close()


def test_mlp_learns_a_ranking():
    t = G.torch()
    rng = np.random.default_rng(9)
    rows, held = 2048, 1024
    # low-rank inputs, as behavioural descriptors are: 16 latent factors spread over the 8,192 values
    latent = rng.standard_normal((rows + held, 16)).astype(np.float32)
    basis = (rng.standard_normal((16, 8192)) * 0.25).astype(np.float32)
    x = O.bf16_round(latent @ basis + 0.05 * rng.standard_normal((rows + held, 8192)).astype(np.float32))
    w = rng.standard_normal(16).astype(np.float32)
    targets = (np.tanh(latent @ w / 4) + 0.05 * rng.standard_normal(rows + held)).astype(np.float32)
    xd = _bf16(t, x)
    td = t.from_numpy(targets).cuda()
    net = capi.Mlp(rows, seed=1, learning_rate=1e-4)  # 1e-3 overfits the 8,192-wide first layer (held-out rho ~0.5)
    _, before = net.gradients(xd.data_ptr(), td.data_ptr(), rows)
    for step in range(150):
        b0 = (step % 2) * 1024
        net.train_step(xd[b0:b0 + 1024].data_ptr(), td[b0:b0 + 1024].data_ptr(), 1024)
    _, after = net.gradients(xd.data_ptr(), td.data_ptr(), rows)
    assert after < 0.25 * before
    y = t.zeros(held, dtype=t.float32, device="cuda")
    net.forward(xd[rows:].data_ptr(), held, y.data_ptr())
    t.cuda.synchronize()
    pred = y.cpu().numpy()
    rank = lambda v: np.argsort(np.argsort(v))
    rho = np.corrcoef(rank(pred), rank(targets[rows:]))[0, 1]
    assert rho > 0.8
    net.close()
