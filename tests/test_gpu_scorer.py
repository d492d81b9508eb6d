"""The learned frontier scorer: gradients and logits against a CPU restatement, and what it gains.

The CPU restatement below computes the same 2x64 ReLU MLP in float64 from the same BF16-rounded
weights; the device kernels accumulate in FP32, so the tolerances are FP32-level (rtol 2e-3).
The gain test trains the scorer on traces of separately seeded queries and checks that KNN results
stay exact (identical to the FP64 brute force) while reporting the finest-level work with and
without the learned ranking.
"""
import numpy as np
import pytest

from conftest import oracle_from_handler

pytestmark = pytest.mark.gpu

HID = 64


def bf16(x):
    u = np.asarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def split(p, n_in):
    o = 0
    W1 = p[o:o + n_in * HID].reshape(n_in, HID); o += n_in * HID
    b1 = p[o:o + HID]; o += HID
    W2 = p[o:o + HID * HID].reshape(HID, HID); o += HID * HID
    b2 = p[o:o + HID]; o += HID
    w3 = p[o:o + HID]; o += HID
    b3 = p[o]
    return W1, b1, W2, b2, w3, b3


def cpu_loss_grad(p, X, y):
    n_in = X.shape[1]
    W1, b1, W2, b2, w3, b3 = split(bf16(p), n_in)
    X = X.astype(np.float64)
    a1 = X @ W1 + b1; h1 = np.maximum(a1, 0)
    a2 = h1 @ W2 + b2; h2 = np.maximum(a2, 0)
    z = h2 @ w3 + b3
    loss = np.mean(np.logaddexp(0, z) - y * z)
    dz = (1 / (1 + np.exp(-z)) - y) / len(y)
    dw3 = h2.T @ dz; db3 = dz.sum()
    dh2 = np.outer(dz, w3) * (a2 > 0)
    dW2 = h1.T @ dh2; db2 = dh2.sum(0)
    dh1 = (dh2 @ W2.T) * (a1 > 0)
    dW1 = X.T @ dh1; db1 = dh1.sum(0)
    g = np.concatenate([dW1.ravel(), db1, dW2.ravel(), db2, dw3, [db3]])
    return loss, g, z


@pytest.fixture(scope="module")
def env(tb, oracle_mod, tmp_path_factory, cuda):
    h = tb.QueryHandler.generate(400000, 8, 1.0, 100.0, False, 4, (100, 50, 20), 41, 2.5)
    h.prepare_for_query(tb.LevelPolicy.L0)
    o = oracle_from_handler(oracle_mod, h, tmp_path_factory.mktemp("idx"))
    pts, ids = oracle_mod.decoded_points(o)
    return h, o, pts, ids


def test_scorer_gradients_and_logits_match_cpu(tb, env):
    h = env[0]
    p0 = h.scorer_params()
    n_in = (p0.size - 1 - 3 * HID - HID * HID) // HID
    rng = np.random.default_rng(0)
    p = rng.normal(0, 0.2, p0.size).astype(np.float32)
    h.scorer_set_params(p)
    X = rng.uniform(0, 1, (96, n_in)).astype(np.float32)
    y = (rng.uniform(0, 1, 96) < 0.3).astype(np.float32)
    loss, g = h.scorer_loss_grad(X, y)
    ref_loss, ref_g, ref_z = cpu_loss_grad(p.astype(np.float64), X, y.astype(np.float64))
    assert abs(loss - ref_loss) <= 2e-3 * abs(ref_loss) + 1e-6
    scale = np.abs(ref_g).max()
    assert np.allclose(g, ref_g, rtol=2e-3, atol=2e-4 * scale)
    z = h.scorer_logits(X)
    assert np.allclose(z, ref_z, rtol=2e-3, atol=1e-3)


def test_tensor_core_logits_match_bf16_model(tb, env):
    """The frontier-scoring kernel (tcgen05, BF16 operands, FP32 accumulation in tensor memory)
    against the float64 model with the same roundings: features and h1 in BF16. Sizes cover one
    row, a ragged tile and many tiles per CTA (the persistent loop)."""
    h = env[0]
    p0 = h.scorer_params()
    n_in = (p0.size - 1 - 3 * HID - HID * HID) // HID
    rng = np.random.default_rng(4)
    p = rng.normal(0, 0.2, p0.size).astype(np.float32)
    h.scorer_set_params(p)
    W1, b1, W2, b2, w3, b3 = split(bf16(p), n_in)
    for n in (1, 300, 200000):
        X = rng.uniform(-1, 1, (n, n_in)).astype(np.float32)
        h1 = bf16(np.maximum(bf16(X) @ W1 + b1, 0))
        ref = np.maximum(h1 @ W2 + b2, 0) @ w3 + b3
        z = h.scorer_logits(X, tensor=True)
        assert np.allclose(z, ref, rtol=2e-3, atol=2e-3 * np.abs(ref).max()), n
        # against the CUDA-core forward (FP32 features and h1): the BF16 roundings only
        z32 = h.scorer_logits(X)
        assert np.abs(z - z32).max() <= 0.05 * np.abs(z32).max() + 0.05, n
    assert h.scorer_logits(np.zeros((0, n_in), np.float32), tensor=True).size == 0


def _points(pts, n, seed, noise):
    rng = np.random.default_rng(seed)
    return np.ascontiguousarray(pts[rng.integers(0, len(pts), n)] + rng.normal(0, noise, (n, pts.shape[1])))


def test_learned_ranking_keeps_results_exact_and_reports_gain(tb, env, oracle_mod, capsys):
    h, o, pts, ids = env
    train = _points(pts, 3000, 100, 1.0)
    losses = h.scorer_train(train, K=20, max_samples=200000, epochs=6, lr=3e-3, seed=5)
    assert losses[-1] < losses[0]
    test = _points(pts, 256, 200, 1.0)
    b = oracle_mod.brute_query(pts, ids, oracle_mod.KNN, test, K=20)
    work = {}
    for name, two_wave, learned in (("one-pass", False, False), ("two-wave lb", True, False),
                                    ("two-wave learned", True, True)):
        h.set_two_wave(two_wave)
        h.scorer_enable(learned)
        r = h.query_batch(tb.QueryType.POINT, test, tb.Mode.EXACT, K=20)
        assert np.array_equal(r.offsets.numpy(), b.offsets)
        assert np.array_equal(r.ids.numpy(), b.ids)
        assert np.array_equal(r.dist2.numpy(), b.dist2)
        work[name] = h.knn_counters()["rows"]
    h.set_two_wave(True)
    with capsys.disabled():
        print("\nfinest-level points tested per query:", {k: v / 256 for k, v in work.items()})
    assert work["two-wave lb"] < work["one-pass"]
    # The learned ranking bounds tau sooner than the lower bound does (measured 1.76x fewer rows).
    assert work["two-wave learned"] < 0.9 * work["two-wave lb"]


def test_scorer_save_load_round_trip(tb, env, tmp_path):
    h = env[0]
    path = str(tmp_path / "scorer.bin")
    h.scorer_save(path)
    p = h.scorer_params()
    h.scorer_set_params(np.zeros_like(p))
    h.scorer_load(path)
    assert np.array_equal(h.scorer_params(), p)
    with open(path, "r+b") as f:
        f.truncate(40)
    with pytest.raises(tb.TblaeqError):
        h.scorer_load(path)
