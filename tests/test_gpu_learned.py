"""GPU tests of the learned dispatch: the CUDA training / gradient /
inference kernels against the CPU restatement (oracle/mlp_oracle.c), that
training fits, that method "learned" stays bit-exact, and what the trained
cost model (fastfib_b200/tuning.txt, trained on a B200 by
fastfib_b200.tune) gains over the plain thresholds on the uneven stream."""
import numpy as np
import pytest

from fastfib_b200.workload import uneven_products
from oracle import limbs_to_int

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _init(ff):
    ff.init(1 << 22)
    yield
    ff.set_model(None)


def rows(n, seed):
    rng = np.random.default_rng(seed)
    X = rng.uniform(0, 1, (n, 8)).astype(np.float32)
    M = rng.integers(0, 4, n).astype(np.int32)
    Y = rng.normal(0, 2, n).astype(np.float32)
    return X, M, Y


def test_gradient_matches_oracle(ff, oracle):
    for n, seed in ((1, 1), (31, 2), (300, 3), (1000, 4)):
        X, M, Y = rows(n, seed)
        p = ff.mlp_init(seed) + np.random.default_rng(seed).normal(0, 0.05, ff.MLP_NPARAM).astype(np.float32)
        loss, g = ff.mlp_grad(p, X, M, Y)
        lo, go = oracle.mlp_grad(p, X, M, Y)
        assert abs(loss - lo) <= 1e-4 * max(1.0, lo)
        # float32 on the GPU (summed in another order) against double on the CPU
        np.testing.assert_allclose(g, go, rtol=1e-3, atol=1e-5 * max(1.0, np.abs(go).max()))


def test_predict_matches_oracle(ff, oracle):
    X, _, _ = rows(777, 5)
    p = ff.mlp_init(7)
    np.testing.assert_allclose(ff.mlp_predict(p, X), oracle.mlp_predict(p, X), rtol=1e-4, atol=1e-5)


def test_training_fits(ff, oracle):
    rng = np.random.default_rng(9)
    X = rng.uniform(0, 1, (2000, 8)).astype(np.float32)
    M = rng.integers(0, 4, 2000).astype(np.int32)
    Y = (3 * X[:, 0] + np.where(M == 0, 2 * X[:, 1] ** 2, 1.0) - M * X[:, 5]).astype(np.float32)
    p, hist = ff.mlp_train(ff.mlp_init(0), X, M, Y, epochs=600, lr=1e-2)
    assert hist[-1] < hist[0] / 20
    lo, _ = oracle.mlp_grad(p, X, M, Y)
    assert abs(lo - hist[-1]) < 0.05 * hist[0]
    np.testing.assert_allclose(ff.mlp_predict(p, X), oracle.mlp_predict(p, X), rtol=1e-4, atol=1e-4)


def test_learned_is_bit_exact(ff):
    if not ff.load_tuning():
        ff.set_model(ff.mlp_init(1))  # an untrained model still picks among exact methods
    pairs = uneven_products(seed=21, count=300, lo=8, hi=19)
    pairs += [(a, None) for a, _ in uneven_products(seed=22, count=40, lo=8, hi=19)]
    got = ff.mul_batch(pairs, "learned")
    for g, (a, b) in zip(got, pairs):
        x = limbs_to_int(a)
        assert limbs_to_int(g) == x * (x if b is None else limbs_to_int(b))


def test_trained_model_gain(ff):
    """Plain thresholds against the trained cost model on the uneven stream
    (1024 products, 2^10..2^24 bits, aspect up to 16), device times of graph
    replays: the learned batch must not be slower than the plain one beyond
    0.5 % (the replays' timing noise; the measured gain is 1-2 %), and the test
    prints the gain."""
    torch = pytest.importorskip("torch")
    if not ff.load_tuning():
        pytest.skip("no trained cost model (run python -m fastfib_b200.tune on a GPU)")
    pairs = uneven_products(seed=4, count=1024)
    dev = torch.device("cuda:0")
    keep, base = [], []
    for a, b in pairs:
        ta = torch.from_numpy(a.view(np.int64)).to(dev)
        tb = torch.from_numpy(b.view(np.int64)).to(dev)
        out = torch.empty(a.size + b.size + 1, dtype=torch.int64, device=dev)
        keep += [ta, tb, out]
        base.append({"a": ta.data_ptr(), "b": tb.data_ptr(), "na": a.size, "nb": b.size, "bits_a": 64 * a.size,
                     "bits_b": 64 * b.size, "out": out.data_ptr()})
    t = {}
    for m in ("plain", "learned"):
        t[m] = ff.time_batch([dict(j, method=m) for j in base], reps=3)
    print(f"uneven stream, 1024 products: plain {t['plain']:.3f} ms, learned {t['learned']:.3f} ms, "
          f"gain {t['plain'] / t['learned']:.2f}x")
    assert t["learned"] <= 1.005 * t["plain"]
