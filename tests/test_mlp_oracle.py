"""CPU tests of the cost model's CPU restatement (oracle/mlp_oracle.c), the
side the GPU kernels' gradients are checked against: its backpropagated
gradient equals central finite differences of its own loss."""
import numpy as np


def rows(n, seed):
    rng = np.random.default_rng(seed)
    X = rng.uniform(0, 1, (n, 8)).astype(np.float32)
    M = rng.integers(0, 4, n).astype(np.int32)
    Y = rng.normal(0, 2, n).astype(np.float32)
    return X, M, Y


def params(seed):
    rng = np.random.default_rng(seed)
    return rng.normal(0, 0.3, 1476).astype(np.float32)


def loss_of(oracle, p, X, M, Y):
    out = oracle.mlp_predict(p, X)
    e = out[np.arange(len(M)), M] - Y.astype(np.float64)
    return 0.5 * np.mean(e * e)


def test_gradient_matches_finite_differences(oracle):
    X, M, Y = rows(40, 1)
    p = params(2)
    loss, g = oracle.mlp_grad(p, X, M, Y)
    assert abs(loss - loss_of(oracle, p, X, M, Y)) < 1e-9
    rng = np.random.default_rng(3)
    idx = list(rng.choice(1476, 60, replace=False)) + [0, 255, 256, 287, 288, 1311, 1312, 1343, 1344, 1471, 1472, 1475]
    for i in idx:
        h = np.float32(1e-2)
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (loss_of(oracle, pp, X, M, Y) - loss_of(oracle, pm, X, M, Y)) / (float(pp[i]) - float(pm[i]))
        assert abs(fd - g[i]) <= 1e-4 * max(1.0, abs(g[i])) + 2e-6, (i, fd, g[i])
