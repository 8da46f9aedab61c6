"""The FP64 network restatement (oracle/mlp_oracle.py) is pinned by finite
differences, so it can serve as the gradient check of the BF16 kernels."""
import numpy as np

from oracle import mlp_oracle as M


def test_parameter_layout():
    assert M.N_PARAMS == 5768
    p = M.init_params(1)
    W1 = p[M.OFF_W1:M.OFF_B1].reshape(64, 16)
    assert np.all(W1[:, 6:] == 0) and np.any(W1[:, :6] != 0)
    W3 = p[M.OFF_W3:M.OFF_B3].reshape(8, 64)
    assert np.all(W3[1:] == 0)


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = M.init_params(3).astype(np.float64)
    p[M.OFF_B1:M.OFF_W2] = rng.normal(0, 0.1, 64)
    X = rng.normal(0, 1, (40, 6))
    y = (rng.random(40) < 0.3).astype(np.float64)
    loss, g = M.loss_and_grad(p, X, y)
    idx = np.concatenate([rng.choice(np.arange(M.OFF_W1, M.OFF_B1).reshape(64, 16)[:, :6].ravel(), 10),
                          rng.integers(M.OFF_B1, M.OFF_W2, 5), rng.integers(M.OFF_W2, M.OFF_B2, 10),
                          rng.integers(M.OFF_B2, M.OFF_W3, 5), rng.integers(M.OFF_W3, M.OFF_W3 + 64, 8), [M.OFF_B3]])
    for i in idx:
        h = 1e-6
        pp = p.copy(); pp[i] += h
        pm = p.copy(); pm[i] -= h
        fd = (M.loss_and_grad(pp, X, y)[0] - M.loss_and_grad(pm, X, y)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])
    # padding stays zero
    assert np.all(g[M.OFF_W1:M.OFF_B1].reshape(64, 16)[:, 6:] == 0)
    assert np.all(g[M.OFF_W3 + 64:M.OFF_B3] == 0)


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.14159], np.float32)
    r = M.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0  # halfway rounds to even
    assert r[2] == 1.0078125
    assert abs(r[3] + 3.140625) < 1e-9
