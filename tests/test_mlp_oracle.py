"""The network restatement itself (oracle/mlp_oracle.py) on the CPU: its
backward pass against central differences of its forward pass, with the
bf16 rounding switched off so that the loss is smooth in the parameters."""
import numpy as np
import pytest


def test_oracle_backward_matches_finite_differences(monkeypatch):
    import mlp_oracle as M

    monkeypatch.setattr(M, "bf16", lambda a: np.asarray(a, dtype=np.float64))
    monkeypatch.setattr(M, "PARAM_DTYPE", np.float64)
    rng = np.random.default_rng(2)
    x = rng.uniform(0, 1, (64, 7))
    y = np.sin(x.sum(axis=1))
    p = np.zeros(M.PARAMS)
    p[M.W0:M.B0] = (rng.uniform(-1, 1, (128, 16)) * (np.arange(16) < 7)).ravel() * 0.4
    for a, b in [(M.W1, M.B1), (M.W2, M.B2)]:
        p[a:b] = rng.uniform(-1, 1, b - a) * 0.09
    p[M.W3:M.B3] = rng.uniform(-1, 1, 128) * 0.09
    p[M.B0:M.W1] = rng.uniform(-0.1, 0.1, 128)
    p[M.B3] = 0.05
    loss, G = M.grad(p, x, y)

    def f(q):
        g, _ = M.forward(q, x)
        return np.mean((g - y) ** 2)

    h = 1e-6
    for idx in [M.W0 + 3, M.W0 + 16 * 5 + 6, M.B0 + 7, M.W1 + 1000, M.B1 + 3, M.W2 + 4242,
                M.B2 + 100, M.W3 + 17, M.B3]:
        q1, q2 = p.copy(), p.copy()
        q1[idx] += h
        q2[idx] -= h
        fd = (f(q1) - f(q2)) / (2 * h)
        assert abs(fd - G[idx]) <= 1e-6 * max(1.0, abs(fd)), (idx, fd, G[idx])
    assert abs(loss - f(p)) <= 1e-15
