"""The float64 network restatement used as the gradient checker, checked
against finite differences (no GPU)."""
import numpy as np

from oracle import mlp_oracle as M


def test_parameter_count():
    assert M.N_PARAMS == 112 * 64 + 64 + 3 * (64 * 64 + 64) + 64 + 1


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    P = rng.normal(0, 0.2, M.N_PARAMS)
    X = rng.normal(0, 1, (16, M.K_IN))
    X[:, M.K_USED:] = 0
    t = rng.uniform(0, 1, 16)
    # exact arithmetic version for the finite difference: no bf16 rounding
    real_bf16 = M.bf16
    M.bf16 = lambda x: np.asarray(x, np.float64)
    try:
        loss, g, _ = M.forward_backward(P, X, t)
        idx = rng.choice(M.N_PARAMS, 40, replace=False)
        for i in idx:
            e = np.zeros_like(P)
            e[i] = 1e-6
            num = (M.forward_backward(P + e, X, t)[0] - M.forward_backward(P - e, X, t)[0]) / 2e-6
            assert abs(num - g[i]) <= 1e-6 + 1e-4 * abs(num), (i, num, g[i])
    finally:
        M.bf16 = real_bf16


def test_encoding_shape_and_range():
    X = M.encode(np.array([[0.25, 0.5, 0.75]]), np.array([[0, 0, 1.0]]), (0, 0, 0), (1, 1, 1))
    assert X.shape == (1, 112) and np.all(np.abs(X) <= 1) and np.all(X[:, 102:] == 0)
    assert np.isclose(X[0, 0], -0.5) and np.isclose(X[0, 6], np.sin(np.pi * 0.25))
