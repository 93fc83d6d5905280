"""Pins the NumPy perceptron oracle: analytic gradients against central
finite differences."""
import numpy as np

from oracle import mlp


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(3)
    n_in, n_out = 27, 2
    n = 64 * n_in + 64 + 64 * 64 + 64 + n_out * 64 + n_out
    p = rng.normal(0, 0.2, n)
    x = rng.normal(0, 1, (10, n_in))
    t = rng.normal(0, 1, (10, n_out))
    loss, g = mlp.loss_and_grad(p, x, t)
    idx = rng.choice(n, 40, replace=False)
    for i in idx:
        e = np.zeros(n)
        e[i] = 1e-6
        fd = (mlp.loss_and_grad(p + e, x, t)[0] - mlp.loss_and_grad(p - e, x, t)[0]) / 2e-6
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i])), (i, fd, g[i])
