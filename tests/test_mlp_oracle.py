"""The surrogate network's oracle (oracle/mlp.py): its hand-written
backpropagation against central finite differences in float64."""
import numpy as np

from mlp import NPARAM, forward, init_params, loss_and_grad


def test_oracle_gradient_finite_differences():
    rng = np.random.default_rng(0)
    p = init_params(3) + rng.normal(0, 0.05, NPARAM)
    x = np.zeros((40, 8))
    x[:, :5] = rng.normal(size=(40, 5))
    t = rng.normal(size=(40, 2))
    _, g = loss_and_grad(p, x, t)
    n = len(x)
    for i in rng.choice(NPARAM, 60, replace=False):
        if i < 64 * 8 and i % 8 >= 5:
            continue                        # padded inputs: zero gradient both ways
        e = np.zeros(NPARAM)
        e[i] = 1e-6
        lp, _ = loss_and_grad(p + e, x, t)
        lm, _ = loss_and_grad(p - e, x, t)
        fd = (lp - lm) / (2e-6) / n
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i])), (i, fd, g[i])


def test_oracle_forward_shapes():
    p = init_params(1)
    y = forward(p, np.zeros((3, 8)))
    assert y.shape == (3, 2) and np.all(np.isfinite(y))
