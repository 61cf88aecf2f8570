"""The MLP oracle pinned by central finite differences of its own loss (CPU)."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "oracle"))
import mlp_oracle as mo  # noqa: E402


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(5)
    shapes = mo.layer_shapes(5, 7, 3, 4)
    p = rng.normal(size=mo.num_params(5, 7, 3, 4)) * 0.5
    x = rng.normal(size=(9, 5))
    t = rng.normal(size=(9, 4))
    m = (rng.random((9, 4)) > 0.3).astype(float)
    _, g = mo.loss_grad(p, shapes, x, t, m)
    h = 1e-6
    fd = np.zeros_like(p)
    for i in range(len(p)):
        e = np.zeros_like(p)
        e[i] = h
        fd[i] = (mo.loss_grad(p + e, shapes, x, t, m)[0] - mo.loss_grad(p - e, shapes, x, t, m)[0]) / (2 * h)
    assert np.allclose(g, fd, rtol=1e-6, atol=1e-9)


def test_oracle_adam_reduces_loss():
    rng = np.random.default_rng(6)
    shapes = mo.layer_shapes(2, 16, 2, 1)
    p = rng.normal(size=mo.num_params(2, 16, 2, 1)) * 0.3
    x = rng.uniform(-1, 1, size=(64, 2))
    t = np.sin(2 * x[:, :1]) * np.cos(x[:, 1:])
    m = np.ones_like(t)
    l0 = mo.loss_grad(p, shapes, x, t, m)[0]
    p2 = mo.adam_steps(p, shapes, [(x, t, m)] * 200, 1e-2)
    assert mo.loss_grad(p2, shapes, x, t, m)[0] < 0.1 * l0
