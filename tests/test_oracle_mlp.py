"""The NumPy surrogate oracle is itself checked: analytic gradient equals
central finite differences (CPU)."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import mlp_oracle  # noqa: E402


def test_oracle_gradient_finite_differences():
    rng = np.random.default_rng(0)
    npar = 64 * 3 + 64 + 64 * 64 + 64 + 2 * 64 + 2
    p = rng.normal(scale=0.2, size=npar)
    x = np.column_stack([rng.uniform(-5.5, 3.1, 64), rng.uniform(0, 2, 64), rng.integers(0, 2, 64)])
    t = rng.normal(size=(64, 2))
    loss, g = mlp_oracle.loss_grad(p, x, t)
    for k in rng.choice(npar, 40, replace=False):
        h = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[k] += h
        pm[k] -= h
        fd = (mlp_oracle.loss_grad(pp, x, t)[0] - mlp_oracle.loss_grad(pm, x, t)[0]) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(fd))
