"""The closure MLP's CPU oracle (oracle/mlp_oracle.py) against central finite
differences, so that it can check the CUDA training gradients."""
import numpy as np

from oracle import mlp_oracle as mo


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(5)
    p = rng.normal(0, 0.3, mo.N_PARAMS)
    x = rng.normal(0, 1, (64, mo.N_IN))
    y = rng.normal(0, 1, 64)
    _, g = mo.loss_grad(p, x, y)
    h = 1e-6
    for k in rng.choice(mo.N_PARAMS, 60, replace=False):
        e = np.zeros_like(p)
        e[k] = h
        fd = (mo.loss_grad(p + e, x, y)[0] - mo.loss_grad(p - e, x, y)[0]) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 + 1e-5 * abs(fd), (k, fd, g[k])
