"""CPU test of the float64 selector-network oracle: its analytic gradient
against central finite differences."""
import numpy as np

from oracle import mlp_oracle as M


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = M.init_params(1).astype(np.float64)
    p += rng.normal(0, 0.05, size=p.shape)  # non-zero biases too
    X = rng.random((12, M.D_IN))
    Y = rng.normal(0, 1, (12, M.D_OUT))
    Mk = (rng.random((12, M.D_OUT)) > 0.2).astype(np.float64)
    loss, g = M.loss_and_grad(p, X, Y, Mk)
    eps = 1e-6
    for idx in rng.choice(len(p), 60, replace=False):
        q = p.copy(); q[idx] += eps
        lp, _ = M.loss_and_grad(q, X, Y, Mk)
        q[idx] -= 2 * eps
        lm, _ = M.loss_and_grad(q, X, Y, Mk)
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g[idx]) <= 1e-6 + 1e-4 * abs(fd), (idx, fd, g[idx])
    assert loss > 0
