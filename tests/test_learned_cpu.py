"""CPU checks of the CDF-network restatement used to verify the GPU training
kernels: its analytic gradient against central finite differences."""
import numpy as np

from oracle import cdf_mlp as M


def test_restatement_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = rng.normal(0, 0.5, M.P)
    z = rng.standard_normal(64)
    u = rng.random(64)
    u[::7] = -1.0  # masked samples
    loss, g = M.loss_and_grad(p, z, u)
    nv = (u >= 0).sum()
    assert np.isclose(loss / nv, M.mse(p, z, u))
    idx = rng.choice(M.P, 60, replace=False)
    eps = 1e-6
    for k in idx:
        d = np.zeros(M.P)
        d[k] = eps
        num = (M.mse(p + d, z, u) - M.mse(p - d, z, u)) / (2 * eps)
        assert abs(num - g[k]) <= 1e-6 + 1e-5 * abs(num), k


def test_layout_size():
    assert M.P == 1153
