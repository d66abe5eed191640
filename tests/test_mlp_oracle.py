"""CPU: the network oracle's analytic gradient against central differences."""
import numpy as np

import mlp_oracle as M


def test_oracle_gradient_finite_differences():
    dims = [7, 9, 9, 9, 2]
    rng = np.random.default_rng(3)
    p = M.init_params(dims, seed=1) + 0.05 * rng.standard_normal(M.layout(dims)[1])
    X = rng.standard_normal((23, dims[0]))
    Y = rng.standard_normal((23, dims[-1]))
    loss, g = M.loss_and_grad(p, dims, X, Y)
    h = 1e-6
    for i in rng.choice(len(p), 60, replace=False):
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (M.loss_and_grad(pp, dims, X, Y)[0] - M.loss_and_grad(pm, dims, X, Y)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-7 + 1e-5 * abs(fd)


def test_oracle_layout_matches_flat_count():
    dims = [22, 64, 64, 64, 2]
    _, total = M.layout(dims)
    assert total == 22 * 64 + 64 + 2 * (64 * 64 + 64) + 64 * 2 + 2
