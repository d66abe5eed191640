"""GPU: the chooser network's CUDA kernels against the FP64 numpy oracle, and
what the trained chooser gains over the fixed setting."""
import numpy as np
import pytest

import mlp_oracle as M

pytestmark = pytest.mark.gpu

DIMS = [22, 64, 64, 64, 2]


def test_forward_and_gradients_match_oracle(ctx):
    ctx.mlp_create(22, 64, 3, 2, seed=7)
    p = ctx.mlp_params().astype(np.float64)
    rng = np.random.default_rng(1)
    X = rng.standard_normal((300, 22)).astype(np.float32)
    Y = rng.standard_normal((300, 2)).astype(np.float32)
    yo, _ = M.forward(p, DIMS, X)
    yg = ctx.mlp_forward(X)
    assert np.max(np.abs(yg - yo)) <= 1e-4 * max(1.0, np.max(np.abs(yo)))
    g, loss = ctx.mlp_gradients(X, Y)
    lo, go = M.loss_and_grad(p, DIMS, X, Y)
    assert abs(loss - lo) <= 1e-5 * abs(lo)
    # FP32 kernels vs FP64 oracle: relative error of the whole gradient vector
    assert np.linalg.norm(g - go) <= 1e-4 * np.linalg.norm(go)
    assert np.max(np.abs(g - go)) <= 1e-3 * np.max(np.abs(go))


def test_training_fits_a_smooth_map(ctx):
    rng = np.random.default_rng(2)
    X = rng.uniform(-1, 1, (2000, 22)).astype(np.float32)
    Y = np.stack([np.sin(X[:, 0] * 2) + X[:, 1] * X[:, 2], np.cos(X[:, 3]) - X[:, 4]],
                 axis=1).astype(np.float32)
    ctx.mlp_create(22, 64, 3, 2, seed=3)
    hist = ctx.mlp_train(X, Y, epochs=120, batch=64, lr=2e-3, seed=0)
    assert hist[-1] < 0.1 * hist[0]
    assert hist[-1] < 0.02


def test_learned_chooser_against_fixed_setting(tb):
    """Held-out seeded systems with random tolerances in [1e-7, 1e-3]: the
    learned choice meets the tolerance far more often than the fixed P=10,
    theta=0.4, ncrit=64 setting, and where both meet it the learned choice is
    faster than the fixed FP64 form."""
    from tapas_reduce_b200 import chooser, train_chooser
    if not chooser.MODEL_PATH.exists():
        pytest.skip("no trained chooser model in the package")
    summary, recs = train_chooser.evaluate(n_systems=30, seed_base=95_000, targets=128)
    assert summary["hit_rate_learned"] >= 0.8
    assert summary["hit_rate_learned"] >= summary["hit_rate_fixed_fp64"] + 0.15
    assert summary["n_both_meet"] >= 5
    assert summary["geomean_speedup_vs_fixed_fp64_where_both_meet"] > 1.0
