"""CPU: the network oracle's backward pass against finite differences (float64,
no rounding), so that it can serve as the GPU gradient check."""
import numpy as np

from oracle import mlp


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    theta = rng.normal(scale=0.2, size=mlp.N_PARAMS)
    X = rng.normal(size=(16, mlp.IN))
    t = rng.normal(size=16)
    loss, g = mlp.loss_grad(theta, X, t, rounding=False)
    idx = rng.choice(mlp.N_PARAMS, size=60, replace=False)
    idx = np.concatenate([idx, [mlp.N_PARAMS - 1]])  # include b4
    for i in idx:
        e = np.zeros_like(theta)
        e[i] = 1e-6
        lp, _ = mlp.loss_grad(theta + e, X, t, rounding=False)
        lm, _ = mlp.loss_grad(theta - e, X, t, rounding=False)
        fd = (lp - lm) / 2e-6
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.00390625, 1.0078125, 1.01171875, -2.5], np.float32)
    # 1 + 2^-8 is halfway between 1 and 1 + 2^-7: ties go to the even mantissa (1.0)
    assert mlp.bf16(x).tolist() == [1.0, 1.0, 1.0078125, 1.015625, -2.5]
