"""The indicator network's CPU oracle checked against finite differences
(without the BF16 rounding, whose straight-through gradient has no finite
difference to compare with) and its BF16 rounding against torch's."""
import numpy as np
import torch

import mlp_oracle


def test_bf16_rounding_matches_torch():
    rng = np.random.Generator(np.random.PCG64(1))
    a = (rng.standard_normal(10000) * 10.0 ** rng.uniform(-5, 5, 10000)).astype(np.float32)
    a[:4] = [1.00390625, 1.01171875, -2.0078125, 0.0]  # ties
    assert np.array_equal(mlp_oracle.bf16(a), torch.tensor(a).bfloat16().float().numpy())


def test_gradient_matches_finite_differences():
    rng = np.random.Generator(np.random.PCG64(2))
    F = 16
    n = 20
    o = mlp_oracle.shape(F)
    params = (0.3 * rng.standard_normal(o["count"])).astype(np.float64)
    x = rng.standard_normal((n, F)).astype(np.float32)
    y = (rng.uniform(size=n) < 0.3).astype(np.float64)
    loss, grad = mlp_oracle.loss_and_gradient(params, x, y, 3.0, rounding=False)
    for i in rng.choice(o["count"], 40, replace=False):
        h = 1e-3
        p1, p2 = params.copy(), params.copy()
        p1[i] += h
        p2[i] -= h
        # forward() works in float32 inputs but float64 arithmetic
        l1, _ = mlp_oracle.loss_and_gradient(p1.astype(np.float32), x, y, 3.0, rounding=False)
        l2, _ = mlp_oracle.loss_and_gradient(p2.astype(np.float32), x, y, 3.0, rounding=False)
        fd = (l1 - l2) / (np.float32(params[i] + h) - np.float32(params[i] - h))
        assert abs(fd - grad[i]) <= 2e-3 * max(1.0, abs(grad[i])), (i, fd, grad[i])
