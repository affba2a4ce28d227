"""The CPU reference MLP (checker of the GPU training kernels) against finite differences."""
import numpy as np

import mlp_ref


def test_reference_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = rng.standard_normal(mlp_ref.NPARAM) * 0.2
    X = rng.uniform(-1, 1, (64, 4))
    t = rng.uniform(-1, 1, 64)
    _, g = mlp_ref.loss_and_grad(p, X, t, use_bf16=False)
    eps = 1e-6
    for i in [0, 3, 255, 300, 1000, 2222, 4415, 4420, 4470, 4500, 4544]:
        pp, pm = p.copy(), p.copy()
        pp[i] += eps
        pm[i] -= eps
        fd = (mlp_ref.loss_and_grad(pp, X, t, False)[0] - mlp_ref.loss_and_grad(pm, X, t, False)[0]) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 + 1e-6 * abs(g[i])


def test_bf16_rounding():
    v = np.array([1.0, 1.00390625, 1.001953125, -3.14159, 65504.0])
    r = mlp_ref.bf16(v)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0  # 1 + 2^-8 is a tie: rounds to even
    assert abs(r[3] + 3.140625) < 1e-12
