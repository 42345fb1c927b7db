"""The MLP oracle's backward pass against central finite differences of its own forward pass
(float64, no bfloat16 rounding): the formulas the GPU kernels are checked against are right."""
import numpy as np

import mlp_oracle as MO


def test_oracle_gradient_matches_finite_differences():
    dims = [7, 12, 9, 5]
    rng = np.random.default_rng(3)
    p = MO.init_params(dims, seed=1).astype(np.float64)
    X = rng.standard_normal((11, dims[0]))
    T = rng.standard_normal((11, dims[-1]))
    loss, g = MO.loss_grad(p, dims, X, T, rounding=False)
    h = 1e-6
    for k in rng.choice(p.size, 40, replace=False):
        e = np.zeros_like(p)
        e[k] = h
        lp = MO.loss_grad(p + e, dims, X, T, rounding=False)[0]
        lm = MO.loss_grad(p - e, dims, X, T, rounding=False)[0]
        assert abs((lp - lm) / (2 * h) - g[k]) <= 1e-6 * max(1.0, abs(g[k]))


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 65504.0], dtype=np.float32)
    r = MO.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0           # halfway between 1 and 1.0078125: ties to even
    assert r[2] == np.float32(1.0078125)
    assert abs(r[3] - x[3]) <= 2 ** -7 * abs(x[3])
