"""The CPU FP64 network restatement used as the checker of the tensor-core kernels: its
back-propagation agrees with central finite differences (FP64, no bf16 rounding)."""
import numpy as np

import cnn_reference as R


def test_backprop_matches_finite_differences():
    shape = (5, 4, 3)
    n = int(np.prod(shape))
    rng = np.random.default_rng(0)
    params = R.random_params(5).astype(np.float64)
    x2 = rng.standard_normal((n, 2))
    dy = rng.standard_normal(n)
    _, g = R.grad(params, x2, dy, shape, bf=False)
    def f(p):
        y, _ = R.forward(p, x2, shape, bf=False)
        return float(dy @ y)
    idx = [5, 300, R.LAYER + 17, R.LAYER + 27 * 256 + 3, 2 * R.LAYER + 999, 3 * R.LAYER + 40, 3 * R.LAYER + 27 * 256]
    for q in idx:
        h = 1e-6
        e = np.zeros_like(params); e[q] = h
        fd = (f(params + e) - f(params - e)) / (2 * h)
        assert abs(fd - g[q]) <= 1e-6 * max(1.0, abs(fd)), (q, fd, g[q])


def test_adjoint_identity():
    rng = np.random.default_rng(1)
    x = rng.standard_normal((4, 5, 6, 16))
    gy = rng.standard_normal((4, 5, 6, 16))
    W = rng.standard_normal((27, 16, 16))
    lhs = np.sum(R.conv(x, W) * gy)
    rhs = np.sum(x * R.conv_T(gy, W))
    assert abs(lhs - rhs) <= 1e-9 * abs(lhs)
