"""The CNN oracle's own backward pass against central finite differences of its FP64
forward pass (the oracle is then the checker of the CUDA kernels, test_gpu_cnn.py)."""
import numpy as np

import cnn_oracle as co


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    n = 2
    theta = rng.standard_normal(co.nparams()) * 0.2
    x = rng.standard_normal((n, 400, 2))
    t = rng.standard_normal((n, 256))
    loss, g = co.gradients(x, t, theta, bf16=False)
    idx = rng.choice(co.nparams(), 40, replace=False)
    # always probe some biases and the first and last layers
    sl = co.layer_slices()
    idx = np.concatenate([idx, [sl[0][0][0], sl[0][1][0], sl[-1][0][0], sl[-1][1][0], sl[2][1][0] + 5]])
    eps = 1e-6
    for i in idx:
        tp, tm = theta.copy(), theta.copy()
        tp[i] += eps
        tm[i] -= eps
        fd = (co.gradients(x, t, tp, bf16=False)[0] - co.gradients(x, t, tm, bf16=False)[0]) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-5 * max(1.0, abs(fd)), (i, fd, g[i])


def test_bf16_rounding_is_nearest_even():
    v = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 3.0e38])
    r = co.bf16_round(v)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2 ** -7 and r[3] == -2.5


def test_oracle_residual_loss_gradient():
    rng = np.random.default_rng(1)
    n = 2
    theta = rng.standard_normal(co.nparams()) * 0.2
    x = rng.standard_normal((n, 400, 2))
    t = rng.standard_normal((n, 256))
    ir0 = np.array([0, 48])
    loss, g = co.gradients(x, t, theta, bf16=False, ir0=ir0, lam=0.7)
    idx = rng.choice(co.nparams(), 25, replace=False)
    eps = 1e-6
    for i in idx:
        tp, tm = theta.copy(), theta.copy()
        tp[i] += eps
        tm[i] -= eps
        fp = co.gradients(x, t, tp, bf16=False, ir0=ir0, lam=0.7)[0]
        fm = co.gradients(x, t, tm, bf16=False, ir0=ir0, lam=0.7)[0]
        fd = (fp - fm) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-5 * max(1.0, abs(fd)), (i, fd, g[i])
