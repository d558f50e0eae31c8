"""CPU checks of the U-Net oracle: its backward pass against central finite
differences of its forward pass (FP64, BF16 rounding off), its BF16 rounding
against torch's, and Adam against the textbook update."""

import numpy as np
import torch

import oracle.unet_oracle as U


def _case(seed=0, B=2, h=16, w=16):
    rng = np.random.default_rng(seed)
    theta = U.init_params(seed).astype(np.float64)
    theta[-1] = 0.05  # non-zero output bias
    x = rng.standard_normal((B, 3, h, w))
    x[:, 1] = (rng.random((B, h, w)) > 0.2).astype(np.float64)  # mask channel
    t = rng.standard_normal((B, 1, h, w))
    return theta, x, t


def test_backward_matches_finite_differences():
    theta, x, t = _case()
    L, g, _ = U.loss_and_grad(theta, x, t, round_weights=False)
    rng = np.random.default_rng(1)
    # every bias and a spread of weights, across all eight layers
    idx = np.unique(np.concatenate([rng.choice(theta.size, 60, replace=False),
                                    np.cumsum([co * ci * 9 + co for ci, co, *_ in U.LAYERS]) - 1]))
    h = 1e-6
    for k in idx:
        tp = theta.copy(); tp[k] += h
        tm = theta.copy(); tm[k] -= h
        fd = (U.loss_and_grad(tp, x, t, False)[0] - U.loss_and_grad(tm, x, t, False)[0]) / (2 * h)
        assert abs(fd - g[k]) <= 1e-6 * max(1.0, abs(g).max()), (k, fd, g[k])


def test_bf16_rounding_matches_torch():
    v = np.random.default_rng(4).standard_normal(10000).astype(np.float32) * 3
    ref = torch.from_numpy(v).to(torch.bfloat16).to(torch.float64).numpy()
    np.testing.assert_array_equal(U.bf16_round(v), ref)


def test_adam_textbook():
    th = np.array([1.0, -2.0]); g = np.array([0.5, -0.1])
    m = np.zeros(2); v = np.zeros(2)
    th1, m1, v1 = U.adam(th, g, m, v, 1, lr=0.01)
    # first bias-corrected step moves every weight by lr * sign(g)
    np.testing.assert_allclose(th1, th - 0.01 * np.sign(g), rtol=1e-6)


def test_param_count():
    assert U.n_params() == 32993
