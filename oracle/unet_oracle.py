"""CPU oracle for the learned coarse-grid preconditioner's network.

TEST INFRASTRUCTURE ONLY: the checker for the CUDA U-Net kernels
(finitevolx_b200/csrc/unet.cu).  Nothing in the package imports it.

finitevolX has no learned component, so there is no reference code to
follow; this module restates the network of the CUDA library in FP64 NumPy
and is pinned instead by a finite-difference check of its own backward pass
(tests/test_unet_oracle.py).  The forward pass rounds the weights to BF16
exactly like the device (round to nearest even) and keeps the biases in
full precision; gradients are those of that function (the straight-through
rule for the BF16 rounding), which is what the device computes.

Layout: tensors [B, C, h, w]; weights [Cout, Cin, 3, 3] flattened with the
bias after each layer's weights, layers in the order of ``LAYERS``.
"""

from __future__ import annotations

import numpy as np

DIRECT, POOL, UP = 0, 1, 2
# (cin, cout, input mode, input slot, skip slot, output slot, level, relu)
LAYERS = (
    (3, 16, DIRECT, 0, -1, 1, 0, True),
    (16, 16, POOL, 1, -1, 2, 1, True),
    (16, 32, POOL, 2, -1, 3, 2, True),
    (32, 32, POOL, 3, -1, 4, 3, True),
    (32, 32, UP, 4, 3, 5, 2, True),
    (32, 16, UP, 5, 2, 6, 1, True),
    (16, 16, UP, 6, 1, 7, 0, True),
    (16, 1, DIRECT, 7, -1, 8, 0, False),
)


def n_params() -> int:
    return sum(co * ci * 9 + co for ci, co, *_ in LAYERS)


def unpack(theta):
    """Flat parameter vector -> list of (W [Cout, Cin, 3, 3], b [Cout])."""
    out, off = [], 0
    for ci, co, *_ in LAYERS:
        W = theta[off:off + co * ci * 9].reshape(co, ci, 3, 3)
        off += co * ci * 9
        b = theta[off:off + co]
        off += co
        out.append((W, b))
    return out


def bf16_round(x):
    """FP32 -> nearest BF16 (ties to even), returned as float64."""
    u = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def transform(src, mode):
    if mode == DIRECT:
        return src
    if mode == POOL:
        return 0.25 * (src[..., 0::2, 0::2] + src[..., 1::2, 0::2] + src[..., 0::2, 1::2] + src[..., 1::2, 1::2])
    return np.repeat(np.repeat(src, 2, axis=-2), 2, axis=-1)


def transform_adjoint(d, mode):
    if mode == DIRECT:
        return d
    if mode == POOL:
        return 0.25 * np.repeat(np.repeat(d, 2, axis=-2), 2, axis=-1)
    return d[..., 0::2, 0::2] + d[..., 1::2, 0::2] + d[..., 0::2, 1::2] + d[..., 1::2, 1::2]


def conv3x3(x, W, b):
    """Zero-padded 3x3 cross-correlation: y[co] = sum W[co, ci, dy, dx] x[ci, y+dy-1, x+dx-1] + b."""
    B, C, h, w = x.shape
    xp = np.zeros((B, C, h + 2, w + 2))
    xp[:, :, 1:-1, 1:-1] = x
    y = np.zeros((B, W.shape[0], h, w))
    for dy in range(3):
        for dx in range(3):
            y += np.einsum("oc,bcyx->boyx", W[:, :, dy, dx], xp[:, :, dy:dy + h, dx:dx + w])
    return y + b[None, :, None, None]


def forward(theta, x, round_weights=True):
    """Activations of every slot (0 = x, 8 = output y)."""
    params = unpack(np.asarray(theta, np.float64))
    rnd = bf16_round if round_weights else (lambda a: a)  # noqa: E731
    acts = [None] * 9
    acts[0] = np.asarray(x, np.float64)
    for (ci, co, mode, si, sk, so, lvl, relu), (W, b) in zip(LAYERS, params):
        z = conv3x3(transform(acts[si], mode), rnd(W), b)
        if sk >= 0:
            z = z + acts[sk]
        acts[so] = np.maximum(z, 0.0) if relu else z
    return acts


def loss_and_grad(theta, x, target, round_weights=True):
    """L = sum(m (y - t)^2) / (B h w), m = channel 1 of x; returns (L, dL/dtheta, acts).

    ``round_weights=False`` drops the BF16 rounding (used to check the
    backward pass against finite differences)."""
    theta = np.asarray(theta, np.float64)
    rnd = bf16_round if round_weights else (lambda a: a)  # noqa: E731
    acts = forward(theta, x, round_weights)
    y = acts[8]
    m = acts[0][:, 1:2]
    N = y.shape[0] * y.shape[2] * y.shape[3]
    d = (y - target) * m
    L = float(np.sum(d * d) / N)
    grads = [None] * 9
    for k in range(1, 9):
        grads[k] = np.zeros_like(acts[k])
    grads[8] = 2.0 * d * m / N
    params = unpack(theta)
    gtheta = []
    for (ci, co, mode, si, sk, so, lvl, relu), (W, b) in reversed(list(zip(LAYERS, params))):
        G = grads[so] * (acts[so] > 0) if relu else grads[so]
        if sk >= 0:
            grads[sk] += G
        xin = transform(acts[si], mode)
        B, C, h, w = xin.shape
        xp = np.zeros((B, C, h + 2, w + 2))
        xp[:, :, 1:-1, 1:-1] = xin
        dW = np.zeros_like(W)
        for dy in range(3):
            for dx in range(3):
                dW[:, :, dy, dx] = np.einsum("boyx,bcyx->oc", G, xp[:, :, dy:dy + h, dx:dx + w])
        db = G.sum(axis=(0, 2, 3))
        gtheta.append(np.concatenate([dW.ravel(), db]))
        if si > 0:
            Gp = np.zeros((B, co, h + 2, w + 2))
            Gp[:, :, 1:-1, 1:-1] = G
            Wr = rnd(W)
            dxin = np.zeros_like(xin)
            for dy in range(3):
                for dx in range(3):
                    # input pixel p receives G at p - (dy - 1, dx - 1)
                    dxin += np.einsum("oc,boyx->bcyx", Wr[:, :, dy, dx], Gp[:, :, 2 - dy:2 - dy + h, 2 - dx:2 - dx + w])
            grads[si] += transform_adjoint(dxin, mode)
    return L, np.concatenate(gtheta[::-1]), acts


def adam(theta, grad, m, v, step, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
    """Kingma & Ba (2015), bias-corrected; returns new (theta, m, v)."""
    m = b1 * m + (1 - b1) * grad
    v = b2 * v + (1 - b2) * grad * grad
    mh = m / (1 - b1 ** step)
    vh = v / (1 - b2 ** step)
    return theta - lr * mh / (np.sqrt(vh) + eps), m, v


def init_params(seed=0):
    """He-uniform weights (fan-in Cin * 9), zero biases; the output layer scaled by 0.1."""
    rng = np.random.default_rng(seed)
    parts = []
    for k, (ci, co, *_rest) in enumerate(LAYERS):
        bound = np.sqrt(6.0 / (ci * 9))
        if k == len(LAYERS) - 1:
            bound *= 0.1
        parts.append(rng.uniform(-bound, bound, co * ci * 9))
        parts.append(np.zeros(co))
    return np.concatenate(parts).astype(np.float32)
