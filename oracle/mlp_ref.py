"""CPU oracle (test infrastructure only) for the learned-guess network's kernels.

The reference has no learned guess, so there is no reference file to follow: this is the
plain FP64 statement of the network the GPU kernels train -- hidden layers
h_{i+1} = SiLU(h_i W_i^T + b_i), a linear output layer, and the masked squared-error loss
L = inv_count * sum mask (out - target)^2 -- with its gradients by reverse-mode
differentiation written out by hand.  The gradients are pinned by central finite
differences in the CPU tests, and the GPU kernels (BF16 operands, FP32 accumulation) are
checked against them.  Parity pinned by finite differences, not by reference outputs.
"""
from __future__ import annotations

import numpy as np


def silu(z):
    return z / (1.0 + np.exp(-z))


def silu_grad(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(X, W, b):
    """Returns the output and the per-layer (input, pre-activation) list."""
    h = np.asarray(X, dtype=np.float64)
    cache = []
    for i, (w, c) in enumerate(zip(W, b)):
        z = h @ np.asarray(w, dtype=np.float64).T + c
        cache.append((h, z))
        h = z if i == len(W) - 1 else silu(z)
    return h, cache


def loss(out, target, mask, inv_count):
    d = out - target
    return inv_count * float(np.sum(mask * d * d))


def backward(out, target, mask, inv_count, W, cache):
    """Gradients (dW list, db list) of the masked squared-error loss."""
    dY = 2.0 * inv_count * mask * (out - target)
    nl = len(W)
    gW, gb = [None] * nl, [None] * nl
    for i in range(nl - 1, -1, -1):
        h, z = cache[i]
        dz = dY if i == nl - 1 else dY * silu_grad(z)
        gW[i] = dz.T @ h
        gb[i] = dz.sum(0)
        dY = dz @ np.asarray(W[i], dtype=np.float64)
    return gW, gb


def adam_step(w, g, m1, m2, step, lr, b1=0.9, b2=0.999, eps=1e-8, wd=0.0):
    """One bias-corrected Adam update (weight decay added to the gradient), in place."""
    g = g + wd * w
    m1[...] = b1 * m1 + (1 - b1) * g
    m2[...] = b2 * m2 + (1 - b2) * g * g
    w -= lr * (m1 / (1 - b1 ** step)) / (np.sqrt(m2 / (1 - b2 ** step)) + eps)
    return w
