"""CPU oracle (test infrastructure) of the radiation surrogate's MLP: forward
and backward of the 4-layer GELU (tanh form) network in float64, with the BF16 roundings
placed where the GPU path stores BF16 (inputs, weights, hidden activations,
output and hidden gradients).  Used only by tests to check the GPU gradients.
"""

from __future__ import annotations

import math

import numpy as np


def bf16(x: np.ndarray) -> np.ndarray:
    """Round float values to bfloat16 (round to nearest even), returned as float64."""
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    rounded = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return rounded.astype(np.uint32).view(np.float32).astype(np.float64)


_C = math.sqrt(2.0 / math.pi)


def gelu(z):
    """GELU in the tanh form (Hendrycks & Gimpel 2016), exact tanh."""
    return 0.5 * z * (1.0 + np.tanh(_C * (z + 0.044715 * z ** 3)))


def gelu_grad(z):
    t = np.tanh(_C * (z + 0.044715 * z ** 3))
    return 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * _C * (1.0 + 3.0 * 0.044715 * z * z)


def forward_backward(X, T, weights, biases, loss_w, scale):
    """X [B, K_in] (BF16 values), T [B, N_out] targets, weights [(out, in)] (BF16
    values), biases, per-output loss weights; returns (Y, grads_w, grads_b)."""
    X = np.asarray(X, np.float64)
    Ws = [np.asarray(w, np.float64) for w in weights]
    bs = [np.asarray(b, np.float64) for b in biases]
    Z, H = [], [X]
    h = X
    for i in range(3):
        z = (h @ Ws[i].T + bs[i]).astype(np.float32).astype(np.float64)
        Z.append(z)
        h = bf16(gelu(z))
        H.append(h)
    Y = (h @ Ws[3].T + bs[3]).astype(np.float32).astype(np.float64)
    dY = bf16(loss_w[None, :] * 2.0 * (Y - T) * scale)
    gw, gb = [None] * 4, [None] * 4
    g = dY
    for layer in (3, 2, 1, 0):
        gw[layer] = g.T @ H[layer]
        gb[layer] = g.sum(axis=0)
        if layer > 0:
            g = bf16((g @ Ws[layer]) * gelu_grad(Z[layer - 1]))
    return Y, gw, gb
