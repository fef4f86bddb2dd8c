"""CPU restatement of the library's per-bead network (test infrastructure only).

The network of the learned initial guess has no counterpart in the reference; this module
is the CPU check of its tensor-core kernels (forward values, loss and every parameter
gradient).  It follows the kernels' arithmetic: features, W1, W2 and the hidden
activations H1 are rounded to BF16 before each product, as are the back-propagated dZ2
and dZ1 (their bias gradients are sums of the rounded values, as the kernels form them
with a ones row); products accumulate in float64 here and in FP32 on the GPU.

Parameter vector (float32): W1[128][48], b1[128], W2[128][128], b2[128], w3[128], b3.
"""
from __future__ import annotations

import numpy as np
from scipy.special import erf

F, H = 48, 128
OFF_W1 = 0
OFF_B1 = OFF_W1 + H * F
OFF_W2 = OFF_B1 + H
OFF_B2 = OFF_W2 + H * H
OFF_W3 = OFF_B2 + H
OFF_B3 = OFF_W3 + H
NPARAM = OFF_B3 + 1


def bf16_round(a) -> np.ndarray:
    """Round float32 values to the nearest BF16 (ties to even), returned as float64."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def bf16_bits(a) -> np.ndarray:
    """BF16 bit patterns (uint16) of float values, round to nearest even."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    return (((u + 0x7FFF + ((u >> 16) & 1)) >> 16) & 0xFFFF).astype(np.uint16)


def from_bits(b) -> np.ndarray:
    return (np.asarray(b, dtype=np.uint16).astype(np.uint32) << 16).view(np.float32).astype(np.float64)


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    return (p[OFF_W1:OFF_B1].reshape(H, F), p[OFF_B1:OFF_W2], p[OFF_W2:OFF_B2].reshape(H, H), p[OFF_B2:OFF_W3],
            p[OFF_W3:OFF_B3], p[OFF_B3])


def gelu(x):
    return 0.5 * x * (1.0 + erf(x / np.sqrt(2.0)))


def gelu_grad(x):
    return 0.5 * (1.0 + erf(x / np.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / np.sqrt(2.0 * np.pi)


def forward(params, x_bits):
    """y[n] for BF16 feature rows x_bits[n][48] (uint16)."""
    W1, b1, W2, b2, w3, b3 = unpack(params)
    X = from_bits(x_bits)
    a1 = X @ bf16_round(W1).T + b1
    H1 = bf16_round(gelu(a1))
    a2 = H1 @ bf16_round(W2).T + b2
    return gelu(a2) @ w3 + b3


def loss_and_grad(params, x_bits, t, rounding=True):
    """(loss, gradient vector) of (1/n) sum (y - t)^2.  rounding=False drops the BF16
    rounding of weights and intermediates (exact float64 backpropagation, for
    finite-difference checks of the formulas)."""
    W1, b1, W2, b2, w3, b3 = unpack(params)
    n = len(t)
    X = from_bits(x_bits)
    rnd = bf16_round if rounding else (lambda a: np.asarray(a, dtype=np.float64))
    W1r, W2r = rnd(W1), rnd(W2)
    a1 = X @ W1r.T + b1
    H1 = rnd(gelu(a1))
    a2 = H1 @ W2r.T + b2
    h2 = gelu(a2)
    y = h2 @ w3 + b3
    e = y - np.asarray(t, dtype=np.float64)
    loss = float((e * e).sum() / n)
    dy = 2.0 * e / n
    dZ2 = rnd(dy[:, None] * w3[None, :] * gelu_grad(a2))
    g = np.zeros(NPARAM)
    g[OFF_W3:OFF_B3] = dy @ h2
    g[OFF_B3] = dy.sum()
    g[OFF_W2:OFF_B2] = (dZ2.T @ H1).ravel()
    g[OFF_B2:OFF_W3] = dZ2.sum(0)
    dH1 = dZ2 @ W2r
    dZ1 = rnd(dH1 * gelu_grad(a1))
    g[OFF_W1:OFF_B1] = (dZ1.T @ X).ravel()
    g[OFF_B1:OFF_W2] = dZ1.sum(0)
    return loss, g
