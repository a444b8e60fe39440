"""CPU oracle of the tensor-core MLP (test infrastructure only).

A NumPy restatement of the forward pass, mean-squared-error loss and
backward pass that the library's BF16 tensor-core kernels compute
(include/hexmlp.h): products accumulate in float64 here, and values are
rounded to bfloat16 exactly where the kernels store bf16 (inputs, weights,
pre-activations Z, activations H, output and hidden gradients).  The
learned corrector has no counterpart in the reference, so this oracle is
pinned by calculus (finite differences in the tests), not by reference
vectors.
"""

from __future__ import annotations

import math

import numpy as np


def bf16(x: np.ndarray) -> np.ndarray:
    """Round float32 values to bfloat16 (round to nearest even), returned as float32."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((u >> 16) & 1) + 0x7FFF
    out = (((u + r) >> 16) << 16).astype(np.uint32)
    return out.view(np.float32)


GELU_C = math.sqrt(2.0 / math.pi)
GELU_A = 0.044715


def gelu(x):
    """GELU in its tanh form (the kernels evaluate tanh with the hardware
    approximation, relative error about 2^-11, below bf16 resolution)."""
    x = np.asarray(x, dtype=np.float64)
    return 0.5 * x * (1.0 + np.tanh(GELU_C * (x + GELU_A * x ** 3)))


def gelu_grad(x):
    x = np.asarray(x, dtype=np.float64)
    t = np.tanh(GELU_C * (x + GELU_A * x ** 3))
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * GELU_C * (1.0 + 3.0 * GELU_A * x * x)


def forward(weights, biases, X):
    """weights[i]: float32 [out][in] (bf16-rounded as the GEMMs read them);
    returns (Y float64, Z list, H list) with Z and H rounded to bf16."""
    a = bf16(X).astype(np.float64)
    Zs, Hs = [], []
    for W, b in zip(weights[:-1], biases[:-1]):
        z = a @ bf16(W).astype(np.float64).T + b
        zb = bf16(z.astype(np.float32)).astype(np.float64)
        h = bf16(gelu(z).astype(np.float32)).astype(np.float64)
        Zs.append(zb)
        Hs.append(h)
        a = h
    Y = a @ bf16(weights[-1]).astype(np.float64).T + biases[-1]
    return Y, Zs, Hs


def gradients(weights, biases, X, T, m_valid: int, n_valid: int):
    """Loss (summed squared error) and gradients of mean((Y - T)^2) over
    rows < m_valid and outputs < n_valid."""
    Y, Zs, Hs = forward(weights, biases, X)
    diff = np.zeros_like(Y)
    diff[:m_valid, :n_valid] = Y[:m_valid, :n_valid] - T[:m_valid, :n_valid]
    loss = float(np.sum(diff.astype(np.float32) ** 2))
    scale = 1.0 / (m_valid * n_valid)
    d = bf16((2.0 * diff * scale).astype(np.float32)).astype(np.float64)
    acts = [bf16(X).astype(np.float64)] + Hs
    gw, gb = [None] * len(weights), [None] * len(weights)
    for i in range(len(weights) - 1, -1, -1):
        gw[i] = d.T @ acts[i]
        gb[i] = d.sum(axis=0)
        if i > 0:
            dh = d @ bf16(weights[i]).astype(np.float64)
            d = bf16((dh * gelu_grad(Zs[i - 1])).astype(np.float32)).astype(np.float64)
    return loss, gw, gb
