"""CPU oracle of the learned warm start's network -- test infrastructure only.

A numpy restatement of the MLP the engine trains on the tensor cores
(sovereign-solver_b200/csrc/mlp.cu): n_in -> hidden -> hidden -> n_out, ReLU,
loss L = sum (y - t)^2 / (batch n_out). It rounds to BF16 at the points where
the GPU path does (the GEMM operands: inputs, weights, hidden activations and
the back-propagated errors) and computes everything else in FP64, so the
GPU's FP32-accumulated results must match it to FP32 accumulation error.
No counterpart in the reference (its PDHG has no warm start); only the tests
use this module.
"""
from __future__ import annotations

import numpy as np


def bf16(x: np.ndarray) -> np.ndarray:
    """Round FP32 values to the nearest BF16 (ties to even), returned as FP64."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    r = ((u + 0x7FFF + lsb) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def split(params: np.ndarray, n_in: int, hidden: int, n_out: int):
    sizes = [hidden * n_in, hidden, hidden * hidden, hidden, n_out * hidden, n_out]
    out, o = [], 0
    for s in sizes:
        out.append(np.asarray(params[o:o + s], dtype=np.float64))
        o += s
    W1, b1, W2, b2, W3, b3 = out
    return (W1.reshape(hidden, n_in), b1, W2.reshape(hidden, hidden), b2,
            W3.reshape(n_out, hidden), b3)


def forward(params, x, n_in, hidden, n_out):
    W1, b1, W2, b2, W3, b3 = split(params, n_in, hidden, n_out)
    xb = bf16(x)
    h1 = bf16(np.maximum(xb @ bf16(W1).T + b1, 0.0))
    h2 = bf16(np.maximum(h1 @ bf16(W2).T + b2, 0.0))
    y = h2 @ bf16(W3).T + b3
    return xb, h1, h2, y


def gradients(params, x, t, n_in, hidden, n_out):
    """(gradient in parameter order, loss)."""
    W1, b1, W2, b2, W3, b3 = split(params, n_in, hidden, n_out)
    xb, h1, h2, y = forward(params, x, n_in, hidden, n_out)
    cnt = y.size
    d = y - np.asarray(t, dtype=np.float64)
    loss = float(np.sum(d * d) / cnt)
    dy = 2.0 * d / cnt
    dyb = bf16(dy)
    gW3 = dyb.T @ h2
    gb3 = dy.sum(axis=0)
    dz2 = (dyb @ bf16(W3)) * (h2 > 0)
    dz2b = bf16(dz2)
    gW2 = dz2b.T @ h1
    gb2 = dz2.sum(axis=0)
    dz1 = (dz2b @ bf16(W2)) * (h1 > 0)
    gW1 = bf16(dz1).T @ xb
    gb1 = dz1.sum(axis=0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return g, loss


def init_params(n_in, hidden, n_out, seed=0):
    """He-normal weights, zero biases."""
    rng = np.random.default_rng(seed)
    W1 = rng.standard_normal((hidden, n_in)) * np.sqrt(2.0 / n_in)
    W2 = rng.standard_normal((hidden, hidden)) * np.sqrt(2.0 / hidden)
    W3 = rng.standard_normal((n_out, hidden)) * np.sqrt(1.0 / hidden)
    return np.concatenate([W1.ravel(), np.zeros(hidden), W2.ravel(), np.zeros(hidden),
                           W3.ravel(), np.zeros(n_out)]).astype(np.float32)
