"""TEST INFRASTRUCTURE: the CPU oracle of the learned screen's network (tests/ only).

numpy restatement of chaos_b200/mlp.py's forward and backward passes: every operand the tensor cores read (inputs,
weights, GELU outputs, output gradients) is rounded to BF16 exactly as the device rounds it, everything else is
FP64, so the device's FP32-accumulated results must agree to accumulation-order rounding.
"""
from __future__ import annotations

import math

import numpy as np


def bf16_round(x):
    """Round to BF16 (nearest even), returned as float64."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


_K = math.sqrt(2.0 / math.pi)


def gelu(x):
    """GELU, tanh form (Hendrycks & Gimpel 2016): x (1 + tanh u) / 2 = x / (1 + exp(-2u)),
    u = sqrt(2/pi) (x + 0.044715 x^3)."""
    x = np.asarray(x, dtype=np.float64)
    with np.errstate(over="ignore"):
        return x / (1.0 + np.exp(-2.0 * _K * (x + 0.044715 * x ** 3)))


def gelu_grad(x):
    """d gelu / dx = s + x s (1 - s) 2 sqrt(2/pi) (1 + 3 0.044715 x^2), s = 1 / (1 + exp(-2u))."""
    x = np.asarray(x, dtype=np.float64)
    with np.errstate(over="ignore"):
        sg = 1.0 / (1.0 + np.exp(-2.0 * _K * (x + 0.044715 * x ** 3)))
    return sg + x * sg * (1.0 - sg) * 2.0 * _K * (1.0 + 3.0 * 0.044715 * x * x)


def forward(weights, X):
    """weights: [(W (rows x in), b)], X (B x 64). Returns outputs (B x rows_last), pre-activations, activations."""
    A = bf16_round(X)
    acts, pres = [A], []
    for li, (W, b) in enumerate(weights):
        Z = A @ bf16_round(W).T + b.astype(np.float64)
        if li == len(weights) - 1:
            acts.append(Z)
            pres.append(None)
        else:
            pres.append(Z)
            A = bf16_round(gelu(Z))
            acts.append(A)
    return acts[-1], pres, acts


def head(out, label, target, w_reg):
    """Mean BCE on column 0 + w_reg * mean squared error on column 1; returns per-row losses and dL/dout."""
    B = out.shape[0]
    z, e = out[:, 0], out[:, 1] - target
    p = 1.0 / (1.0 + np.exp(-z))
    loss = np.maximum(z, 0) - z * label + np.log1p(np.exp(-np.abs(z))) + w_reg * e * e
    g = np.zeros_like(out)
    g[:, 0] = (p - label) / B
    g[:, 1] = 2 * w_reg * e / B
    return loss, g


def backward(weights, pres, acts, gout):
    """Gradients [(dW, db)] of the loss whose output gradient is gout (FP64, BF16 where the tensor cores read)."""
    grads = [None] * len(weights)
    dZ32, dZb = gout, bf16_round(gout)
    for li in range(len(weights) - 1, -1, -1):
        W, _ = weights[li]
        grads[li] = (dZb.T @ acts[li], dZ32.sum(axis=0))
        if li == 0:
            break
        dA = dZb @ bf16_round(W)
        dZ32 = dA * gelu_grad(pres[li - 1])
        dZb = bf16_round(dZ32)
    return grads
