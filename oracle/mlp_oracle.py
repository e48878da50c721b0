"""Test infrastructure only: the conflict predictor's network (csrc/mlp.cu) restated in numpy, forward and
backward, with the same rounding points as the device:

  x, W1, W2 rounded to bf16; h1 = bf16(relu(x W1^T + b1)); h2 = bf16(relu(h1 W2^T + b2)); z = h2 . w3 + b3;
  loss = sum_b w_b BCE(z_b, y_b) / sum_b w_b;
  dz = (sigmoid(z) - y) w / sum w; dz2 = bf16(dz w3 * (h2 > 0)); dz1 = bf16((dz2 W2) * (h1 > 0));
  dW1 = dz1^T x, dW2 = dz2^T h1, db1 / db2 column sums of dz1 / dz2, dw3 = dz^T h2, db3 = sum dz.

Products accumulate in float64 here, in float32 on the device, so the comparison carries a tolerance. With
rounding=False every bf16 step is skipped and the arithmetic is float64 throughout, which the finite-difference
check of the backward formulas uses.
"""
from __future__ import annotations

import numpy as np

D0, H = 2176, 128


def bf16_bits(a: np.ndarray) -> np.ndarray:
    """float32 -> bf16 bit patterns, round to nearest even."""
    u = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) & 0xFFFF
    return r.astype(np.uint16)


def bf16_to_f32(b: np.ndarray) -> np.ndarray:
    return (np.ascontiguousarray(b, np.uint16).astype(np.uint32) << 16).view(np.float32)


def bf16(a: np.ndarray) -> np.ndarray:
    return bf16_to_f32(bf16_bits(a))


def unpack(p: np.ndarray):
    n1, n2 = H * D0, H * H
    W1 = p[:n1].reshape(H, D0)
    W2 = p[n1:n1 + n2].reshape(H, H)
    o = n1 + n2
    return W1, W2, p[o:o + H], p[o + H:o + 2 * H], p[o + 2 * H:o + 3 * H], p[o + 3 * H]


def forward_backward(p: np.ndarray, x: np.ndarray, y: np.ndarray, w: np.ndarray, rounding: bool = True):
    """x: float32 (already bf16 values when rounding). Returns (probabilities, loss, packed gradient)."""
    rnd = bf16 if rounding else (lambda a: a)
    W1, W2, b1, b2, w3, b3 = unpack(np.asarray(p, np.float64 if not rounding else np.float32))
    W1 = rnd(W1).astype(np.float64)
    W2 = rnd(W2).astype(np.float64)
    x = np.asarray(x, np.float64)
    z1 = x @ W1.T + b1
    h1 = rnd(np.maximum(z1, 0).astype(np.float32) if rounding else np.maximum(z1, 0)).astype(np.float64)
    z2 = h1 @ W2.T + b2
    h2 = rnd(np.maximum(z2, 0).astype(np.float32) if rounding else np.maximum(z2, 0)).astype(np.float64)
    z = h2 @ np.asarray(w3, np.float64) + float(b3)
    sg = 1.0 / (1.0 + np.exp(-z))
    wsum = float(np.sum(w))
    loss = float(np.sum(w * (np.maximum(z, 0) - z * y + np.log1p(np.exp(-np.abs(z))))) / wsum)
    dz = (sg - y) * w / wsum
    dw3 = dz @ h2
    db3 = dz.sum()
    dz2 = np.outer(dz, w3) * (h2 > 0)
    dz2 = rnd(dz2.astype(np.float32) if rounding else dz2).astype(np.float64)
    dW2 = dz2.T @ h1
    db2 = dz2.sum(axis=0)
    dz1 = (dz2 @ W2) * (h1 > 0)
    dz1 = rnd(dz1.astype(np.float32) if rounding else dz1).astype(np.float64)
    dW1 = dz1.T @ x
    db1 = dz1.sum(axis=0)
    g = np.concatenate([dW1.ravel(), dW2.ravel(), db1, db2, dw3, [db3]])
    return sg, loss, g
