"""float64 CPU oracle of the probe MLP (test infrastructure only).

Restates the forward pass and the gradient of the mean softmax cross-entropy
of extended-rabitq_b200/csrc/mlp.cuh: features standardised with the model's
mean/std, W1..W3 rounded to bf16 as the GPU forward pass uses them, biases in
float32, ReLU hidden layers.  The GPU gradients (FP32 accumulation) are
checked against these float64 values.
"""
from __future__ import annotations

import numpy as np

IN, HID, BINS = 320, 256, 8
W1, B1 = 0, HID * IN
W2, B2 = B1 + HID, B1 + HID + HID * HID
W3, B3 = B2 + HID, B2 + HID + BINS * HID
N_PARAMS = B3 + BINS


def to_bf16(x: np.ndarray) -> np.ndarray:
    """Round float32 to the nearest bfloat16 (ties to even), returned as float32."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def unpack(params):
    p = np.asarray(params, np.float32)
    w1 = to_bf16(p[W1:B1]).reshape(HID, IN).astype(np.float64)
    b1 = p[B1:W2].astype(np.float64)
    w2 = to_bf16(p[W2:B2]).reshape(HID, HID).astype(np.float64)
    b2 = p[B2:W3].astype(np.float64)
    w3 = to_bf16(p[W3:B3]).reshape(BINS, HID).astype(np.float64)
    b3 = p[B3:].astype(np.float64)
    return w1, b1, w2, b2, w3, b3


def probabilities(params, mean, std, features):
    """Softmax output [n, 8] of the forward pass, float64."""
    w1, b1, w2, b2, w3, b3 = unpack(params)
    x = (np.asarray(features, np.float32) - mean) / std
    x = x.astype(np.float32).astype(np.float64)
    h1 = np.maximum(x @ w1.T + b1, 0.0)
    h2 = np.maximum(h1 @ w2.T + b2, 0.0)
    z = h2 @ w3.T + b3
    z -= z.max(axis=1, keepdims=True)
    p = np.exp(z)
    return p / p.sum(axis=1, keepdims=True)


def loss_and_grads(params, mean, std, features, labels):
    w1, b1, w2, b2, w3, b3 = unpack(params)
    x = (np.asarray(features, np.float32) - mean) / std
    x = x.astype(np.float32).astype(np.float64)
    h1 = np.maximum(x @ w1.T + b1, 0.0)
    h2 = np.maximum(h1 @ w2.T + b2, 0.0)
    z = h2 @ w3.T + b3
    z -= z.max(axis=1, keepdims=True)
    p = np.exp(z)
    p /= p.sum(axis=1, keepdims=True)
    n = x.shape[0]
    y = np.asarray(labels, np.int64)
    loss = float(-np.mean(np.log(p[np.arange(n), y])))
    dz = p.copy()
    dz[np.arange(n), y] -= 1.0
    dz /= n
    g = np.zeros(N_PARAMS, np.float64)
    g[W3:B3] = (dz.T @ h2).ravel()
    g[B3:] = dz.sum(0)
    dh2 = (dz @ w3) * (h2 > 0)
    g[W2:B2] = (dh2.T @ h1).ravel()
    g[B2:W3] = dh2.sum(0)
    dh1 = (dh2 @ w2) * (h1 > 0)
    g[W1:B1] = (dh1.T @ x).ravel()
    g[B1:W2] = dh1.sum(0)
    return loss, g
