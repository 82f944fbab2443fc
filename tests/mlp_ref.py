"""CPU FP64 reference of the power proxy's MLP (test checker only).

Forward and backward of  y = W3 relu(W2 relu(W1 x + b1) + b2) + b3  under
mean squared error on standardised targets, mirroring where the GPU path
rounds to BF16 (weights, inputs, hidden activations and the back-propagated
activation gradients) so that the remaining difference is FP32 vs FP64
accumulation. With bf16=False it is the plain FP64 network, which the
finite-difference test checks.
"""
from __future__ import annotations

import numpy as np


def to_bf16(x: np.ndarray) -> np.ndarray:
    """Round to the nearest BF16 (ties to even) through FP32; returns FP64."""
    f = np.ascontiguousarray(x, dtype=np.float32)
    b = f.view(np.uint32).astype(np.uint64)
    b = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return (b.astype(np.uint32)).view(np.float32).astype(np.float64)


def forward_backward(P: dict, X: np.ndarray, T: np.ndarray, bf16: bool = True):
    """P: W1 [H,I], b1 [H], W2 [H,H], b2 [H], W3 [O,H], b3 [O]. X [B,I],
    T [B,O] standardised targets. Returns (loss, grads dict, Y)."""
    r = to_bf16 if bf16 else (lambda a: np.asarray(a, dtype=np.float64))
    W1, W2, W3 = r(P["W1"]), r(P["W2"]), r(P["W3"])
    b1, b2, b3 = (np.asarray(P[k], np.float64) for k in ("b1", "b2", "b3"))
    X = r(X)
    B, O = T.shape
    H1 = r(np.maximum(X @ W1.T + b1, 0.0))
    H2 = r(np.maximum(H1 @ W2.T + b2, 0.0))
    Y = H2 @ W3.T + b3
    G = Y - T
    loss = float(np.mean(G * G))
    dY = 2.0 * G / (B * O)
    db3 = dY.sum(0)
    dYb = r(dY)
    dW3 = dYb.T @ H2
    dH2 = (dYb @ W3) * (H2 > 0)
    db2 = dH2.sum(0)
    dH2b = r(dH2)
    dW2 = dH2b.T @ H1
    dH1 = (dH2b @ W2) * (H1 > 0)
    db1 = dH1.sum(0)
    dW1 = r(dH1).T @ X
    return loss, dict(W1=dW1, b1=db1, W2=dW2, b2=db2, W3=dW3, b3=db3), Y


def adam_update(p, g, m, v, t, lr, b1, b2, eps, wd=0.0, is_w=None):
    """One Adam(W) step in FP32, as the GPU kernel does it."""
    p, g, m, v = (np.asarray(a, np.float32) for a in (p, g, m, v))
    f = np.float32
    m = f(b1) * m + f(1 - b1) * g
    v = f(b2) * v + f(1 - b2) * g * g
    bc1 = f(1) - np.power(f(b1), f(t))
    bc2 = f(1) - np.power(f(b2), f(t))
    if wd > 0 and is_w is not None:
        p = np.where(is_w, p - f(lr) * f(wd) * p, p)
    p = p - f(lr) * (m / bc1) / (np.sqrt(v / bc2) + f(eps))
    return p, m, v
