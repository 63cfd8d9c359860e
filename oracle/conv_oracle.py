"""FP64 CPU oracle of the surrogate's 3x3 convolutions (test infrastructure
only: the tensor-core kernels are checked against it; nothing in the product
calls it).

The reference has no convolution; these are the textbook definitions of a
3x3 "same" (zero-padded) cross-correlation and its two gradients, in float64
with numpy, on images stored channels-last. They are pinned by central finite
differences in the CPU tests.

Shapes: x (B, H, W, Cin), w (Cout, Cin, 3, 3), y / dy (B, H, W, Cout).
"""
from __future__ import annotations

import numpy as np


def _pad(x: np.ndarray) -> np.ndarray:
    return np.pad(x, ((0, 0), (1, 1), (1, 1), (0, 0)))


def conv3x3(x: np.ndarray, w: np.ndarray, bias: np.ndarray | None = None) -> np.ndarray:
    """y[b, i, j, o] = sum_{c, ky, kx} x[b, i + ky - 1, j + kx - 1, c] w[o, c, ky, kx] + bias[o]."""
    x = np.asarray(x, np.float64)
    w = np.asarray(w, np.float64)
    B, H, W, _ = x.shape
    xp = _pad(x)
    y = np.zeros((B, H, W, w.shape[0]))
    for ky in range(3):
        for kx in range(3):
            y += xp[:, ky:ky + H, kx:kx + W, :] @ w[:, :, ky, kx].T
    if bias is not None:
        y += np.asarray(bias, np.float64)
    return y


def conv3x3_dgrad(dy: np.ndarray, w: np.ndarray) -> np.ndarray:
    """dx = d(sum dy * conv3x3(x, w)) / dx."""
    dy = np.asarray(dy, np.float64)
    w = np.asarray(w, np.float64)
    B, H, W, _ = dy.shape
    dxp = np.zeros((B, H + 2, W + 2, w.shape[1]))
    for ky in range(3):
        for kx in range(3):
            dxp[:, ky:ky + H, kx:kx + W, :] += dy @ w[:, :, ky, kx]
    return dxp[:, 1:H + 1, 1:W + 1, :]


def conv3x3_wgrad(x: np.ndarray, dy: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """(dw, db) = d(sum dy * conv3x3(x, w, b)) / (w, b)."""
    x = np.asarray(x, np.float64)
    dy = np.asarray(dy, np.float64)
    B, H, W, cin = x.shape
    cout = dy.shape[-1]
    xp = _pad(x)
    dw = np.zeros((cout, cin, 3, 3))
    dyf = dy.reshape(-1, cout)
    for ky in range(3):
        for kx in range(3):
            dw[:, :, ky, kx] = dyf.T @ xp[:, ky:ky + H, kx:kx + W, :].reshape(-1, cin)
    return dw, dyf.sum(0)


def to_padded(x: np.ndarray) -> np.ndarray:
    """(B, H, W, C) -> padded channels-last (B, (H + 2) * (W + 2), C) with a zero border."""
    B, H, W, C = x.shape
    return _pad(x).reshape(B, (H + 2) * (W + 2), C)


def from_padded(xp: np.ndarray, H: int, W: int) -> np.ndarray:
    B, _, C = xp.shape
    return xp.reshape(B, H + 2, W + 2, C)[:, 1:H + 1, 1:W + 1, :]
