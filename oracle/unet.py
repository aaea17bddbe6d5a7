"""Oracle of the learned prior: the 3D U-Net's operations in float64 numpy.

TEST INFRASTRUCTURE ONLY: tests use it as the checker of the GPU kernels;
the product never imports it. The reference (rexlib) has no learned
component, so there is no reference code to follow and nothing to pin it
against but the mathematics: these are the textbook definitions (a 3x3x3
convolution with zero padding 1, its gradients, 2x2x2 mean pooling, a 2x2x2
stride-2 transposed convolution, ReLU, the mean squared error), checked
against finite differences in tests/test_prior_oracle.py.

Layout: volumes (D, H, W, C) channels last; 3x3x3 weights (C_out, 27, C_in)
with tap t = (dz * 3 + dy) * 3 + dx; transposed-convolution weights
(8, C_out, C_in) with sub-position s = (a * 2 + b) * 2 + c.
"""

from __future__ import annotations

import numpy as np

TAPS = [(dz, dy, dx) for dz in range(3) for dy in range(3) for dx in range(3)]


def conv3d(x: np.ndarray, w: np.ndarray, bias: np.ndarray | None = None) -> np.ndarray:
    """out[v, o] = bias[o] + sum_t sum_i x[v + t - 1, i] w[o, t, i]."""
    D, H, W, _ = x.shape
    xp = np.pad(np.asarray(x, np.float64), ((1, 1), (1, 1), (1, 1), (0, 0)))
    w = np.asarray(w, np.float64)
    out = np.zeros((D, H, W, w.shape[0]))
    for t, (dz, dy, dx) in enumerate(TAPS):
        out += xp[dz:dz + D, dy:dy + H, dx:dx + W] @ w[:, t, :].T
    if bias is not None:
        out += np.asarray(bias, np.float64)
    return out


def conv3d_backward(x: np.ndarray, w: np.ndarray, g: np.ndarray):
    """Gradients of conv3d: (dx, dw, dbias) for the output gradient g."""
    D, H, W, _ = x.shape
    xp = np.pad(np.asarray(x, np.float64), ((1, 1), (1, 1), (1, 1), (0, 0)))
    w = np.asarray(w, np.float64)
    g = np.asarray(g, np.float64)
    dxp = np.zeros_like(xp)
    dw = np.zeros_like(w)
    for t, (dz, dy, dx) in enumerate(TAPS):
        window = xp[dz:dz + D, dy:dy + H, dx:dx + W]
        dw[:, t, :] = np.einsum("zyxo,zyxi->oi", g, window)
        dxp[dz:dz + D, dy:dy + H, dx:dx + W] += g @ w[:, t, :]
    return dxp[1:-1, 1:-1, 1:-1], dw, g.sum(axis=(0, 1, 2))


def relu(x):
    return np.maximum(x, 0.0)


def pool(x: np.ndarray) -> np.ndarray:
    """2x2x2 mean."""
    D, H, W, C = x.shape
    return np.asarray(x, np.float64).reshape(D // 2, 2, H // 2, 2, W // 2, 2, C).mean(axis=(1, 3, 5))


def pool_backward(g: np.ndarray) -> np.ndarray:
    return np.repeat(np.repeat(np.repeat(np.asarray(g, np.float64), 2, 0), 2, 1), 2, 2) / 8.0


def up(x: np.ndarray, w: np.ndarray, bias: np.ndarray | None = None) -> np.ndarray:
    """2x2x2 stride-2 transposed convolution: out[2v + s, o] = bias[o] +
    sum_i x[v, i] w[s, o, i]."""
    D, H, W, _ = x.shape
    w = np.asarray(w, np.float64)
    out = np.zeros((2 * D, 2 * H, 2 * W, w.shape[1]))
    x = np.asarray(x, np.float64)
    for s in range(8):
        a, b, c = s // 4, (s // 2) % 2, s % 2
        out[a::2, b::2, c::2] = x @ w[s].T
    if bias is not None:
        out += np.asarray(bias, np.float64)
    return out


def up_backward(x: np.ndarray, w: np.ndarray, g: np.ndarray):
    w = np.asarray(w, np.float64)
    x = np.asarray(x, np.float64)
    g = np.asarray(g, np.float64)
    dx = np.zeros_like(x)
    dw = np.zeros_like(w)
    for s in range(8):
        a, b, c = s // 4, (s // 2) % 2, s % 2
        gs = g[a::2, b::2, c::2]
        dx += gs @ w[s]
        dw[s] = np.einsum("zyxo,zyxi->oi", gs, x)
    return dx, dw, g.sum(axis=(0, 1, 2))
