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


# --------------------------------------------------------------------------
# The whole network (rexlib_b200/csrc/unet.cu's architecture)

# (kind, input channels a, input channels b, output channels), encoder to decoder.
LAYERS = [
    ("first", 1, 0, 16), ("conv", 16, 0, 16), ("conv", 16, 0, 32), ("conv", 32, 0, 32), ("conv", 32, 0, 64),
    ("conv", 64, 0, 64), ("conv", 64, 0, 128), ("conv", 128, 0, 128), ("up", 128, 0, 64), ("conv", 64, 64, 64),
    ("conv", 64, 0, 64), ("up", 64, 0, 32), ("conv", 32, 32, 32), ("conv", 32, 0, 32), ("up", 32, 0, 16),
    ("conv", 16, 16, 16), ("conv", 16, 0, 16), ("head", 16, 0, 1),
]
(FIRST, E0, E1A, E1, E2A, E2, B1, B2, UP2, D2A, D2, UP1, D1A, D1, UP0, D0A, D0, HEAD) = range(18)


def weight_shape(layer):
    kind, ca, cb, co = LAYERS[layer]
    if kind == "first":
        return (co, 27)
    if kind == "conv":
        return (co, 27, ca + cb)
    if kind == "up":
        return (8, co, ca)
    return (ca,)


def to_bf16(x):
    """Round to the nearest BF16 (ties to even), kept in float64."""
    f = np.asarray(x, np.float32)
    bits = f.view(np.uint32).astype(np.uint64)
    rounded = ((bits + 0x7FFF + ((bits >> 16) & 1)) >> 16) << 16
    out = rounded.astype(np.uint32).view(np.float32).astype(np.float64)
    return np.where(np.isfinite(f), out, f.astype(np.float64))


class Network:
    """params: {layer: (weights, bias)} in float64. bf16=True rounds what the
    GPU stores in BF16 (activations, their gradients, the tensor-core
    convolutions' weights) at the same points; False is the exact float64
    network."""

    def __init__(self, params, bf16=True):
        self.p = params
        self.r = to_bf16 if bf16 else (lambda a: np.asarray(a, np.float64))

    def _w(self, layer):
        w, b = self.p[layer]
        return (self.r(w) if LAYERS[layer][0] == "conv" else w), b

    def forward(self, x):
        r, a = self.r, {}
        self.x = np.asarray(x, np.float64)
        w, b = self.p[FIRST]
        a[FIRST] = r(relu(conv3d(self.x[..., None], w[:, :, None], b)))
        conv = lambda l, *ins: r(relu(conv3d(np.concatenate(ins, -1), *self._w(l))))  # noqa: E731
        a[E0] = conv(E0, a[FIRST])
        self.pools = [r(pool(a[E0]))]
        a[E1A] = conv(E1A, self.pools[0])
        a[E1] = conv(E1, a[E1A])
        self.pools.append(r(pool(a[E1])))
        a[E2A] = conv(E2A, self.pools[1])
        a[E2] = conv(E2, a[E2A])
        self.pools.append(r(pool(a[E2])))
        a[B1] = conv(B1, self.pools[2])
        a[B2] = conv(B2, a[B1])
        a[UP2] = r(up(a[B2], *self.p[UP2]))
        a[D2A] = conv(D2A, a[UP2], a[E2])
        a[D2] = conv(D2, a[D2A])
        a[UP1] = r(up(a[D2], *self.p[UP1]))
        a[D1A] = conv(D1A, a[UP1], a[E1])
        a[D1] = conv(D1, a[D1A])
        a[UP0] = r(up(a[D1], *self.p[UP0]))
        a[D0A] = conv(D0A, a[UP0], a[E0])
        a[D0] = conv(D0, a[D0A])
        w, b = self.p[HEAD]
        self.a = a
        self.y = self.x + a[D0] @ w + b[0]
        return self.y

    def backward(self, target):
        """(loss, {layer: (dw, db)}) of 0.5 mean (y - target)^2."""
        r, a, g = self.r, self.a, {}
        V = self.y.size
        diff = self.y - target
        loss = 0.5 * np.sum(diff * diff) / V
        gy = diff / V
        grads = {}
        w, _ = self.p[HEAD]
        grads[HEAD] = (np.einsum("zyx,zyxi->i", gy, a[D0]), np.array([gy.sum()]))
        g[D0] = r((a[D0] > 0) * (gy[..., None] * w))

        def conv_back(l, dz, *ins):
            w, _ = self._w(l)
            dx, dw, db = conv3d_backward(np.concatenate(ins, -1), w, dz)
            grads[l] = (dw, db)
            return dx

        def up_back(l, x, dz):
            dx, dw, db = up_backward(x, self.p[l][0], dz)
            grads[l] = (dw, db)
            return r((x > 0) * dx)

        g[D0A] = r((a[D0A] > 0) * conv_back(D0, g[D0], a[D0A]))
        dx = conv_back(D0A, g[D0A], a[UP0], a[E0])
        g[UP0], skip0 = r(dx[..., :16]), r((a[E0] > 0) * dx[..., 16:])
        g[D1] = up_back(UP0, a[D1], g[UP0])
        g[D1A] = r((a[D1A] > 0) * conv_back(D1, g[D1], a[D1A]))
        dx = conv_back(D1A, g[D1A], a[UP1], a[E1])
        g[UP1], skip1 = r(dx[..., :32]), r((a[E1] > 0) * dx[..., 32:])
        g[D2] = up_back(UP1, a[D2], g[UP1])
        g[D2A] = r((a[D2A] > 0) * conv_back(D2, g[D2], a[D2A]))
        dx = conv_back(D2A, g[D2A], a[UP2], a[E2])
        g[UP2], skip2 = r(dx[..., :64]), r((a[E2] > 0) * dx[..., 64:])
        g[B2] = up_back(UP2, a[B2], g[UP2])
        g[B1] = r((a[B1] > 0) * conv_back(B2, g[B2], a[B1]))
        gp2 = r(conv_back(B1, g[B1], self.pools[2]))
        g[E2] = r((a[E2] > 0) * (skip2 + pool_backward(gp2)))
        g[E2A] = r((a[E2A] > 0) * conv_back(E2, g[E2], a[E2A]))
        gp1 = r(conv_back(E2A, g[E2A], self.pools[1]))
        g[E1] = r((a[E1] > 0) * (skip1 + pool_backward(gp1)))
        g[E1A] = r((a[E1A] > 0) * conv_back(E1, g[E1], a[E1A]))
        gp0 = r(conv_back(E1A, g[E1A], self.pools[0]))
        g[E0] = r((a[E0] > 0) * (skip0 + pool_backward(gp0)))
        g[FIRST] = r((a[FIRST] > 0) * conv_back(E0, g[E0], a[FIRST]))
        w, _ = self.p[FIRST]
        _, dw, db = conv3d_backward(self.x[..., None], w[:, :, None], g[FIRST])
        grads[FIRST] = (dw[:, :, 0], db)
        self.g = g
        return loss, grads


def unpack(flat, offsets):
    """{layer: (weights, bias)} from a flat parameter vector and each
    layer's (weight offset, bias offset)."""
    out = {}
    for layer, (wo, bo) in offsets.items():
        shape = weight_shape(layer)
        out[layer] = (np.asarray(flat[wo:wo + int(np.prod(shape))], np.float64).reshape(shape),
                      np.asarray(flat[bo:bo + LAYERS[layer][3]], np.float64))
    return out
