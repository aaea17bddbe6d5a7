"""The float64 oracle of the learned prior against finite differences, on
the CPU: its convolution, pooling and transposed-convolution gradients, and
the whole network's gradient at 16^3 (the exact float64 network, no BF16
rounding). The GPU tests then hold the kernels to this oracle."""

import numpy as np
import pytest

from oracle import unet as ref


def numeric(f, x, index, h=1e-6):
    xp = x.copy()
    xm = x.copy()
    xp[index] += h
    xm[index] -= h
    return (f(xp) - f(xm)) / (2 * h)


def test_conv3d_gradients_match_finite_differences():
    rng = np.random.default_rng(1)
    x = rng.standard_normal((4, 5, 6, 3))
    w = rng.standard_normal((2, 27, 3))
    b = rng.standard_normal(2)
    g = rng.standard_normal((4, 5, 6, 2))
    dx, dw, db = ref.conv3d_backward(x, w, g)
    loss = lambda x_, w_, b_: float(np.sum(ref.conv3d(x_, w_, b_) * g))  # noqa: E731
    for idx in [(0, 0, 0, 0), (3, 4, 5, 2), (2, 1, 3, 1)]:
        assert abs(numeric(lambda v: loss(v, w, b), x, idx) - dx[idx]) < 1e-6
    for idx in [(0, 0, 0), (1, 26, 2), (1, 13, 1)]:
        assert abs(numeric(lambda v: loss(x, v, b), w, idx) - dw[idx]) < 1e-6
    assert abs(numeric(lambda v: loss(x, w, v), b, (1,)) - db[1]) < 1e-6


def test_pool_and_up_gradients_match_finite_differences():
    rng = np.random.default_rng(2)
    x = rng.standard_normal((4, 4, 4, 3))
    g = rng.standard_normal((2, 2, 2, 3))
    px = ref.pool_backward(g)
    for idx in [(0, 0, 0, 0), (3, 2, 1, 2)]:
        assert abs(numeric(lambda v: float(np.sum(ref.pool(v) * g)), x, idx) - px[idx]) < 1e-6
    w = rng.standard_normal((8, 2, 3))
    b = rng.standard_normal(2)
    gu = rng.standard_normal((8, 8, 8, 2))
    dx, dw, db = ref.up_backward(x, w, gu)
    loss = lambda x_, w_: float(np.sum(ref.up(x_, w_, b) * gu))  # noqa: E731
    assert abs(numeric(lambda v: loss(v, w), x, (1, 2, 3, 0)) - dx[1, 2, 3, 0]) < 1e-6
    assert abs(numeric(lambda v: loss(x, v), w, (5, 1, 2)) - dw[5, 1, 2]) < 1e-6
    assert np.allclose(db, gu.sum(axis=(0, 1, 2)))


@pytest.mark.parametrize("layer", [ref.FIRST, ref.E0, ref.E2A, ref.B2, ref.UP2, ref.D2A, ref.UP0, ref.D0A, ref.HEAD])
def test_network_gradient_matches_finite_differences(layer):
    rng = np.random.default_rng(3)
    params = {}
    for l in range(len(ref.LAYERS)):
        shape = ref.weight_shape(l)
        fan = np.prod(shape[1:]) if ref.LAYERS[l][0] != "up" else shape[2]
        params[l] = (rng.standard_normal(shape) * np.sqrt(2.0 / fan), rng.standard_normal(ref.LAYERS[l][3]) * 0.1)
    x = rng.standard_normal((16, 16, 16))
    target = x + 0.3 * rng.standard_normal((16, 16, 16))
    net = ref.Network(params, bf16=False)
    net.forward(x)
    _, grads = net.backward(target)

    def loss(w, b):
        p = dict(params)
        p[layer] = (w, b)
        n = ref.Network(p, bf16=False)
        n.forward(x)
        return n.backward(target)[0]

    w, b = params[layer]
    flat = np.argsort(np.abs(grads[layer][0]).ravel())[-2:]  # the largest entries: well above the FD noise
    for k in flat:
        idx = np.unravel_index(k, w.shape)
        got = numeric(lambda v: loss(v, b), w, idx, h=1e-5)
        assert abs(got - grads[layer][0][idx]) <= 1e-5 * max(1.0, abs(got)) + 1e-9, (layer, idx)
    got = numeric(lambda v: loss(w, v), b, (0,), h=1e-5)
    assert abs(got - grads[layer][1][0]) <= 1e-5 * max(1.0, abs(got)) + 1e-9
