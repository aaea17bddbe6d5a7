"""The 3x3x3 convolution on the tcgen05 tensor cores against the float64
oracle (oracle/unet.py), on the BF16 values the kernel reads.

Tolerance: the kernel accumulates in FP32 and rounds its output to BF16
(a relative step of 2^-8), so every element must lie within 2^-8 of the
float64 result relative to the largest magnitude of its output channel,
plus the FP32 sum-order error."""

import numpy as np
import pytest
import torch

from oracle import unet as ref
from rexlib_b200 import prior

pytestmark = pytest.mark.gpu


def bf16(shape, rng, scale=1.0):
    return torch.from_numpy((rng.standard_normal(shape) * scale).astype(np.float32)).to(torch.bfloat16).cuda()


def host(t):
    return t.float().cpu().numpy().astype(np.float64)


def close(got, want):
    scale = np.maximum(np.abs(want).max(axis=(0, 1, 2), keepdims=True), 1e-3)
    err = np.abs(got - want) / scale
    assert err.max() <= 2.0 ** -7, err.max()


@pytest.mark.parametrize("cin,cout", [(16, 16), (16, 32), (32, 64), (64, 64), (64, 128), (128, 128), (128, 16)])
@pytest.mark.parametrize("extent", [(8, 8, 8), (16, 16, 16), (32, 32, 32), (4, 8, 256), (2, 4, 128), (4, 4, 64),
                                    (2, 8, 16), (2, 4, 32)])
def test_conv3d_matches_float64(cin, cout, extent):
    # Widths of 128 and more run the x-row kernel with its x halo; widths of
    # 16 to 64 whose height holds 128 / W rows run it without the halo for
    # up to 64 output channels; the others run the box kernel.
    rng = np.random.default_rng(cin * 1000 + cout + sum(extent))
    x = bf16(extent + (cin,), rng)
    w = bf16((cout, 27, cin), rng, 1.0 / np.sqrt(27 * cin))
    b = torch.from_numpy(rng.standard_normal(cout).astype(np.float32)).cuda()
    error = torch.zeros(1, dtype=torch.int32, device="cuda")
    (y,) = prior.conv3d([x], w, b, prior.EPILOGUE_NONE, error=error)
    torch.cuda.synchronize()
    assert int(error.item()) == 0
    close(host(y), ref.conv3d(host(x), host(w), host(b)))


@pytest.mark.parametrize("cin,cout", [(16, 16), (32, 32), (64, 64), (128, 64)])
def test_box_kernel_at_widths_the_row_kernel_takes(cin, cout, monkeypatch):
    # REXLIB_B200_CONV_BOXES sends every width to the box kernel: both
    # kernels hold to the oracle where both apply.
    monkeypatch.setenv("REXLIB_B200_CONV_BOXES", "1")
    rng = np.random.default_rng(cin + 7 * cout)
    x = bf16((4, 4, 128, cin), rng)
    w = bf16((cout, 27, cin), rng, 1.0 / np.sqrt(27 * cin))
    (y,) = prior.conv3d([x], w, None, prior.EPILOGUE_NONE)
    torch.cuda.synchronize()
    close(host(y), ref.conv3d(host(x), host(w)))


@pytest.mark.parametrize("width", [16, 128])
def test_conv3d_relu_and_two_sources_at(width):
    rng = np.random.default_rng(width)
    a = bf16((4, 8, width, 32), rng)
    s = bf16((4, 8, width, 32), rng)
    w = bf16((32, 27, 64), rng, 0.05)
    b = torch.from_numpy(rng.standard_normal(32).astype(np.float32)).cuda()
    (y,) = prior.conv3d([a, s], w, b, prior.EPILOGUE_RELU)
    torch.cuda.synchronize()
    want = ref.relu(ref.conv3d(np.concatenate([host(a), host(s)], -1), host(w), host(b)))
    close(host(y), want)


@pytest.mark.parametrize("channels", [(16, 64), (32, 16), (128, 64)])
@pytest.mark.parametrize("width", [16, 128])
def test_two_sources_of_different_widths(width, channels):
    # Sources of different channel counts concatenated: the wider source is
    # read in more chunks of the narrower one's width.
    ca, cs = channels
    rng = np.random.default_rng(40 + width + ca)
    a = bf16((4, 4, width, ca), rng)
    s = bf16((4, 4, width, cs), rng)
    w = bf16((32, 27, ca + cs), rng, 0.05)
    (y,) = prior.conv3d([a, s], w, None, prior.EPILOGUE_NONE)
    torch.cuda.synchronize()
    close(host(y), ref.conv3d(np.concatenate([host(a), host(s)], -1), host(w)))


def test_conv3d_relu_and_two_sources():
    # A decoder convolution: the upsampled and skip volumes concatenated,
    # ReLU in the epilogue.
    rng = np.random.default_rng(3)
    a = bf16((16, 16, 16, 32), rng)
    s = bf16((16, 16, 16, 32), rng)
    w = bf16((32, 27, 64), rng, 0.05)
    b = torch.from_numpy(rng.standard_normal(32).astype(np.float32)).cuda()
    (y,) = prior.conv3d([a, s], w, b, prior.EPILOGUE_RELU)
    torch.cuda.synchronize()
    want = ref.relu(ref.conv3d(np.concatenate([host(a), host(s)], -1), host(w), host(b)))
    close(host(y), want)


def test_conv3d_mask_epilogue_and_split_output():
    # The backward pass's form: the output channels split over two volumes
    # (the gradients of the two concatenated inputs), each zeroed where its
    # mask (the forward activation) is not positive.
    rng = np.random.default_rng(4)
    g = bf16((16, 16, 16, 32), rng)
    w = bf16((64, 27, 32), rng, 0.05)
    m0 = bf16((16, 16, 16, 32), rng)
    m1 = bf16((16, 16, 16, 32), rng)
    out0 = torch.empty((16, 16, 16, 32), dtype=torch.bfloat16, device="cuda")
    out1 = torch.empty_like(out0)
    prior.conv3d([g], w, None, prior.EPILOGUE_MASK, out=[out0, out1], masks=[m0, m1])
    torch.cuda.synchronize()
    full = ref.conv3d(host(g), host(w))
    close(host(out0), full[..., :32] * (host(m0) > 0))
    close(host(out1), full[..., 32:] * (host(m1) > 0))


@pytest.mark.parametrize("extent,channels", [((32, 32, 32), 64), ((8, 8, 128), 64), ((4, 8, 256), 16)])
def test_wait_that_runs_out_reports_and_leaves_the_context_usable(extent, channels):
    # Waits limited to a single test of their barrier run out at once (the
    # epilogue's first accumulator is many copies and MMAs away): the kernel
    # (box or x-row) records a nonzero error word, drains its copies and
    # MMAs, frees its tensor memory and returns. The next call on the same
    # context is exact.
    rng = np.random.default_rng(11)
    x = bf16(extent + (channels,), rng)
    w = bf16((channels, 27, channels), rng, 1.0 / np.sqrt(27 * channels))
    error = torch.zeros(1, dtype=torch.int32, device="cuda")
    prior.conv3d([x], w, None, prior.EPILOGUE_NONE, error=error, wait_limit_ns=1)
    torch.cuda.synchronize()
    assert int(error.item()) != 0
    error.zero_()
    (y,) = prior.conv3d([x], w, None, prior.EPILOGUE_NONE, error=error)
    torch.cuda.synchronize()
    assert int(error.item()) == 0
    close(host(y), ref.conv3d(host(x), host(w)))


@pytest.mark.parametrize("width", [16, 128])
def test_input_whose_voxels_hold_more_channels_than_it_reads(width):
    # A channel slice of a wider volume: input_strides counts the wider
    # rows, both kernels read only the sliced channels.
    rng = np.random.default_rng(50 + width)
    wide = bf16((4, 4, width, 48), rng)
    x = wide[..., 16:48]  # 32 channels, voxel stride 48
    w = bf16((16, 27, 32), rng, 0.05)
    (y,) = prior.conv3d([x], w, None, prior.EPILOGUE_NONE)
    torch.cuda.synchronize()
    close(host(y), ref.conv3d(host(x), host(w)))
