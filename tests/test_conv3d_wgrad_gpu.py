"""The convolution's weight and bias gradients on the tcgen05 tensor cores
against the float64 oracle (oracle/unet.py `conv3d_backward`), on the BF16
values the kernel reads.

Tolerance: the products of two BF16 values are exact in FP32 and the kernel
sums them in FP32 (tensor memory, then FP32 reductions over CTAs), so the
largest error is a few FP32 rounding steps of the partial sums: every
element within 1e-5 of the largest magnitude of the gradient."""

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


def close(got, want, tol=1e-5):
    err = np.abs(got - want).max() / max(np.abs(want).max(), 1e-30)
    assert err <= tol, err


def gradients(inputs, g, bias=True):
    cout = g.shape[3]
    cin = sum(t.shape[3] for t in inputs)
    dw = torch.zeros((cout, 27, cin), dtype=torch.float32, device="cuda")
    db = torch.zeros(cout, dtype=torch.float32, device="cuda") if bias else None
    prior.conv3d_wgrad(inputs, g, dw, db)
    torch.cuda.synchronize()
    return dw, db


def expected(inputs, g):
    x = np.concatenate([host(t) for t in inputs], -1)
    cout, cin = g.shape[3], x.shape[3]
    _, dw, db = ref.conv3d_backward(x, np.zeros((cout, 27, cin)), host(g))
    return dw, db


@pytest.mark.parametrize("cin,cout", [(16, 16), (16, 32), (32, 32), (32, 64), (64, 64), (64, 128), (128, 16),
                                      (256, 32)])
@pytest.mark.parametrize("extent", [(4, 4, 16), (4, 8, 32), (4, 4, 64), (2, 4, 128), (2, 2, 256)])
def test_weight_grad_matches_float64(cin, cout, extent):
    # Input chunks of 32 channels where the output chunk is 32 or fewer,
    # of 16 otherwise; output chunks of up to 64; segments of up to 128
    # voxels (two a row at width 256).
    rng = np.random.default_rng(cin * 7 + cout + extent[2])
    x = bf16(extent + (cin,), rng)
    g = bf16(extent + (cout,), rng)
    dw, db = gradients([x], g)
    want_w, want_b = expected([x], g)
    close(dw.cpu().numpy(), want_w)
    close(db.cpu().numpy(), want_b)


@pytest.mark.parametrize("extent", [(16, 16, 16), (8, 32, 32), (16, 4, 128)])
def test_weight_grad_over_many_segments(extent):
    # More segments than CTAs: each CTA sums a range of them in tensor memory.
    rng = np.random.default_rng(extent[0])
    x = bf16(extent + (16,), rng)
    g = bf16(extent + (16,), rng)
    dw, db = gradients([x], g)
    want_w, want_b = expected([x], g)
    close(dw.cpu().numpy(), want_w)
    close(db.cpu().numpy(), want_b)


@pytest.mark.parametrize("channels", [(16, 16), (32, 32), (32, 16), (64, 64), (128, 64)])
@pytest.mark.parametrize("width", [16, 128])
def test_weight_grad_of_two_sources(channels, width):
    # A decoder convolution's two inputs, concatenated in the weights.
    ca, cs = channels
    rng = np.random.default_rng(ca + 3 * cs + width)
    a = bf16((4, 4, width, ca), rng)
    s = bf16((4, 4, width, cs), rng)
    g = bf16((4, 4, width, 32), rng)
    dw, db = gradients([a, s], g)
    want_w, want_b = expected([a, s], g)
    close(dw.cpu().numpy(), want_w)
    close(db.cpu().numpy(), want_b)


def test_weight_grad_adds_to_what_the_arrays_hold_and_takes_sliced_inputs():
    rng = np.random.default_rng(8)
    wide = bf16((4, 4, 32, 48), rng)
    x = wide[..., 16:48]  # 32 channels, voxel stride 48
    g = bf16((4, 4, 32, 16), rng)
    dw = torch.from_numpy(rng.standard_normal((16, 27, 32)).astype(np.float32)).cuda()
    db = torch.from_numpy(rng.standard_normal(16).astype(np.float32)).cuda()
    dw0, db0 = dw.cpu().numpy().astype(np.float64), db.cpu().numpy().astype(np.float64)
    prior.conv3d_wgrad([x], g, dw)  # no bias gradient
    prior.conv3d_wgrad([x], g, dw, db)
    torch.cuda.synchronize()
    want_w, want_b = expected([x], g)
    close(dw.cpu().numpy(), dw0 + 2 * want_w)
    close(db.cpu().numpy(), db0 + want_b)


def test_weight_grad_refuses_narrow_volumes():
    rng = np.random.default_rng(1)
    x = bf16((8, 8, 8, 16), rng)
    g = bf16((8, 8, 8, 16), rng)
    dw = torch.zeros((16, 27, 16), dtype=torch.float32, device="cuda")
    with pytest.raises(Exception, match="width"):
        prior.conv3d_wgrad([x], g, dw)


def test_weight_grad_wait_that_runs_out_reports_and_leaves_the_context_usable():
    # Waits limited to a single test of their barrier run out at once: the
    # kernel records a nonzero error word, drains its copies and MMAs, frees
    # its tensor memory and returns. The next call is exact.
    rng = np.random.default_rng(12)
    x = bf16((16, 16, 128, 16), rng)
    g = bf16((16, 16, 128, 16), rng)
    dw = torch.zeros((16, 27, 16), dtype=torch.float32, device="cuda")
    error = torch.zeros(1, dtype=torch.int32, device="cuda")
    prior.conv3d_wgrad([x], g, dw, None, error=error, wait_limit_ns=1)
    torch.cuda.synchronize()
    assert int(error.item()) != 0
    error.zero_()
    dw.zero_()
    db = torch.zeros(16, dtype=torch.float32, device="cuda")
    prior.conv3d_wgrad([x], g, dw, db, error=error)
    torch.cuda.synchronize()
    assert int(error.item()) == 0
    want_w, want_b = expected([x], g)
    close(dw.cpu().numpy(), want_w)
    close(db.cpu().numpy(), want_b)
