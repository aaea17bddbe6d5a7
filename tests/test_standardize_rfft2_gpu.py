"""The fused standardization + R2C (rexlib_b200_standardize_rfft2) against
the two calls it replaces (rexlib_b200_standardize_background, then
rexlib_b200_rfft2 with the same epilogue): spectra, CTF weights, statistics
and the standardized images bit for bit. The two calls are themselves checked
against the oracle and numpy elsewhere; here the standardized images are also
compared with the oracle, and the spectra with numpy's FFT of them."""

import numpy as np
import pytest
import torch

import oracle
from rexlib_b200 import _capi, em, fourier
from tests.cases import rel_l2

pytestmark = pytest.mark.gpu

OPTICS = em.CtfOptics(300.0, 2.7, 0.1)


def images_of(batch, n, seed):
    rng = np.random.default_rng(seed)
    v = (rng.standard_normal((batch, n, n)) * rng.uniform(0.5, 3.0, (batch, 1, 1)) +
         rng.uniform(-2, 2, (batch, 1, 1))).astype(np.float32)
    # Elements the map replaces with draws: not finite, or far out of bounds.
    v[0, 3, 4] = np.nan
    v[-1, 1, 1] = -np.inf
    v[1 % batch, 2, 2] = 1e6
    v[batch // 2, n // 2, n // 2] = np.inf
    return v, rng


def ctf_of(batch, rng):
    return np.stack([rng.uniform(5000, 40000, batch), rng.uniform(5000, 40000, batch), rng.uniform(0, np.pi, batch),
                     rng.uniform(0, 0.3, batch)], -1).astype(np.float32)


def bits(t: torch.Tensor) -> np.ndarray:
    a = t.detach().cpu().contiguous()
    if a.dtype == torch.complex64:
        a = torch.view_as_real(a)
    return a.numpy().view(np.uint32 if a.dtype == torch.float32 else np.uint64)


@pytest.mark.parametrize("n", [64, 128, 256])
@pytest.mark.parametrize("bounds", [(-np.inf, np.inf), (-3.0, 3.0), 2.5])
@pytest.mark.parametrize("epilogue", ["none", "ctf", "flip", "ctf_no_weights"])
@pytest.mark.parametrize("shared_key", [False, True])
def test_fused_equals_two_calls(cuda, n, bounds, epilogue, shared_key):
    batch = 37
    v, rng = images_of(batch, n, n + batch)
    images = torch.from_numpy(v).cuda()
    keys = torch.from_numpy(rng.integers(0, 2**63, 1 if shared_key else batch, dtype=np.uint64).view(np.int64)).cuda()
    ctf = torch.from_numpy(ctf_of(batch, rng)).cuda()
    volts = torch.from_numpy(np.where(rng.uniform(0, 1, batch) < 0.5, 200.0, 300.0).astype(np.float32)).cuda()
    radius = 0.45 * n

    stats2 = torch.zeros(2 * batch, dtype=torch.float64, device="cuda")
    std2 = em.standardize_background_2d(images, keys.reshape(()) if shared_key else keys, radius, bounds,
                                        statistics=stats2)
    stats1 = torch.zeros_like(stats2)
    std1 = torch.empty_like(images)
    if epilogue == "none":
        spec2, w2 = fourier.rfft2(std2), None
        spec1, w1 = fourier.standardize_rfft2_ctf(images, keys, radius, bounds, standardized=std1, statistics=stats1)
    else:
        kwargs = dict(voltage=volts, phase_flip=epilogue == "flip", weights=epilogue != "ctf_no_weights")
        spec2, w2 = fourier.rfft2_ctf(std2, ctf, OPTICS, 1.1, **kwargs)
        spec1, w1 = fourier.standardize_rfft2_ctf(images, keys, radius, bounds, ctf, OPTICS, 1.1, **kwargs,
                                                  standardized=std1, statistics=stats1)
    assert np.array_equal(bits(spec1), bits(spec2))
    assert (w1 is None) == (w2 is None)
    if w1 is not None:
        assert np.array_equal(bits(w1), bits(w2))
    assert np.array_equal(bits(stats1), bits(stats2))
    assert np.array_equal(bits(std1), bits(std2))


@pytest.mark.parametrize("n", [64, 128, 256])
def test_fused_against_the_oracle_and_numpy(cuda, n):
    batch = 9
    v, rng = images_of(batch, n, 3 * n)
    keys = rng.integers(0, 2**63, batch, dtype=np.uint64)
    spectra, _ = fourier.standardize_rfft2_ctf(torch.from_numpy(v).cuda(), torch.from_numpy(keys.view(np.int64)).cuda(),
                                               0.45 * n, (-3.0, 3.0))
    want_std = oracle.standardize(v, keys, 0.45 * n, -3.0, 3.0)
    want = np.fft.rfft2(want_std.astype(np.float64))
    assert rel_l2(spectra.cpu().numpy(), want) <= 2e-6


def test_standardized_images_are_optional(cuda):
    v, rng = images_of(11, 128, 5)
    images = torch.from_numpy(v).cuda()
    keys = torch.from_numpy(rng.integers(0, 2**63, 11, dtype=np.uint64).view(np.int64)).cuda()
    ctf = torch.from_numpy(ctf_of(11, rng)).cuda()
    a, wa = fourier.standardize_rfft2_ctf(images, keys, 57.6, (-np.inf, np.inf), ctf, OPTICS, 1.0)
    std = torch.empty_like(images)
    b, wb = fourier.standardize_rfft2_ctf(images, keys, 57.6, (-np.inf, np.inf), ctf, OPTICS, 1.0, standardized=std)
    assert np.array_equal(bits(a), bits(b)) and np.array_equal(bits(wa), bits(wb))
    # the input is not touched
    assert np.array_equal(images.cpu().numpy().view(np.uint32), v.view(np.uint32))


def test_refusals(cuda):
    keys = torch.ones(2, dtype=torch.int64, device="cuda")
    with pytest.raises(_capi.RexlibB200Error) as e:
        fourier.standardize_rfft2_ctf(torch.zeros(2, 96, 96, device="cuda"), keys, 40.0, 3.0)
    assert e.value.status == _capi.UNSUPPORTED
    # the images must be 16-byte aligned
    buf = torch.zeros(2 * 64 * 64 + 1, device="cuda")
    with pytest.raises(_capi.RexlibB200Error) as e:
        fourier.standardize_rfft2_ctf(buf[1:].view(2, 64, 64), keys, 28.0, 3.0)
    assert e.value.status == _capi.INVALID_ARGUMENT
    with pytest.raises(ValueError, match="one per equal run"):
        fourier.standardize_rfft2_ctf(torch.zeros(3, 64, 64, device="cuda"), keys, 28.0, 3.0)
    # the reference's parameter checks
    with pytest.raises(_capi.RexlibB200Error, match="bounds must lie on either side of 0"):
        fourier.standardize_rfft2_ctf(torch.zeros(2, 64, 64, device="cuda"), keys, 28.0, (1.0, 2.0))
