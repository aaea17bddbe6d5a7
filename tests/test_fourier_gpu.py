"""Real FFTs, the CTF epilogue and the Wiener C2R on the B200 against numpy
(pocketfft, the FFT family the reference's CPU backend calls) in float64.
Tolerance: relative L2 <= 2e-6 for the float32 transforms; 5e-5 where the
CTF enters, whose phase (hundreds of radians at 4 um of defocus) the CPU
backend also evaluates in float32 (about 2e-5 against FP64)."""

import numpy as np
import pytest
import torch

from rexlib_b200 import fourier
from rexlib_b200.em import CtfOptics
from tests.cases import rel_l2

pytestmark = pytest.mark.gpu

TOL = 2e-6


@pytest.mark.parametrize("n", [32, 64, 96, 128, 160, 192, 200, 256])
def test_rfft2_matches_numpy(n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal((3, n, n)).astype(np.float32)
    got = fourier.rfft2(torch.from_numpy(x).cuda()).cpu().numpy()
    want = np.fft.rfft2(x.astype(np.float64))
    assert got.shape == want.shape
    assert rel_l2(got, want) <= TOL


@pytest.mark.parametrize("n", [64, 128])
def test_rfft2_of_an_input_only_8_byte_aligned(n):
    # The 64 and 128 paths stage images with 16-byte copies; an input that
    # starts 8 bytes into an allocation takes the general kernel and gives the same.
    rng = np.random.default_rng(9)
    x = rng.standard_normal((2, n, n)).astype(np.float32)
    flat = torch.zeros(2 * n * n + 2, dtype=torch.float32, device="cuda")
    flat[2:] = torch.from_numpy(x.ravel()).cuda()
    shifted = flat[2:].view(2, n, n)
    assert shifted.data_ptr() % 16 == 8
    got = fourier.rfft2(shifted).cpu().numpy()
    assert rel_l2(got, np.fft.rfft2(x.astype(np.float64))) <= TOL


@pytest.mark.parametrize("n", [32, 64, 96, 128, 160, 192, 200])
def test_irfft2_matches_numpy(n):
    rng = np.random.default_rng(n + 1)
    X = np.fft.rfft2(rng.standard_normal((2, n, n)))
    got = fourier.irfft2(torch.from_numpy(X.astype(np.complex64)).cuda()).cpu().numpy()
    want = np.fft.irfft2(X, s=(n, n))
    assert rel_l2(got, want) <= TOL


def test_irfft2_ignores_the_imaginary_parts_of_the_real_columns():
    n = 64
    rng = np.random.default_rng(5)
    X = (rng.standard_normal((1, n, n // 2 + 1)) + 1j * rng.standard_normal((1, n, n // 2 + 1)))
    got = fourier.irfft2(torch.from_numpy(X.astype(np.complex64)).cuda()).cpu().numpy()
    want = np.fft.irfft2(X, s=(n, n))
    assert rel_l2(got, want) <= TOL


def test_round_trip():
    rng = np.random.default_rng(6)
    x = rng.standard_normal((4, 128, 128)).astype(np.float32)
    back = fourier.irfft2(fourier.rfft2(torch.from_numpy(x).cuda())).cpu().numpy()
    assert rel_l2(back, x) <= TOL


@pytest.mark.parametrize("big", [32, 64, 96, 128, 200, 256])
def test_irfft3_matches_numpy(big):
    rng = np.random.default_rng(big)
    X = np.fft.rfftn(rng.standard_normal((big, big, big)))
    got = fourier.irfft3(torch.from_numpy(X.astype(np.complex64)).cuda()).cpu().numpy()
    want = np.fft.irfftn(X, s=(big, big, big), axes=(0, 1, 2))
    assert rel_l2(got, want) <= TOL


@pytest.mark.parametrize("threshold", [False, True])
def test_wiener_irfft3_matches_numpy(threshold):
    big = 64
    rng = np.random.default_rng(7)
    H = big // 2 + 1
    num = (rng.standard_normal((big, big, H)) + 1j * rng.standard_normal((big, big, H))).astype(np.complex64)
    den = rng.uniform(0, 2, (big, big, H)).astype(np.float32)
    den[0, 0, :4] = 0.0
    got = fourier.wiener_irfft3(torch.from_numpy(num).cuda(), torch.from_numpy(den).cuda(), 1e-3,
                                threshold=threshold).cpu().numpy()
    n64, d64 = num.astype(np.complex128), den.astype(np.float64)
    if threshold:
        X = np.where(d64 > 1e-3, n64 / np.where(d64 > 1e-3, d64, 1.0), 0.0)
    else:
        X = n64 / (d64 + 1e-3)
    want = np.fft.irfftn(X, s=(big, big, big), axes=(0, 1, 2))
    assert rel_l2(got, want) <= 1e-5


def reference_ctf(optics, pixel, n, params):
    """The CTF expression of insert_ctf_slices_operation.hpp:40-55 in float64."""
    ky = np.fft.fftfreq(n, 1.0 / n)[:, None]
    kx = np.arange(n // 2 + 1)[None, :]
    du, dv, angle, shift = [float(v) for v in params]
    wl = optics.wavelength
    s2 = (kx * kx + ky * ky) / (n * pixel) ** 2
    t = np.arctan2(ky, kx)
    d = 0.5 * (du + dv) + 0.5 * (du - dv) * np.cos(2 * (t - angle))
    return np.sin(np.pi * wl * d * s2 - 0.5 * np.pi * optics.spherical_aberration * 1e7 * wl ** 3 * s2 * s2 + shift
                  + np.arcsin(optics.amplitude_contrast))


@pytest.mark.parametrize("n", [64, 128, 256])
def test_rfft2_ctf_epilogue(n):
    rng = np.random.default_rng(n + 3)
    optics = CtfOptics(300.0, 2.7, 0.1)
    x = rng.standard_normal((3, n, n)).astype(np.float32)
    params = np.stack([rng.uniform(5000, 40000, 3), rng.uniform(5000, 40000, 3), rng.uniform(0, np.pi, 3),
                       np.zeros(3)], -1).astype(np.float32)
    spectra, weights = fourier.rfft2_ctf(torch.from_numpy(x).cuda(), torch.from_numpy(params).cuda(), optics, 1.0)
    X = np.fft.rfft2(x.astype(np.float64))
    c = np.stack([reference_ctf(optics, 1.0, n, p) for p in params])
    assert rel_l2(spectra.cpu().numpy(), c * X) <= 5e-5
    assert rel_l2(weights.cpu().numpy(), c * c) <= 5e-5


@pytest.mark.parametrize("n", [64, 128, 256])
def test_rfft2_phase_flip_and_per_image_voltage(n):
    rng = np.random.default_rng(9)
    optics = CtfOptics(300.0, 2.7, 0.1)
    x = rng.standard_normal((4, n, n)).astype(np.float32)
    params = np.stack([rng.uniform(5000, 40000, 4), rng.uniform(5000, 40000, 4), rng.uniform(0, np.pi, 4),
                       np.zeros(4)], -1).astype(np.float32)
    volts = np.array([200.0, 300.0, 200.0, 300.0], np.float32)
    spectra, weights = fourier.rfft2_ctf(torch.from_numpy(x).cuda(), torch.from_numpy(params).cuda(), optics, 1.0,
                                         voltage=torch.from_numpy(volts).cuda(), phase_flip=True)
    X = np.fft.rfft2(x.astype(np.float64))
    c = np.stack([reference_ctf(CtfOptics(float(v), 2.7, 0.1), 1.0, n, p) for p, v in zip(params, volts)])
    # Away from the zeros of the CTF the sign is unambiguous.
    mask = np.abs(c) > 1e-3
    got = spectra.cpu().numpy()
    assert rel_l2(got[mask], (np.sign(c) * X)[mask]) <= 5e-5
    assert rel_l2(weights.cpu().numpy()[mask], np.abs(c)[mask]) <= 5e-5


# Every transform here is deterministic by construction (no atomics), so
# repeated calls on one input give the same bits; a missing barrier or a race
# on a shared table shows up here as a difference between calls.
@pytest.mark.parametrize("n", [32, 64, 96, 128, 160, 192, 200, 256])
def test_rfft2_and_its_ctf_epilogue_are_repeatable(n):
    rng = np.random.default_rng(40 + n)
    x = torch.from_numpy(rng.standard_normal((48, n, n)).astype(np.float32)).cuda()
    params = np.stack([rng.uniform(8000, 25000, 48), rng.uniform(8000, 25000, 48), rng.uniform(0, np.pi, 48),
                       np.zeros(48)], -1).astype(np.float32)
    ctf = torch.from_numpy(params).cuda()
    optics = CtfOptics(300.0, 2.7, 0.1)
    first = fourier.rfft2(x).cpu().numpy()
    first_ctf = [t.cpu().numpy() for t in fourier.rfft2_ctf(x, ctf, optics, 1.0)]
    for _ in range(4):
        np.testing.assert_array_equal(fourier.rfft2(x).cpu().numpy(), first)
        for a, b in zip(fourier.rfft2_ctf(x, ctf, optics, 1.0), first_ctf):
            np.testing.assert_array_equal(a.cpu().numpy(), b)


@pytest.mark.parametrize("n", [32, 64, 128, 200])
def test_irfft2_is_repeatable(n):
    rng = np.random.default_rng(50 + n)
    X = torch.from_numpy(np.fft.rfft2(rng.standard_normal((48, n, n))).astype(np.complex64)).cuda()
    first = fourier.irfft2(X).cpu().numpy()
    for _ in range(4):
        np.testing.assert_array_equal(fourier.irfft2(X).cpu().numpy(), first)


@pytest.mark.parametrize("big", [64, 96, 128, 256])
def test_irfft3_and_wiener_are_repeatable(big):
    rng = np.random.default_rng(60 + big)
    H = big // 2 + 1
    num = torch.from_numpy((rng.standard_normal((big, big, H)) + 1j * rng.standard_normal((big, big, H)))
                           .astype(np.complex64)).cuda()
    den = torch.from_numpy(rng.uniform(0, 2, (big, big, H)).astype(np.float32)).cuda()
    first = fourier.irfft3(num).cpu().numpy()
    first_w = fourier.wiener_irfft3(num, den, 1e-3).cpu().numpy()
    for _ in range(3):
        np.testing.assert_array_equal(fourier.irfft3(num).cpu().numpy(), first)
        np.testing.assert_array_equal(fourier.wiener_irfft3(num, den, 1e-3).cpu().numpy(), first_w)
