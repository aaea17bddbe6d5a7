"""The prior's volume tools on the B200 against numpy in float64: the 3D
R2C, the Fourier shell correlation, the prior-regularised Wiener
combination, the analytic blob spectrum and the noiseless CTF-modulated
phantom slices."""

import ctypes

import numpy as np
import pytest
import torch

from rexlib_b200 import _capi, prior
from tests.cases import rel_l2

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [32, 64, 128, 256])
def test_rfft3_matches_numpy(n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal((n, n, n)).astype(np.float32)
    got = prior.rfft3(torch.from_numpy(x).cuda()).cpu().numpy()
    assert rel_l2(got, np.fft.rfftn(x.astype(np.float64))) <= 2e-6


def test_fsc_matches_numpy():
    n = 32
    rng = np.random.default_rng(1)
    a = (rng.standard_normal((n, n, n // 2 + 1)) + 1j * rng.standard_normal((n, n, n // 2 + 1))).astype(np.complex64)
    b = (a + 0.5 * (rng.standard_normal(a.shape) + 1j * rng.standard_normal(a.shape))).astype(np.complex64)
    got = prior.fsc(torch.from_numpy(a).cuda(), torch.from_numpy(b).cuda())
    kz = np.fft.fftfreq(n, 1 / n)[:, None, None]
    ky = np.fft.fftfreq(n, 1 / n)[None, :, None]
    kx = np.arange(n // 2 + 1)[None, None, :]
    shell = np.floor(np.sqrt(kx ** 2 + ky ** 2 + kz ** 2) + 0.5).astype(int)
    w = np.where((kx == 0) | (kx == n // 2), 1.0, 2.0) * np.ones(a.shape)
    a64, b64 = a.astype(np.complex128), b.astype(np.complex128)
    want = []
    for s in range(n // 2 + 1):
        m = shell == s
        num = np.sum(w[m] * (a64[m] * np.conj(b64[m])).real)
        want.append(num / np.sqrt(np.sum(w[m] * np.abs(a64[m]) ** 2) * np.sum(w[m] * np.abs(b64[m]) ** 2)))
    assert np.allclose(got, want, atol=1e-9)
    same = prior.fsc(torch.from_numpy(a).cuda(), torch.from_numpy(a).cuda())
    assert np.allclose(same, 1.0)


def render(blobs, n):
    z, y, x = np.meshgrid(*[np.arange(n, dtype=np.float64)] * 3, indexing="ij")
    v = np.zeros((n, n, n))
    for a, s, cx, cy, cz in blobs.astype(np.float64):
        v += a * np.exp(-((x - n / 2 - cx) ** 2 + (y - n / 2 - cy) ** 2 + (z - n / 2 - cz) ** 2) / (2 * s * s))
    return v


def central_blobs(n, count, rng):
    b = prior.blob_phantom(rng, n, count)
    b[:, 2:] *= 0.5  # well inside the box: no tails wrap around
    return b


def test_blob_spectrum_is_the_rendered_phantom():
    n = 64
    b = central_blobs(n, 12, np.random.default_rng(2))
    got = prior.blob_spectrum(b, n).cpu().numpy()
    assert rel_l2(got, np.fft.rfftn(render(b, n))) <= 1e-4
    # Low-passed: nothing beyond the cutoff shell.
    lp = prior.blob_spectrum(b, n, cutoff=n / 4).cpu().numpy()
    kz = np.fft.fftfreq(n, 1 / n)[:, None, None]
    ky = np.fft.fftfreq(n, 1 / n)[None, :, None]
    kx = np.arange(n // 2 + 1)[None, None, :]
    outside = kx ** 2 + ky ** 2 + kz ** 2 > (n / 4) ** 2
    assert np.all(lp[outside] == 0) and rel_l2(lp[~outside], got[~outside]) <= 1e-6


def test_phantom_slices_are_ctf_weighted_projections():
    n = 64
    rng = np.random.default_rng(3)
    b = central_blobs(n, 10, rng)
    tr = prior.random_orientations(4, rng)
    ctf = np.stack([rng.uniform(8000, 25000, 4), rng.uniform(8000, 25000, 4), rng.uniform(0, np.pi, 4),
                    np.zeros(4)], -1).astype(np.float32)
    got = prior._slices(torch.from_numpy(b).cuda(), n, torch.from_numpy(tr).cuda(), torch.from_numpy(ctf).cuda(), 0.0,
                        0).cpu().numpy()
    y, x = np.meshgrid(np.arange(n, dtype=np.float64), np.arange(n, dtype=np.float64), indexing="ij")
    wl = 12.2643247 / np.sqrt(300e3 * (1.0 + 0.978466e-6 * 300e3))
    ky = np.fft.fftfreq(n, 1.0 / n)[:, None]
    kx = np.arange(n // 2 + 1)[None, :]
    s2 = (kx * kx + ky * ky) / float(n * n)
    ang = np.arctan2(ky, kx)
    for p in range(4):
        img = np.zeros((n, n))
        for a, s, cx, cy, cz in b.astype(np.float64):
            c = np.array([cx, cy, cz])
            u, v = tr[p, 0, :3] @ c, tr[p, 1, :3] @ c
            img += a * np.sqrt(2 * np.pi) * s * np.exp(-((x - n / 2 - u) ** 2 + (y - n / 2 - v) ** 2) / (2 * s * s))
        du, dv, theta = ctf[p, :3].astype(np.float64)
        d = 0.5 * (du + dv) + 0.5 * (du - dv) * np.cos(2 * (ang - theta))
        c = np.sin(np.pi * wl * d * s2 - 0.5 * np.pi * 2.7e7 * wl ** 3 * s2 * s2 + np.arcsin(0.1))
        assert rel_l2(got[p], np.fft.rfft2(img) * c) <= 1e-4, p


def test_prior_wiener_combination():
    rng = np.random.default_rng(4)
    n = 32
    shape = (n, n, n // 2 + 1)
    num = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)
    den = rng.uniform(0, 3, shape).astype(np.float32)
    pr = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)
    out = torch.empty(shape, dtype=torch.complex64, device="cuda")
    d_num, d_den, d_pr = (torch.from_numpy(a).cuda() for a in (num, den, pr))
    torch.cuda.synchronize()
    _capi.check(_capi.load().rexlib_b200_prior_wiener(
        ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(d_num.data_ptr()), ctypes.c_void_p(d_den.data_ptr()),
        ctypes.c_void_p(d_pr.data_ptr()), n, 0.7, ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
    torch.cuda.synchronize()
    want = (num.astype(np.complex128) + 0.7 * pr) / (den + 0.7)
    assert rel_l2(out.cpu().numpy(), want) <= 1e-6


def test_more_particles_reconstruct_further():
    # The plain Wiener map's FSC-0.143 shell against the phantom grows with
    # the particle count.
    rng = np.random.default_rng(5)
    b = prior.blob_phantom(rng, 64, 20)
    few = prior.Dataset(b, 64, 500, 0.1, seed=6)
    many = prior.Dataset(b, 64, 4000, 0.1, seed=6)
    r_few, _ = few.resolution(few.wiener())
    r_many, _ = many.resolution(many.wiener())
    assert 2 < r_few < r_many, (r_few, r_many)


def test_phantom_slices_of_many_blobs_are_the_sum_of_their_groups():
    # More blobs than one shared-memory table holds are summed in chunks:
    # the noiseless slices of 150 blobs are those of its first 70 plus
    # those of the other 80 (the CTF is linear over the sum).
    rng = np.random.default_rng(21)
    n = 64
    blobs = prior.blob_phantom(rng, n, 150)
    tr = torch.from_numpy(prior.random_orientations(6, rng)).cuda()
    ctf = torch.from_numpy(np.stack([rng.uniform(8000, 25000, 6), rng.uniform(8000, 25000, 6),
                                     rng.uniform(0, np.pi, 6), np.zeros(6)], -1).astype(np.float32)).cuda()
    whole = prior._slices(torch.from_numpy(blobs).cuda(), n, tr, ctf, 0.0, 0)
    part = (prior._slices(torch.from_numpy(np.ascontiguousarray(blobs[:70])).cuda(), n, tr, ctf, 0.0, 0)
            + prior._slices(torch.from_numpy(np.ascontiguousarray(blobs[70:])).cuda(), n, tr, ctf, 0.0, 0))
    torch.cuda.synchronize()
    err = float((whole - part).abs().max()) / float(whole.abs().max())
    assert err < 1e-5, err
