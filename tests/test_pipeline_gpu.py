"""The whole path on the B200: standardization, R2C, CTF insertion, the Wiener
divide and the C2R, against the same path on the CPU (the oracle for
standardization and insertion, numpy/pocketfft for the FFTs)."""

import numpy as np
import pytest
import torch

import oracle
from rexlib_b200 import em, fourier
from tests.cases import rel_l2, rotations

pytestmark = pytest.mark.gpu


def gaussian_image(n, width):
    c = n // 2
    y, x = np.mgrid[:n, :n] - c
    return np.exp(-(x * x + y * y) / (2 * width * width))


def test_gaussian_blob_is_reconstructed():
    # A Gaussian projects onto the same Gaussian in every direction, so one
    # image serves all orientations; 400 random orientations inserted with
    # the linear window, divided where the weight exceeds 1e-3 and brought
    # back correlate above 0.99 with the blob over the images' box (the check
    # of test_cpu_reconstruction.cpp:418-503, here on the GPU path).
    n, big, width, count = 32, 64, 2.0, 400
    image = gaussian_image(n, width).astype(np.float32)
    spectra = fourier.rfft2(torch.from_numpy(image).cuda()[None])
    rng = np.random.default_rng(14)
    tr = np.zeros((count, 3, 4), np.float32)
    tr[:, :, :3] = rotations(count, rng)
    H = big // 2 + 1
    num = torch.zeros((big, big, H), dtype=torch.complex64, device="cuda")
    den = torch.zeros((big, big, H), dtype=torch.float32, device="cuda")
    em.insert_slices(num, den, spectra.expand(count, n, n // 2 + 1), torch.from_numpy(tr).cuda(),
                     torch.ones(n // 2 + 1, device="cuda"), em.GriddingWindow.linear(), numerator_out=num,
                     denominator_out=den)
    volume = fourier.wiener_irfft3(num, den, 1e-3, threshold=True).cpu().numpy().astype(np.float64)
    c = big // 2
    z, y, x = np.mgrid[:big, :big, :big] - c
    inside = (np.abs(z) <= n // 2) & (np.abs(y) <= n // 2) & (np.abs(x) <= n // 2)
    blob = np.exp(-(x * x + y * y + z * z) / (2 * width * width))
    v, b = volume[inside], blob[inside]
    correlation = float(v @ b / np.sqrt((v @ v) * (b @ b)))
    assert correlation > 0.99, correlation


def ctf_of(params, n, pixel, voltage=300.0, cs=2.7, q=0.1):
    """c(k) on the (n, n//2+1) half spectrum, float64 (insert_ctf_slices_operation.hpp:40-55)."""
    volts = voltage * 1e3
    wl = 12.2643247 / np.sqrt(volts * (1.0 + 0.978466e-6 * volts))
    ky = np.fft.fftfreq(n, 1.0 / n)[:, None]
    kx = np.arange(n // 2 + 1)[None, :]
    du, dv, angle, shift = params
    s2 = (kx * kx + ky * ky) / (n * pixel) ** 2
    t = np.arctan2(ky, kx)
    d = 0.5 * (du + dv) + 0.5 * (du - dv) * np.cos(2 * (t - angle))
    return np.sin(np.pi * wl * d * s2 - 0.5 * np.pi * cs * 1e7 * wl ** 3 * s2 * s2 + shift + np.arcsin(q))


def synthetic_particles(count, n, blobs, seed):
    """Projections of a Gaussian-blob phantom at uniform SO(3) orientations,
    CTF-modulated (300 kV, Cs 2.7, Q 0.1, 1 A/px, defocus 0.8-2.5 um) with
    Gaussian noise at SNR 0.1."""
    rng = np.random.default_rng(seed)
    centres = rng.standard_normal((blobs, 3))
    centres *= (rng.uniform(0, 1, blobs) ** (1 / 3) * 24.0 / np.linalg.norm(centres, axis=1))[:, None]
    sigmas = rng.uniform(2.0, 4.0, blobs)
    amps = rng.uniform(0.5, 1.5, blobs)
    R = rotations(count, rng)
    ctf = np.stack([rng.uniform(8000, 25000, count), rng.uniform(8000, 25000, count),
                    rng.uniform(0, np.pi, count), np.zeros(count)], -1)
    c = n // 2
    yy, xx = np.mgrid[:n, :n] - c
    images = np.zeros((count, n, n))
    for p in range(count):
        proj = R[p] @ centres.T  # the image-plane coordinates are rows 0 and 1
        img = np.zeros((n, n))
        for b in range(blobs):
            img += amps[b] * sigmas[b] * np.sqrt(2 * np.pi) * np.exp(
                -((xx - proj[0, b]) ** 2 + (yy - proj[1, b]) ** 2) / (2 * sigmas[b] ** 2))
        images[p] = np.fft.irfft2(np.fft.rfft2(img) * ctf_of(ctf[p], n, 1.0), s=(n, n))
    signal = images.var()
    images += rng.standard_normal(images.shape) * np.sqrt(signal / 0.1)
    tr = np.zeros((count, 3, 4))
    tr[:, :, :3] = R
    return images.astype(np.float32), tr.astype(np.float32), ctf.astype(np.float32)


def test_config0_path_matches_the_cpu_path():
    # 1,000 particles of 64^2 into 64^3: standardize (radius 0.45 n), R2C,
    # CTF insertion (linear), Wiener with 1e-3, C2R.
    n = big = 64
    count = 1000
    images, tr, ctf = synthetic_particles(count, n, 20, seed=2024)
    keys = np.arange(1, count + 1, dtype=np.uint64)
    optics = em.CtfOptics(300.0, 2.7, 0.1)

    # GPU.
    g_std = em.standardize_background_2d(torch.from_numpy(images).cuda(), torch.from_numpy(keys.view(np.int64)).cuda(),
                                         0.45 * n, (-np.inf, np.inf))
    g_spec = fourier.rfft2(g_std)
    H = big // 2 + 1
    num = torch.zeros((big, big, H), dtype=torch.complex64, device="cuda")
    den = torch.zeros((big, big, H), dtype=torch.float32, device="cuda")
    em.insert_ctf_slices(num, den, g_spec, torch.from_numpy(tr).cuda(), torch.from_numpy(ctf).cuda(),
                         torch.ones(n // 2 + 1, device="cuda"), em.GriddingWindow.linear(), optics, 1.0,
                         numerator_out=num, denominator_out=den)
    g_vol = fourier.wiener_irfft3(num, den, 1e-3).cpu().numpy()

    # CPU.
    c_std = oracle.standardize(images, keys, 0.45 * n)
    np.testing.assert_array_equal(g_std.cpu().numpy(), c_std)
    c_spec = np.fft.rfft2(c_std.astype(np.float64)).astype(np.complex64)
    c_num = np.zeros((1, big, big, H), np.complex64)
    c_den = np.zeros((1, big, big, H), np.float32)
    oracle.insert("ctf", c_num, c_den, c_spec, tr[None], np.ones(n // 2 + 1, np.float32), ctf[None],
                  window=oracle.Window("linear"), optics=oracle.Optics(300.0, 2.7, 0.1), pixel_size=1.0)
    assert rel_l2(num.cpu().numpy(), c_num[0]) <= 1e-5
    assert rel_l2(den.cpu().numpy(), c_den[0]) <= 1e-5
    c_vol = np.fft.irfftn(c_num[0].astype(np.complex128) / (c_den[0].astype(np.float64) + 1e-3), s=(big, big, big),
                          axes=(0, 1, 2))
    assert rel_l2(g_vol, c_vol) <= 1e-5


@pytest.mark.parametrize("fused", [False, True])
@pytest.mark.parametrize("deterministic", [False, True])
def test_config0_path_replays_as_a_cuda_graph(deterministic, fused):
    # The whole path (standardization, R2C, CTF insertion, Wiener and C2R)
    # issues no synchronization, and its workspaces come from the caller's
    # allocator, so it captures into one CUDA graph. Replays give what the
    # eager calls give: bit for bit in the deterministic mode, within the
    # insertion tolerance in the throughput mode, whose FP32 sums have no
    # fixed order. `fused` runs standardization and R2C as one call
    # (rexlib_b200_standardize_rfft2).
    n = big = 64
    count = 1000
    images, tr, ctf = synthetic_particles(count, n, 20, seed=2025)
    keys = np.arange(1, count + 1, dtype=np.uint64)
    optics = em.CtfOptics(300.0, 2.7, 0.1)
    d_images = torch.from_numpy(images).cuda()
    d_keys = torch.from_numpy(keys.view(np.int64)).cuda()
    d_tr, d_ctf = torch.from_numpy(tr).cuda(), torch.from_numpy(ctf).cuda()
    radial = torch.ones(n // 2 + 1, device="cuda")
    H = big // 2 + 1
    num = torch.zeros((big, big, H), dtype=torch.complex64, device="cuda")
    den = torch.zeros((big, big, H), dtype=torch.float32, device="cuda")

    def path():
        if fused:
            spectra, _ = fourier.standardize_rfft2_ctf(d_images, d_keys, 0.45 * n, (-np.inf, np.inf))
        else:
            std = em.standardize_background_2d(d_images, d_keys, 0.45 * n, (-np.inf, np.inf))
            spectra = fourier.rfft2(std)
        num.zero_()
        den.zero_()
        em.insert_ctf_slices(num, den, spectra, d_tr, d_ctf, radial, em.GriddingWindow.linear(), optics, 1.0,
                             numerator_out=num, denominator_out=den, deterministic=deterministic)
        return fourier.wiener_irfft3(num, den, 1e-3)

    eager = path().clone()
    eager_num, eager_den = num.clone(), den.clone()
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        path()
    torch.cuda.current_stream().wait_stream(side)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        volume = path()
    for _ in range(2):
        graph.replay()
        torch.cuda.synchronize()
        if deterministic:
            assert torch.equal(num, eager_num) and torch.equal(den, eager_den)
            assert torch.equal(volume, eager)
        else:
            assert rel_l2(num.cpu().numpy(), eager_num.cpu().numpy()) <= 1e-5
            assert rel_l2(volume.cpu().numpy(), eager.cpu().numpy()) <= 1e-5
    del graph
