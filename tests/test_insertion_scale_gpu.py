"""The insertion at the bench's full size (100,000 slices of 256^2 into 256^3),
through properties that hold at any size, and against the oracle at 2,000
slices of the same box.

- The throughput mode (tile-major scatter, FP32 atomics) and the
  deterministic mode (an ordered gather) are independent algorithms; they
  agree within relative L2 1e-5.
- The deterministic mode gives the bits of one call when the batch is
  inserted in two calls (the split-batch property of the CPU backend,
  test_cpu_reconstruction.cpp:505-594).
- At 2,000 slices both modes match the oracle within 1e-5."""

import numpy as np
import pytest
import torch

import oracle
from rexlib_b200 import em
from tests.cases import rel_l2, rotations

pytestmark = pytest.mark.gpu

N = 256
H = N // 2 + 1
OPTICS = em.CtfOptics(300.0, 2.7, 0.1)


def parameters(count, seed):
    rng = np.random.default_rng(seed)
    tr = np.zeros((count, 3, 4), np.float32)
    tr[:, :, :3] = rotations(count, rng)
    tr[:, :, 3] = rng.uniform(-2, 2, (count, 3))
    ctf = np.stack([rng.uniform(8000, 25000, count), rng.uniform(8000, 25000, count), rng.uniform(0, np.pi, count),
                    np.zeros(count)], -1).astype(np.float32)
    return tr, ctf


def spectra(count, seed, device):
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    out = torch.empty((count, N, H), dtype=torch.complex64, device=device)
    for start in range(0, count, 10000):
        stop = min(count, start + 10000)
        out[start:stop] = torch.complex(torch.randn((stop - start, N, H), generator=g, device=device),
                                        torch.randn((stop - start, N, H), generator=g, device=device))
    return out


def insert(slices, tr, ctf, deterministic, num=None, den=None, window=None):
    device = slices.device
    if num is None:
        num = torch.zeros((N, N, H), dtype=torch.complex64, device=device)
        den = torch.zeros((N, N, H), dtype=torch.float32, device=device)
    em.insert_ctf_slices(num, den, slices, torch.from_numpy(tr).to(device), torch.from_numpy(ctf).to(device),
                         torch.ones(H, device=device), window or em.GriddingWindow.linear(), OPTICS, 1.0,
                         numerator_out=num, denominator_out=den, deterministic=deterministic)
    return num, den


@pytest.fixture(scope="module")
def full_size():
    device = torch.device("cuda", 0)
    tr, ctf = parameters(100_000, 7)
    return spectra(100_000, 8, device), tr, ctf


def test_full_size_modes_agree(full_size):
    slices, tr, ctf = full_size
    tnum, tden = insert(slices, tr, ctf, deterministic=False)
    dnum, dden = insert(slices, tr, ctf, deterministic=True)
    assert rel_l2(tnum.cpu().numpy(), dnum.cpu().numpy()) <= 1e-5
    assert rel_l2(tden.cpu().numpy(), dden.cpu().numpy()) <= 1e-5


def test_full_size_deterministic_split_batch_is_bit_identical(full_size):
    slices, tr, ctf = full_size
    whole_num, whole_den = insert(slices, tr, ctf, deterministic=True)
    num, den = insert(slices[:50_000], tr[:50_000], ctf[:50_000], deterministic=True)
    num, den = insert(slices[50_000:], tr[50_000:], ctf[50_000:], deterministic=True, num=num, den=den)
    assert torch.equal(num, whole_num) and torch.equal(den, whole_den)


@pytest.mark.parametrize("deterministic", [False, True])
def test_two_thousand_slices_match_the_oracle(deterministic):
    device = torch.device("cuda", 0)
    tr, ctf = parameters(2000, 9)
    slices = spectra(2000, 10, device)
    num, den = insert(slices, tr, ctf, deterministic)
    onum = np.zeros((1, N, N, H), np.complex64)
    oden = np.zeros((1, N, N, H), np.float32)
    oracle.insert("ctf", onum, oden, slices.cpu().numpy(), tr[None], np.ones(H, np.float32), ctf[None],
                  window=oracle.Window("linear"), optics=oracle.Optics(300.0, 2.7, 0.1), pixel_size=1.0)
    assert rel_l2(num.cpu().numpy(), onum[0]) <= 1e-5
    assert rel_l2(den.cpu().numpy(), oden[0]) <= 1e-5


@pytest.mark.parametrize("deterministic", [False, True])
@pytest.mark.parametrize("half_width,shape", [(1.5, 6.0), (2.0, 9.0)])
def test_kaiser_bessel_at_full_box_matches_the_oracle(deterministic, half_width, shape):
    # The Kaiser-Bessel window at 256^2 into 256^3: 27 or 64 taps a sample,
    # through the tile-major kernel (throughput) or the ordered gather.
    device = torch.device("cuda", 0)
    tr, ctf = parameters(300, 11)
    slices = spectra(300, 12, device)
    num, den = insert(slices, tr, ctf, deterministic, window=em.GriddingWindow.kaiser_bessel(half_width, shape))
    onum = np.zeros((1, N, N, H), np.complex64)
    oden = np.zeros((1, N, N, H), np.float32)
    oracle.insert("ctf", onum, oden, slices.cpu().numpy(), tr[None], np.ones(H, np.float32), ctf[None],
                  window=oracle.Window("kaiser_bessel", half_width, shape), optics=oracle.Optics(300.0, 2.7, 0.1),
                  pixel_size=1.0)
    assert rel_l2(num.cpu().numpy(), onum[0]) <= 1e-5
    assert rel_l2(den.cpu().numpy(), oden[0]) <= 1e-5


@pytest.mark.parametrize("deterministic", [False, True])
@pytest.mark.parametrize("box", [512, 384])
def test_larger_boxes_match_the_oracle(deterministic, box):
    # 512^2 slices into 512^3 (0.8 GB of accumulators) and 384^2 into 384^3:
    # boxes above the bench's, where the tiles, work plans and stages are
    # sized from larger extents.
    device = torch.device("cuda", 0)
    h = box // 2 + 1
    count = 24
    tr, ctf = parameters(count, 13 + box)
    g = torch.Generator(device=device)
    g.manual_seed(box)
    slices = torch.complex(torch.randn((count, box, h), generator=g, device=device),
                           torch.randn((count, box, h), generator=g, device=device))
    num = torch.zeros((box, box, h), dtype=torch.complex64, device=device)
    den = torch.zeros((box, box, h), dtype=torch.float32, device=device)
    em.insert_ctf_slices(num, den, slices, torch.from_numpy(tr).to(device), torch.from_numpy(ctf).to(device),
                         torch.ones(h, device=device), em.GriddingWindow.linear(), OPTICS, 1.0,
                         numerator_out=num, denominator_out=den, deterministic=deterministic)
    onum = np.zeros((1, box, box, h), np.complex64)
    oden = np.zeros((1, box, box, h), np.float32)
    oracle.insert("ctf", onum, oden, slices.cpu().numpy(), tr[None], np.ones(h, np.float32), ctf[None],
                  window=oracle.Window("linear"), optics=oracle.Optics(300.0, 2.7, 0.1), pixel_size=1.0)
    assert rel_l2(num.cpu().numpy(), onum[0]) <= 1e-5
    assert rel_l2(den.cpu().numpy(), oden[0]) <= 1e-5
