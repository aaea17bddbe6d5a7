"""Background standardization on the B200 against the oracle (bit-identical
to the reference's CPU kernels): statistics within 1e-12 relative, masks and
replacement draws exact, outputs within 1e-6 relative L2 (the reference's
float32 tolerance is 1e-5, test_cpu_preprocessing.cpp:316-324)."""

import json
import os

import numpy as np
import pytest
import torch

import oracle
from rexlib_b200 import em
from tests.cases import rel_l2

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def run(value, keys, radius, bounds, image_rank=2):
    v = torch.from_numpy(value).cuda()
    k = torch.from_numpy(keys.astype(np.int64).view(np.int64)).cuda()
    batch = int(np.prod(value.shape[: value.ndim - image_rank]))
    stats = torch.zeros(2 * batch, dtype=torch.float64, device="cuda")
    axes = tuple(range(-image_rank, 0))
    if keys.size == 1:
        k = k.reshape(())
    out = em.standardize_background(v, k, axes, radius, bounds, statistics=stats)
    torch.cuda.synchronize()
    return out.cpu().numpy(), stats.cpu().numpy().reshape(batch, 2)


def compare(value, keys, radius, bounds, image_rank=2):
    got, gstats = run(value, keys, radius, bounds, image_rank)
    want, wstats = oracle.standardize(value, keys, radius, *bounds, image_rank=image_rank, return_statistics=True)
    np.testing.assert_allclose(gstats, wstats, rtol=1e-12, atol=1e-300)
    # The elements replaced by draws are the same ones, with the same draws.
    np.testing.assert_array_equal(got, want)


def test_golden_fixtures():
    with open(os.path.join(GOLDEN, "standardize.json")) as f:
        meta = json.load(f)
    data = np.load(os.path.join(GOLDEN, "standardize.npz"))
    for case in meta["cases"]:
        name = case["name"]
        got, stats = run(data[f"{name}_value"], data[f"{name}_keys"], case["radius"], (case["lower"], case["upper"]),
                         case["rank"])
        np.testing.assert_allclose(stats, data[f"{name}_stats"], rtol=1e-12)
        np.testing.assert_array_equal(got, data[f"{name}_out"])


# Resident in shared memory: 64^2, 128^2, 60 x 100 (column step with carry),
# 8 x 2048 (rows wider than the CTA), 96 x 256 (96 KB, the limit). Resident
# on a cluster of CTAs: 97 x 256 and 200 x 240 (two), 256^2 (four), 384^2
# (eight). Walked from global memory: 50 x 70 and 17 x 13 (rows not a
# multiple of 4).
@pytest.mark.parametrize("shape", [(6, 64, 64), (3, 128, 128), (3, 60, 100), (2, 8, 2048), (2, 96, 256),
                                   (2, 97, 256), (2, 200, 240), (3, 256, 256), (2, 384, 384), (2, 50, 70),
                                   (4, 17, 13)])
@pytest.mark.parametrize("bounds", [(-np.inf, np.inf), (-3.0, 3.0), (-2.0, 2.5)])
def test_matches_oracle(shape, bounds):
    rng = np.random.default_rng(sum(shape))
    v = (rng.standard_normal(shape) * rng.uniform(0.5, 3.0, (shape[0], 1, 1)) + rng.uniform(-2, 2, (shape[0], 1, 1))
         ).astype(np.float32)
    v[0, 3, 4] = np.nan
    v[-1, 1, 1] = -np.inf
    v[1 % shape[0], 2, 2] = 1e6
    keys = rng.integers(0, 2**63, shape[0], dtype=np.uint64)
    compare(v, keys, 0.45 * shape[-1], bounds)


# Resident in one CTA, resident on a cluster of four, walked from global memory.
@pytest.mark.parametrize("image", [(32, 32), (256, 256), (50, 70)])
def test_shared_key_draws_continue_across_images(image):
    rng = np.random.default_rng(3)
    v = rng.standard_normal((5, *image)).astype(np.float32)
    v[:, 10, 10] = np.nan
    compare(v, np.array([12345], dtype=np.uint64), 14.0, (-2.0, 2.0))


def test_three_dimensional_images():
    rng = np.random.default_rng(4)
    v = rng.standard_normal((2, 20, 24, 28)).astype(np.float32)
    v[0, 1, 2, 3] = np.inf
    compare(v, rng.integers(0, 2**63, 2, dtype=np.uint64), 9.0, (-3.0, 3.0), image_rank=3)


def test_no_background_gives_mean_zero_scale_one():
    v = np.random.default_rng(5).standard_normal((2, 16, 16)).astype(np.float32)
    got, stats = run(v, np.array([1, 2], dtype=np.uint64), 100.0, (-np.inf, np.inf))
    np.testing.assert_array_equal(stats, [[0.0, 1.0], [0.0, 1.0]])
    np.testing.assert_array_equal(got, v)


def test_constant_image_is_not_scaled():
    v = np.full((1, 16, 16), 3.0, np.float32)
    got, stats = run(v, np.array([1], dtype=np.uint64), 4.0, (-np.inf, np.inf))
    assert stats[0, 1] == 1.0
    np.testing.assert_array_equal(got, np.zeros_like(v))


@pytest.mark.parametrize("image", [(24, 24), (256, 256), (50, 70)])
def test_draws_independent_of_batching(image):
    # Images with their own keys draw the same values however they are
    # batched (test_cpu_preprocessing.cpp:437-475).
    rng = np.random.default_rng(6)
    v = rng.standard_normal((4, *image)).astype(np.float32)
    v[:, 5, 5] = np.nan
    keys = rng.integers(0, 2**63, 4, dtype=np.uint64)
    whole, _ = run(v, keys, 10.0, (-2.0, 2.0))
    for i in range(4):
        single, _ = run(v[i:i + 1], keys[i:i + 1], 10.0, (-2.0, 2.0))
        np.testing.assert_array_equal(single[0], whole[i])


def test_permuted_axes():
    rng = np.random.default_rng(7)
    v = rng.standard_normal((20, 3, 24)).astype(np.float32)  # images on axes (0, 2)
    keys = rng.integers(0, 2**63, 3, dtype=np.uint64)
    got = em.standardize_background(torch.from_numpy(v).cuda(), torch.from_numpy(keys.view(np.int64)).cuda(),
                                    (0, 2), 9.0, (-2.5, 2.5)).cpu().numpy()
    want = oracle.standardize(np.ascontiguousarray(v.transpose(1, 0, 2)), keys, 9.0, -2.5, 2.5)
    np.testing.assert_array_equal(got, want.transpose(1, 0, 2))


def test_large_batch_relative_error():
    rng = np.random.default_rng(8)
    v = (rng.standard_normal((64, 128, 128)) * 2 + 1).astype(np.float32)
    keys = rng.integers(0, 2**63, 64, dtype=np.uint64)
    got, _ = run(v, keys, 57.6, (-3.0, 3.0))
    want = oracle.standardize(v, keys, 57.6, -3.0, 3.0)
    assert rel_l2(got, want) <= 1e-6


@pytest.mark.parametrize("shape", [(64, 128, 128), (32, 256, 256), (32, 60, 100), (16, 50, 70)])
def test_repeatable(shape):
    # The statistics reduce in a fixed tree order and the map has no atomics,
    # so repeated calls give the same bits (a race would not).
    rng = np.random.default_rng(90 + shape[1])
    v = (rng.standard_normal(shape) * 2 + 1).astype(np.float32)
    keys = rng.integers(0, 2**63, shape[0], dtype=np.uint64)
    first, first_stats = run(v, keys, 0.45 * shape[-1], (-3.0, 3.0))
    for _ in range(3):
        again, again_stats = run(v, keys, 0.45 * shape[-1], (-3.0, 3.0))
        np.testing.assert_array_equal(again, first)
        np.testing.assert_array_equal(again_stats, first_stats)
