"""Insertion on the B200 through the C-ABI, against the oracle.

Tolerance: relative L2 <= 1e-5 against the oracle's float32 result (the
reference CPU backend's arithmetic; only the order of the FP32 sums
differs), and the FP64 recomputation's error is reported beside it."""

import numpy as np
import pytest
import torch

import oracle
from rexlib_b200 import em
from tests.cases import insertion_inputs, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-5
OPTICS = em.CtfOptics(300.0, 2.7, 0.1)
ORACLE_OPTICS = oracle.Optics(300.0, 2.7, 0.1)
PIXEL = 1.3

WINDOWS = {
    "nearest": (em.GriddingWindow.nearest(), oracle.Window("nearest", 0.5, 0.0)),
    "linear": (em.GriddingWindow.linear(), oracle.Window("linear", 1.0, 0.0)),
    "kb15": (em.GriddingWindow.kaiser_bessel(1.5, 6.0), oracle.Window("kaiser_bessel", 1.5, 6.0)),
    "kb2": (em.GriddingWindow.kaiser_bessel(2.0, 9.0), oracle.Window("kaiser_bessel", 2.0, 9.0)),
}


def to_gpu(a):
    return None if a is None else torch.from_numpy(np.ascontiguousarray(a)).cuda()


def gpu_insert(kind, c, window, deterministic=False, in_place=True):
    # Accumulators (V, 1, N, N, H) keep the volume axis and sum the slice axis
    # of transforms (V, P, 3, 4) (insert_slices_operation.hpp:54-58).
    V = c["numerator"].shape[0]
    num = to_gpu(c["numerator"].reshape(V, 1, *c["numerator"].shape[1:]))
    den = to_gpu(c["denominator"].reshape(V, 1, *c["denominator"].shape[1:]))
    args = dict(numerator_out=num if in_place else None, denominator_out=den if in_place else None,
                deterministic=deterministic)
    sl, tr, ra = to_gpu(c["slices"]), to_gpu(c["transforms"]), to_gpu(c["radial"])
    if kind == "plain":
        out = em.insert_slices(num, den, sl, tr, ra, window, **args)
    elif kind == "ctf":
        out = em.insert_ctf_slices(num, den, sl, tr, to_gpu(c["extra"]), ra, window, OPTICS, PIXEL, **args)
    else:
        out = em.insert_weighted_slices(num, den, sl, to_gpu(c["extra"]), tr, ra, window, **args)
    torch.cuda.synchronize()
    shape = c["numerator"].shape
    return (out[0].cpu().numpy().reshape(shape), out[1].cpu().numpy().reshape(shape), num.cpu().numpy().reshape(shape),
            den.cpu().numpy().reshape(shape))


def oracle_insert(kind, c, window, dtype=np.float32):
    cdt = np.complex64 if dtype == np.float32 else np.complex128
    num = c["numerator"].astype(cdt)
    den = c["denominator"].astype(dtype)
    extra = None if c["extra"] is None else c["extra"].astype(dtype)
    oracle.insert(kind, num, den, c["slices"].astype(cdt), c["transforms"].astype(dtype), c["radial"].astype(dtype),
                  extra, window=window, optics=ORACLE_OPTICS, pixel_size=PIXEL)
    return num, den


def check(kind, c, window_name, deterministic=False):
    gw, ow = WINDOWS[window_name]
    gnum, gden, _, _ = gpu_insert(kind, c, gw, deterministic=deterministic)
    onum, oden = oracle_insert(kind, c, ow)
    e_num = rel_l2(gnum, onum)
    e_den = rel_l2(gden, oden)
    assert e_num <= TOL and e_den <= TOL, (kind, window_name, e_num, e_den)
    return gnum, gden


@pytest.mark.parametrize("kind", ["plain", "ctf", "weighted"])
@pytest.mark.parametrize("window_name", ["nearest", "linear", "kb15", "kb2"])
@pytest.mark.parametrize("n,big", [(6, 12), (5, 7), (8, 8), (7, 7), (16, 16), (12, 9)])
def test_insertion_matches_oracle(kind, window_name, n, big):
    c = insertion_inputs(n, big, 7, volumes=2, kind=kind, seed=n * 100 + big, radial_per_particle=True)
    check(kind, c, window_name)


@pytest.mark.parametrize("kind", ["plain", "ctf", "weighted"])
@pytest.mark.parametrize("n,big", [(64, 64), (32, 64), (63, 63)])
def test_insertion_linear_larger(kind, n, big):
    c = insertion_inputs(n, big, 60, kind=kind, seed=7, zero_accumulators=True)
    gnum, gden = check(kind, c, "linear")
    # FP64 recomputation: the GPU and the CPU float32 error stay of one size.
    onum64, oden64 = oracle_insert(kind, c, WINDOWS["linear"][1], dtype=np.float64)
    onum32, oden32 = oracle_insert(kind, c, WINDOWS["linear"][1])
    assert rel_l2(gnum, onum64) <= max(10 * rel_l2(onum32, onum64), 1e-6)
    assert rel_l2(gden, oden64) <= max(10 * rel_l2(oden32, oden64), 1e-6)


def test_out_of_place_keeps_inputs():
    c = insertion_inputs(16, 16, 5, seed=3)
    gw, ow = WINDOWS["linear"]
    onum, oden = oracle_insert("plain", c, ow)
    num_out, den_out, num_in, den_in = gpu_insert("plain", c, gw, in_place=False)
    np.testing.assert_array_equal(num_in, c["numerator"])
    np.testing.assert_array_equal(den_in, c["denominator"])
    assert rel_l2(num_out, onum) <= TOL and rel_l2(den_out, oden) <= TOL


def test_shared_slices_across_volumes():
    # slices (P, n, h) broadcast over V accumulators; transforms (V, P, 3, 4).
    c = insertion_inputs(12, 12, 4, volumes=3, seed=4)
    check("plain", c, "linear")


def test_per_volume_slices():
    c = insertion_inputs(12, 12, 4, volumes=3, seed=5, per_volume_slices=True)
    gw, ow = WINDOWS["linear"]
    gnum, gden, _, _ = gpu_insert("plain", c, gw)
    onum, oden = oracle_insert("plain", c, ow)
    assert rel_l2(gnum, onum) <= TOL and rel_l2(gden, oden) <= TOL


def test_no_slices_leaves_accumulators():
    c = insertion_inputs(8, 8, 0, seed=6)
    gnum, gden, _, _ = gpu_insert("plain", c, WINDOWS["linear"][0], in_place=False)
    np.testing.assert_array_equal(gnum, c["numerator"])
    np.testing.assert_array_equal(gden, c["denominator"])


def test_zero_radial_weights_insert_nothing():
    c = insertion_inputs(8, 8, 3, seed=8)
    c["radial"][:] = 0
    gnum, gden, _, _ = gpu_insert("plain", c, WINDOWS["linear"][0])
    np.testing.assert_array_equal(gnum, c["numerator"])
    np.testing.assert_array_equal(gden, c["denominator"])


def test_ctf_denominator_at_the_origin_is_q_squared():
    # python tests/python/em/functional/test_reconstruction.py:93-111: one
    # slice, identity transform, nearest window: den(0) = Q^2, num(0) = Q X(0).
    n = 8
    c = insertion_inputs(n, n, 1, kind="ctf", seed=9, zero_accumulators=True, shift=0.0)
    c["transforms"][...] = 0
    c["transforms"][0, 0, :3, :3] = np.eye(3)
    c["slices"][...] = 1.0
    c["radial"][:] = 1.0
    c["extra"][..., 3] = 0.0  # no phase shift: c(0) = sin(asin Q) = Q
    gnum, gden, _, _ = gpu_insert("ctf", c, WINDOWS["nearest"][0])
    assert abs(gden[0, 0, 0, 0] - 0.01) < 1e-7
    assert abs(gnum[0, 0, 0, 0] - 0.1) < 1e-6


def test_ctf_equals_weighted_with_premultiplied_slices():
    # insert_ctf(X) == insert_weighted(c X, W = c^2): the weighted path with
    # the CTF applied beforehand (insert_weighted_slices_operation.hpp:33-40).
    n = 16
    c = insertion_inputs(n, n, 6, kind="ctf", seed=10)
    gnum, gden, _, _ = gpu_insert("ctf", c, WINDOWS["linear"][0])
    h = n // 2 + 1
    ky = np.fft.fftfreq(n, 1 / n).astype(np.float32)[:, None]
    kx = np.arange(h, dtype=np.float32)[None, :]
    ctf = np.stack([np.vectorize(lambda a, b, p=p: oracle.ctf_f32(ORACLE_OPTICS, PIXEL, n, *c["extra"][0, p], a, b))(
        kx + 0 * ky, ky + 0 * kx) for p in range(6)]).astype(np.float32)
    w = dict(c)
    w["slices"] = (c["slices"] * ctf).astype(np.complex64)
    w["extra"] = (ctf * ctf).astype(np.float32)
    wnum, wden, _, _ = gpu_insert("weighted", w, WINDOWS["linear"][0])
    assert rel_l2(wnum, gnum) <= 1e-5 and rel_l2(wden, gden) <= 1e-5


def test_split_batches_sum_to_the_whole():
    # test_cpu_reconstruction.cpp:505-594: a batch split across calls.
    c = insertion_inputs(16, 16, 10, kind="ctf", seed=11)
    gw = WINDOWS["linear"][0]
    whole_num, whole_den, _, _ = gpu_insert("ctf", c, gw)
    first = dict(c, slices=c["slices"][:4], transforms=c["transforms"][:, :4], extra=c["extra"][:, :4])
    n1, d1, _, _ = gpu_insert("ctf", first, gw)
    second = dict(c, numerator=n1, denominator=d1, slices=c["slices"][4:], transforms=c["transforms"][:, 4:],
                  extra=c["extra"][:, 4:])
    n2, d2, _, _ = gpu_insert("ctf", second, gw)
    assert rel_l2(n2, whole_num) <= 1e-6 and rel_l2(d2, whole_den) <= 1e-6


@pytest.mark.parametrize("deterministic", [False, True])
def test_non_finite_transform_inserts_nothing(deterministic):
    c = insertion_inputs(8, 8, 2, seed=12)
    c["transforms"][0, 0, 0, 0] = np.nan
    c["transforms"][0, 1, 0, 0] = np.nan
    gnum, gden, _, _ = gpu_insert("plain", c, WINDOWS["linear"][0], deterministic=deterministic)
    np.testing.assert_array_equal(gnum, c["numerator"])
    np.testing.assert_array_equal(gden, c["denominator"])


@pytest.mark.parametrize("deterministic", [False, True])
@pytest.mark.parametrize("window_name", ["nearest", "linear"])
def test_degenerate_frames_match_the_oracle(deterministic, window_name):
    # Frames whose two rows are parallel, or whose second row is zero, put a
    # slice on a line through the origin: the plane has no normal, so no
    # tile or pillar can be ruled out by it, and the rows of the slice fall
    # on the same voxels. Both modes still insert what the CPU inserts.
    c = insertion_inputs(16, 16, 6, kind="ctf", seed=36)
    tr = c["transforms"]
    tr[0, 0, 1, :3] = tr[0, 0, 0, :3]
    tr[0, 1, 1, :3] = 0.0
    tr[0, 2, 1, :3] = -0.5 * tr[0, 2, 0, :3]
    check("ctf", c, window_name, deterministic=deterministic)


@pytest.mark.parametrize("window_name", ["nearest", "linear", "kb15", "kb2"])
@pytest.mark.parametrize("kind", ["plain", "ctf", "weighted"])
def test_tiled_and_scatter_paths_agree(monkeypatch, window_name, kind):
    # The tile-major kernel (shared-memory tiles, device plan) and the
    # slice-parallel kernel both match the oracle on the same inputs.
    c = insertion_inputs(64, 64, 150, kind=kind, seed=21, zero_accumulators=True)
    tiled_num, tiled_den = check(kind, c, window_name)
    monkeypatch.setenv("REXLIB_B200_SCATTER_ONLY", "1")
    scatter_num, scatter_den = check(kind, c, window_name)
    assert rel_l2(tiled_num, scatter_num) <= 1e-5 and rel_l2(tiled_den, scatter_den) <= 1e-5


@pytest.mark.parametrize("window_name", ["kb15", "kb2"])
@pytest.mark.parametrize("kind", ["ctf", "weighted"])
@pytest.mark.parametrize("n,big", [(33, 33), (63, 63), (40, 24), (24, 40)])
def test_tiled_kaiser_bessel_on_odd_and_rescaled_volumes(window_name, kind, n, big):
    # The tile-major kernel with the Kaiser-Bessel window (volumes of 16 and
    # more): odd volumes take the tabulated volume phase, and N != n rescales
    # the frame, so the tiles' anchor ranges and K regions shift with both.
    c = insertion_inputs(n, big, 40, volumes=2, kind=kind, seed=n * 7 + big, radial_per_particle=True)
    check(kind, c, window_name)


@pytest.mark.parametrize("hits", ["1", "7", "100000"])
def test_tiled_work_split_does_not_change_the_sums(monkeypatch, hits):
    # One run per slice, small runs, or one run per tile: same insertion.
    monkeypatch.setenv("REXLIB_B200_TILE_HITS", hits)
    c = insertion_inputs(48, 48, 40, kind="ctf", seed=22)
    check("ctf", c, "linear")


def test_full_box_ctf_insertion():
    # The bench's box: 256^2 slices into 256^3, against the oracle.
    c = insertion_inputs(256, 256, 24, kind="ctf", seed=23, zero_accumulators=True)
    c["radial"][:] = 1.0
    check("ctf", c, "linear")


def test_padded_volume_and_odd_box_tiled():
    # N = 2n (the reference's benchmark padding) and an odd N on the tiled path.
    check("ctf", insertion_inputs(40, 80, 30, kind="ctf", seed=24), "linear")
    check("plain", insertion_inputs(33, 33, 30, seed=25), "linear")
    check("plain", insertion_inputs(33, 33, 30, seed=26), "nearest")


@pytest.mark.parametrize("kind", ["plain", "ctf", "weighted"])
@pytest.mark.parametrize("window_name", ["nearest", "linear", "kb15", "kb2"])
@pytest.mark.parametrize("n,big", [(16, 16), (32, 64), (33, 33), (64, 64)])
def test_deterministic_matches_oracle(kind, window_name, n, big):
    c = insertion_inputs(n, big, 25, volumes=2, kind=kind, seed=31 + n + big, radial_per_particle=True)
    check(kind, c, window_name, deterministic=True)


def test_deterministic_runs_are_bit_identical():
    c = insertion_inputs(64, 64, 120, kind="ctf", seed=32)
    gw = WINDOWS["linear"][0]
    a = gpu_insert("ctf", c, gw, deterministic=True)
    b = gpu_insert("ctf", c, gw, deterministic=True)
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1], b[1])


def test_deterministic_split_batch_is_bit_identical():
    # test_cpu_reconstruction.cpp:505-594: inserting a batch in two calls
    # gives the bits of one call.
    c = insertion_inputs(32, 32, 12, kind="ctf", seed=33)
    gw = WINDOWS["linear"][0]
    whole_num, whole_den, _, _ = gpu_insert("ctf", c, gw, deterministic=True)
    first = dict(c, transforms=c["transforms"][:, :5], extra=c["extra"][:, :5], slices=c["slices"][:5])
    n1, d1, _, _ = gpu_insert("ctf", first, gw, deterministic=True)
    second = dict(c, numerator=n1, denominator=d1, transforms=c["transforms"][:, 5:], extra=c["extra"][:, 5:],
                  slices=c["slices"][5:])
    n2, d2, _, _ = gpu_insert("ctf", second, gw, deterministic=True)
    np.testing.assert_array_equal(n2, whole_num)
    np.testing.assert_array_equal(d2, whole_den)


@pytest.mark.parametrize("window_name", ["kb15", "kb2"])
def test_deterministic_kaiser_bessel_split_batch_is_bit_identical(window_name):
    # The Kaiser-Bessel window reaches 3 or 4 voxels per axis; a batch split
    # across two calls still gives the bits of one call.
    c = insertion_inputs(33, 33, 10, kind="ctf", seed=37)
    gw = WINDOWS[window_name][0]
    whole_num, whole_den, _, _ = gpu_insert("ctf", c, gw, deterministic=True)
    first = dict(c, transforms=c["transforms"][:, :4], extra=c["extra"][:, :4], slices=c["slices"][:4])
    n1, d1, _, _ = gpu_insert("ctf", first, gw, deterministic=True)
    second = dict(c, numerator=n1, denominator=d1, transforms=c["transforms"][:, 4:], extra=c["extra"][:, 4:],
                  slices=c["slices"][4:])
    n2, d2, _, _ = gpu_insert("ctf", second, gw, deterministic=True)
    np.testing.assert_array_equal(n2, whole_num)
    np.testing.assert_array_equal(d2, whole_den)


def test_deterministic_full_box():
    c = insertion_inputs(256, 256, 16, kind="ctf", seed=34, zero_accumulators=True)
    check("ctf", c, "linear", deterministic=True)


def test_deterministic_scaled_down_frames_stay_exact():
    # A volume smaller than the images (N < n) shrinks the sample spacing
    # below a voxel, so a voxel gathers from more candidate samples (the
    # candidate radius sqrt(3) / sigma_min grows), and the result still
    # matches the oracle.
    check("plain", insertion_inputs(40, 24, 10, seed=35), "linear", deterministic=True)
