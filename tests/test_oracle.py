"""The oracle against the reference: golden fixtures written by the
reference's own CPU path (tests/golden/make_golden.py), the known answers of
the reference's unit tests, and, where the reference build is present, a
randomised bit-for-bit comparison. CPU only."""

import json
import os

import numpy as np
import pytest

import oracle
from tests.cases import insertion_inputs

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_json(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


def test_philox_known_answers(oracle_lib):
    # Random123 vectors held by tests/unitary/src/backends/cpu/kernels/test_philox.cpp:9-38.
    for case in load_json("kat.json")["philox"]:
        assert oracle.philox4x32_10(case["counter"], case["key"]) == tuple(case["out"])


def test_uniform_open_closed_known_answers(oracle_lib):
    # test_standard_normal.cpp:17-31.
    for case in load_json("kat.json")["uniform_open_closed"]:
        assert oracle.uniform_open_closed(case["bits"]) == case["value"]


def test_standard_normal_pairs(oracle_lib):
    for case in load_json("kat.json")["normal_pairs"]:
        assert oracle.standard_normal_pair(case["key"], case["block"]) == tuple(case["pair"])


def test_standard_normal_pair_follows_the_philox_words(oracle_lib):
    # test_standard_normal.cpp:49-70: block 0 under key 0 is the first Random123 answer.
    r = oracle.uniform_open_closed(0xe169c58d6627e8d5)
    a = oracle.uniform_open_closed(0x9b00dbd8bc57ac4c)
    x, y = oracle.standard_normal_pair(0, 0)
    assert abs((x * x + y * y) - (-2.0 * np.log(r))) <= 1e-12 * abs(-2.0 * np.log(r))
    angle = np.arctan2(y, x) % (2 * np.pi)
    assert abs(angle - 2 * np.pi * a) <= 1e-12


def test_ctf_known_answers(oracle_lib):
    kat = load_json("kat.json")
    o = kat["ctf_optics"]
    optics = oracle.Optics(o["voltage"], o["cs"], o["amplitude_contrast"])
    for case in kat["ctf"]:
        got = oracle.ctf_f32(optics, o["pixel_size"], case["extent"], case["defocus_u"], case["defocus_v"],
                             case["angle"], case["phase_shift"], case["k_x"], case["k_y"])
        assert got == np.float32(case["value"])
    # c(0) = Q (test_contrast_transfer_function.cpp:44-54).
    assert abs(oracle.ctf_f32(optics, 1.0, 64, 15000, 14000, 0.3, 0.0, 0.0, 0.0) - 0.1) < 1e-7


@pytest.mark.parametrize("tag", ["f32", "f64"])
def test_insertion_matches_reference_fixtures(oracle_lib, tag):
    meta = load_json(f"insertion_{tag}.json")
    data = np.load(os.path.join(GOLDEN, f"insertion_{tag}.npz"))
    optics = oracle.Optics(**meta["optics"])
    for case in meta["cases"]:
        name = case["name"]
        num = data[f"{name}_numerator"].copy()
        den = data[f"{name}_denominator"].copy()
        extra = data[f"{name}_extra"] if f"{name}_extra" in data else None
        window = oracle.Window(case["profile"], case["half_width"], case["shape"])
        oracle.insert(case["kind"], num, den, data[f"{name}_slices"], data[f"{name}_transforms"],
                      data[f"{name}_radial"], extra, window=window, optics=optics, pixel_size=meta["pixel_size"])
        # Bit-identical: same float operations, same per-voxel order.
        np.testing.assert_array_equal(num, data[f"{name}_out_numerator"], err_msg=str(case))
        np.testing.assert_array_equal(den, data[f"{name}_out_denominator"], err_msg=str(case))


def test_standardization_matches_reference_fixtures(oracle_lib):
    meta = load_json("standardize.json")
    data = np.load(os.path.join(GOLDEN, "standardize.npz"))
    for case in meta["cases"]:
        name = case["name"]
        out, stats = oracle.standardize(data[f"{name}_value"], data[f"{name}_keys"], case["radius"], case["lower"],
                                        case["upper"], image_rank=case["rank"], return_statistics=True)
        np.testing.assert_array_equal(out, data[f"{name}_out"])
        np.testing.assert_array_equal(stats, data[f"{name}_stats"])


def test_background_mask_is_the_integer_disc(oracle_lib):
    mask = oracle.background_mask((8, 8), 0.45 * 8)
    y, x = np.mgrid[:8, :8]
    np.testing.assert_array_equal(mask, (y - 4) ** 2 + (x - 4) ** 2 > (0.45 * 8) ** 2)


def test_central_plane_identity_transform(oracle_lib):
    # With A = I and N = n (even), the slice lands on the z = 0 plane at
    # integer voxels: a nearest insertion copies it times the phases
    # (test_cpu_reconstruction.cpp:320-346 checks the same plane).
    n = 8
    c = insertion_inputs(n, n, 1, zero_accumulators=True, shift=0.0)
    c["transforms"][...] = 0
    c["transforms"][0, 0, :3, :3] = np.eye(3)
    radial = np.ones(n // 2 + 1, np.float32)
    oracle.insert("plain", c["numerator"], c["denominator"], c["slices"], c["transforms"], radial,
                  window=oracle.Window("nearest", 0.5))
    den = c["denominator"][0]
    # Only z = 0 receives.
    assert np.all(den[1:] == 0)
    assert den[0].sum() > 0


@pytest.mark.skipif(oracle.ref() is None, reason="the reference CPU build is absent")
@pytest.mark.parametrize("kind", ["plain", "ctf", "weighted"])
def test_insertion_matches_reference_randomised(oracle_lib, kind):
    for seed, (n, big, profile) in enumerate([(10, 10, "linear"), (9, 9, "linear"), (8, 13, "nearest"),
                                              (11, 16, "kaiser_bessel")]):
        window = oracle.Window(profile, 2.0 if profile == "kaiser_bessel" else 1.0, 9.0 if profile ==
                               "kaiser_bessel" else 0.0)
        c = insertion_inputs(n, big, 6, volumes=2, kind=kind, seed=seed, radial_per_particle=True)
        a = {k: (None if v is None else v.copy()) for k, v in c.items()}
        oracle.insert(kind, a["numerator"], a["denominator"], a["slices"], a["transforms"], a["radial"], a["extra"],
                      window=window)
        oracle.insert(kind, c["numerator"], c["denominator"], c["slices"], c["transforms"], c["radial"], c["extra"],
                      window=window, implementation="ref", threads=3)
        np.testing.assert_array_equal(a["numerator"], c["numerator"])
        np.testing.assert_array_equal(a["denominator"], c["denominator"])
