"""The insertion's index and value work on the B200, bit for bit.

The deterministic mode adds every voxel's contributions in the CPU's order
with the CPU's float operations, so for the plain and weighted kinds its
accumulators are the bits of the reference's CPU functor (oracle/_ref,
compiled from the reference's sources; the oracle's C restatement, which the
CPU suite pins bit for bit to it, where that build is absent). That covers
the shells, row and column clipping, Nyquist exclusion, tap selection,
window weights, shift phases and volume phases.

The CTF kind differs in one operation: the CTF's sine. The CPU takes libm's
float sinf, which is not correctly rounded and is not reproduced here; the
GPU takes CUDA's sinf. Everything before the sine (the phase polynomial) and
after it is the same, so the CTF kind is held to the support of the
accumulators (which voxels are reached) bit for bit and to relative L2 1e-6.

The golden fixtures written by the reference (tests/golden/insertion_*.npz)
are checked on the GPU directly, and at 2,000 slices of 256^2 into 256^3 the
error of the GPU result and of the CPU's float32 result are both stated
against the same insertion in float64."""

import json
import os

import numpy as np
import pytest
import torch

import oracle
from rexlib_b200 import em
from tests.cases import insertion_inputs, rel_l2
from tests.test_insertion_gpu import PIXEL, WINDOWS, gpu_insert

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
ORACLE_OPTICS = oracle.Optics(300.0, 2.7, 0.1)


def reference_insert(kind, c, window):
    """The reference CPU functor's float32 result (the strict build), or the
    oracle restatement pinned to it."""
    num = c["numerator"].copy()
    den = c["denominator"].copy()
    implementation = "ref" if oracle.ref(strict=True) is not None else "oracle"
    oracle.insert(kind, num, den, c["slices"], c["transforms"], c["radial"], c["extra"], window=window,
                  optics=ORACLE_OPTICS, pixel_size=PIXEL, implementation=implementation)
    return num, den


SHAPES = [(16, 16), (32, 64), (33, 33), (64, 64), (12, 9), (40, 24)]


@pytest.mark.parametrize("kind", ["plain", "weighted"])
@pytest.mark.parametrize("window_name", ["nearest", "linear", "kb15", "kb2"])
@pytest.mark.parametrize("n,big", SHAPES)
def test_deterministic_mode_is_the_reference_bit_for_bit(kind, window_name, n, big):
    # Two volumes, per-particle radial weights, even and odd N, N != n.
    c = insertion_inputs(n, big, 25, volumes=2, kind=kind, seed=31 + n + big, radial_per_particle=True)
    gw, ow = WINDOWS[window_name]
    gnum, gden, _, _ = gpu_insert(kind, c, gw, deterministic=True)
    rnum, rden = reference_insert(kind, c, ow)
    np.testing.assert_array_equal(gden, rden)
    np.testing.assert_array_equal(gnum, rnum)


@pytest.mark.parametrize("window_name", ["nearest", "linear", "kb15", "kb2"])
@pytest.mark.parametrize("n,big", SHAPES)
def test_deterministic_ctf_differs_from_the_reference_only_through_the_sine(window_name, n, big):
    c = insertion_inputs(n, big, 25, volumes=2, kind="ctf", seed=131 + n + big, radial_per_particle=True)
    gw, ow = WINDOWS[window_name]
    gnum, gden, _, _ = gpu_insert("ctf", c, gw, deterministic=True)
    zero = dict(c, numerator=np.zeros_like(c["numerator"]), denominator=np.zeros_like(c["denominator"]))
    znum, zden, _, _ = gpu_insert("ctf", zero, gw, deterministic=True)
    rnum, rden = reference_insert("ctf", zero, ow)
    # The voxels reached: the index work alone decides them.
    np.testing.assert_array_equal(zden != 0, rden != 0)
    assert rel_l2(zden, rden) <= 1e-6 and rel_l2(znum, rnum) <= 1e-6
    onum, oden = reference_insert("ctf", c, ow)
    assert rel_l2(gden, oden) <= 1e-6 and rel_l2(gnum, onum) <= 1e-6


def _golden(tag):
    with open(os.path.join(GOLDEN, f"insertion_{tag}.json")) as f:
        meta = json.load(f)
    return meta, np.load(os.path.join(GOLDEN, f"insertion_{tag}.npz"))


def _golden_case(data, name):
    extra = data[f"{name}_extra"] if f"{name}_extra" in data else None
    return dict(numerator=data[f"{name}_numerator"], denominator=data[f"{name}_denominator"],
                slices=data[f"{name}_slices"], transforms=data[f"{name}_transforms"], radial=data[f"{name}_radial"],
                extra=extra)


def _golden_window(case):
    if case["profile"] == "nearest":
        return em.GriddingWindow.nearest()
    if case["profile"] == "linear":
        return em.GriddingWindow.linear()
    return em.GriddingWindow.kaiser_bessel(case["half_width"], case["shape"])


@pytest.mark.parametrize("deterministic", [False, True])
def test_float32_golden_fixtures_on_the_gpu(deterministic):
    # Outputs written by the reference's own CPU path (tests/golden/make_golden.py).
    meta, data = _golden("f32")
    assert meta["pixel_size"] == PIXEL
    for case in meta["cases"]:
        name = case["name"]
        c = _golden_case(data, name)
        gnum, gden, _, _ = gpu_insert(case["kind"], c, _golden_window(case), deterministic=deterministic)
        want_num, want_den = data[f"{name}_out_numerator"], data[f"{name}_out_denominator"]
        if deterministic and case["kind"] != "ctf":
            np.testing.assert_array_equal(gden, want_den, err_msg=str(case))
            np.testing.assert_array_equal(gnum, want_num, err_msg=str(case))
        else:
            tol = 1e-6 if deterministic else 1e-5
            assert rel_l2(gnum, want_num) <= tol and rel_l2(gden, want_den) <= tol, case


def test_float64_golden_fixtures_on_the_gpu():
    meta, data = _golden("f64")
    for case in meta["cases"]:
        name = case["name"]
        c = _golden_case(data, name)
        gnum, gden, _, _ = gpu_insert(case["kind"], c, _golden_window(case))
        assert rel_l2(gnum, data[f"{name}_out_numerator"]) <= 1e-12, case
        assert rel_l2(gden, data[f"{name}_out_denominator"]) <= 1e-12, case


def fp64_errors_at_full_box(count=2000, seed=9):
    """GPU (both modes) and CPU float32 errors against the float64 insertion,
    at `count` CTF slices of 256^2 into 256^3 (linear window): the figures the
    bench reports beside its throughput."""
    from tests.test_insertion_scale_gpu import H, N, insert, parameters, spectra

    device = torch.device("cuda", 0)
    tr, ctf = parameters(count, seed)
    slices = spectra(count, seed + 1, device)
    host = slices.cpu().numpy()
    out = {}
    for mode in ("throughput", "deterministic"):
        num, den = insert(slices, tr, ctf, mode == "deterministic")
        out[mode] = (num.cpu().numpy(), den.cpu().numpy())
    kw = dict(window=oracle.Window("linear"), optics=oracle.Optics(300.0, 2.7, 0.1), pixel_size=1.0,
              implementation="ref_fast" if oracle.ref(strict=False) is not None else "oracle")
    num64 = np.zeros((1, N, N, H), np.complex128)
    den64 = np.zeros((1, N, N, H), np.float64)
    oracle.insert("ctf", num64, den64, host.astype(np.complex128), tr[None].astype(np.float64),
                  np.ones(H, np.float64), ctf[None].astype(np.float64), **kw)
    num32 = np.zeros((1, N, N, H), np.complex64)
    den32 = np.zeros((1, N, N, H), np.float32)
    oracle.insert("ctf", num32, den32, host, tr[None], np.ones(H, np.float32), ctf[None], **kw)
    errors = {"cpu_float32": {"numerator": rel_l2(num32[0], num64[0]), "denominator": rel_l2(den32[0], den64[0])}}
    for mode, (num, den) in out.items():
        errors[f"gpu_{mode}"] = {"numerator": rel_l2(num, num64[0]), "denominator": rel_l2(den, den64[0])}
        errors[f"gpu_{mode}_vs_cpu_float32"] = {"numerator": rel_l2(num, num32[0]),
                                                "denominator": rel_l2(den, den32[0])}
    return errors


def test_error_against_float64_at_the_full_box():
    # Both GPU modes sit as close to the float64 insertion as the CPU's own
    # float32 result does (the float32 sums differ only in order), and within
    # 1e-5 of the CPU's float32 result.
    e = fp64_errors_at_full_box()
    cpu = e["cpu_float32"]
    for mode in ("throughput", "deterministic"):
        g = e[f"gpu_{mode}"]
        for part in ("numerator", "denominator"):
            assert g[part] <= max(2.0 * cpu[part], 1e-6), (mode, part, e)
            assert e[f"gpu_{mode}_vs_cpu_float32"][part] <= 1e-5, (mode, part, e)
