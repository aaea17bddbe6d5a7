"""The B200 plugin reached through rexlib itself, on the GPU.

rexlib's core (compiled from the reference's sources) loads the plugin with
its plugin manager; arrays are created and moved with its functional API
(zeros, to_device_copy, to_host_copy) and the em operations run through
execute() and the eager dispatcher, which asks every registered builder for
its suitability (include/rexlib/core/dispatch/program_builder.hpp:47-97).
With no other backend loaded, a result means the B200 builder was chosen; an
operand it does not take (host memory, a strided core) finds no builder.

Results are compared with the C-ABI path (rexlib_b200.em over torch
tensors) and with the oracle: bit for bit in the deterministic mode, within
relative L2 1e-5 in the throughput mode."""

import os

import numpy as np
import pytest
import torch

import oracle
from rexlib_b200 import em
from tests import plugin_driver as drv
from tests.cases import insertion_inputs, rel_l2
from tests.test_insertion_gpu import PIXEL, WINDOWS, gpu_insert

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not drv.available(), reason="the plugin and its test driver were not built")]

ORACLE_OPTICS = oracle.Optics(300.0, 2.7, 0.1)


@pytest.fixture
def rexlib_session(monkeypatch):
    """A fresh catalog and dispatcher (its program cache empty) on device 0,
    in the mode the test sets before opening it."""
    def open_session(deterministic):
        monkeypatch.setenv("REXLIB_B200_DETERMINISTIC", "1" if deterministic else "0")
        drv.open_plugin()
        drv.open_device(0)
    yield open_session
    drv.lib().driver_close()


def plugin_insert(kind, c, window_name):
    gw, ow = WINDOWS[window_name]
    num = c["numerator"].copy()
    den = c["denominator"].copy()
    drv.insert(kind, num, den, c["slices"], c["transforms"], c["extra"], c["radial"], profile=ow.profile,
               half_width=ow.half_width, shape=ow.shape, pixel_size=PIXEL)
    return num, den


def oracle_insert(kind, c, window_name):
    num = c["numerator"].copy()
    den = c["denominator"].copy()
    oracle.insert(kind, num, den, c["slices"], c["transforms"], c["radial"], c["extra"], window=WINDOWS[window_name][1],
                  optics=ORACLE_OPTICS, pixel_size=PIXEL)
    return num, den


@pytest.mark.parametrize("kind", ["plain", "weighted", "ctf"])
@pytest.mark.parametrize("window_name", ["nearest", "linear", "kb2"])
def test_insertion_through_rexlib_matches_the_c_abi_bit_for_bit(rexlib_session, kind, window_name):
    # Deterministic mode: the program the plugin builds calls the same
    # kernels as the C-ABI path, so the bits are the same; for the plain and
    # weighted kinds they are also the oracle's.
    rexlib_session(True)
    c = insertion_inputs(24, 24, 17, volumes=2, kind=kind, seed=501, radial_per_particle=True)
    # Accumulators (V, 1, N, N, H) against slices (P, n, h): the plugin's
    # own batch plan keeps V and sums P.
    c["numerator"] = c["numerator"][:, None]
    c["denominator"] = c["denominator"][:, None]
    pnum, pden = plugin_insert(kind, c, window_name)
    flat = dict(c, numerator=c["numerator"][:, 0], denominator=c["denominator"][:, 0])
    gnum, gden, _, _ = gpu_insert(kind, flat, WINDOWS[window_name][0], deterministic=True)
    np.testing.assert_array_equal(pnum[:, 0], gnum)
    np.testing.assert_array_equal(pden[:, 0], gden)
    if kind != "ctf":
        onum, oden = oracle_insert(kind, flat, window_name)
        np.testing.assert_array_equal(pnum[:, 0], onum)
        np.testing.assert_array_equal(pden[:, 0], oden)


@pytest.mark.parametrize("kind", ["plain", "ctf"])
def test_throughput_insertion_through_rexlib_matches_the_oracle(rexlib_session, kind):
    rexlib_session(False)
    c = insertion_inputs(64, 64, 40, kind=kind, seed=502, zero_accumulators=True)
    pnum, pden = plugin_insert(kind, c, "linear")
    onum, oden = oracle_insert(kind, c, "linear")
    assert rel_l2(pnum, onum) <= 1e-5 and rel_l2(pden, oden) <= 1e-5


def test_zeros_through_rexlib(rexlib_session):
    rexlib_session(False)
    for dtype in (np.float32, np.float64, np.complex64, np.complex128):
        out = drv.zeros((3, 5, 7), dtype)
        assert out.dtype == dtype and not out.any()


def test_operands_the_plugin_does_not_take_find_no_program(rexlib_session):
    rexlib_session(False)
    c = insertion_inputs(16, 16, 3, kind="plain", seed=503)
    num, den = c["numerator"].copy(), c["denominator"].copy()
    # Slices left in (pinned) host memory: the builder answers unsupported.
    with pytest.raises(drv.DriverError, match="suitable operation program builder"):
        drv.insert("plain", num, den, c["slices"], c["transforms"], None, c["radial"], host_input=2)
    # Slices whose core is strided (every other column of a wider array).
    wide = np.repeat(c["slices"], 2, axis=-1)
    with pytest.raises(drv.DriverError, match="suitable operation program builder"):
        drv.insert("plain", num, den, wide, c["transforms"], None, c["radial"], strided_slices=True)


def test_standardize_background_through_rexlib(rexlib_session):
    rexlib_session(False)
    rng = np.random.default_rng(504)
    images = (rng.standard_normal((6, 32, 32)) * 2 + 1).astype(np.float32)
    keys = rng.integers(0, 2**63, 6, dtype=np.uint64)
    got = drv.standardize(images, keys, 2, 0.45 * 32, -3.0, 3.0)
    want = em.standardize_background_2d(torch.from_numpy(images).cuda(), torch.from_numpy(keys.view(np.int64)).cuda(),
                                        0.45 * 32, (-3.0, 3.0)).cpu().numpy()
    np.testing.assert_array_equal(got, want)
    np.testing.assert_array_equal(got, oracle.standardize(images, keys, 0.45 * 32, -3.0, 3.0))


def test_rfft2_and_irfft2_through_rexlib(rexlib_session):
    rexlib_session(False)
    rng = np.random.default_rng(505)
    images = rng.standard_normal((5, 64, 64)).astype(np.float32)
    spectra, restored = drv.rfft2(images)
    assert rel_l2(spectra, np.fft.rfft2(images.astype(np.float64))) <= 2e-6
    assert rel_l2(restored, images) <= 2e-6
