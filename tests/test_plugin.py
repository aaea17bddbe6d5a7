"""The rexlib plugin of the B200 backend, on the CPU: rexlib's own plugin
manager (librexlib, compiled from the reference's sources) loads it through
the two entry points of REXLIB_DEFINE_PLUGIN and registers its device
backend; a plugin whose constructor throws is refused; the plugin's batch
planning (C++) agrees with the kept / reduced axes of
slice_insertion_layout_plan.cpp:81-185. No GPU is touched: without one the
backend enumerates no device."""

import ctypes
import subprocess

import pytest

from tests import plugin_driver as drv

pytestmark = pytest.mark.skipif(not drv.available(), reason="the plugin and its test driver were not built")


def test_plugin_exports_exactly_the_two_entry_points():
    out = subprocess.run(["nm", "-D", "--defined-only", drv.PLUGIN], capture_output=True, text=True, check=True)
    names = sorted(line.split()[-1] for line in out.stdout.splitlines() if line.strip())
    assert names == ["rexlib_get_plugin", "rexlib_get_plugin_compatibility"]


def test_compatibility_record_names_rexlib_0_1():
    plugin = drv.load_plugin_library(drv.PLUGIN)
    plugin.rexlib_get_plugin_compatibility.restype = ctypes.POINTER(ctypes.c_uint32 * 8)
    record = list(plugin.rexlib_get_plugin_compatibility().contents)
    # size, major, minor, patch (include/rexlib/core/plugin_compatibility.hpp:23-62).
    assert record[0] == 32 and record[1:4] == [0, 1, 0]


def test_rexlib_loads_the_plugin_and_registers_the_b200_backend():
    drv.open_plugin()
    assert "b200" in drv.backends()
    import torch

    # Every visible device of compute capability 10.0, none without a GPU.
    expected = sum(1 for i in range(torch.cuda.device_count()) if torch.cuda.get_device_capability(i) == (10, 0))
    assert drv.device_count() == expected


def test_a_plugin_whose_constructor_throws_is_refused():
    # Built to expect another kernel ABI: its constructor throws, so
    # rexlib_get_plugin returns null and rexlib's loader refuses it.
    plugin = drv.load_plugin_library(drv.PLUGIN_ABI999)
    plugin.rexlib_get_plugin.restype = ctypes.c_void_p
    assert plugin.rexlib_get_plugin() is None
    with pytest.raises(drv.DriverError, match="constructor of the plugin throws"):
        drv.open_plugin(drv.PLUGIN_ABI999)


@pytest.mark.parametrize("acc,inp,strides,core,want", [
    # Accumulators (V, 1) keep their axis; slices (V, P) are summed over P.
    ((3, 1), (3, 5), (5 * 100, 100), 100, (3, 5, 1, 5, 1)),
    # Shared slices (P,) broadcast over the volumes: volume stride 0.
    ((3, 1), (5,), (100,), 100, (3, 5, 1, 0, 1)),
    # One accumulator, two summed axes that flatten: P = 2 x 4.
    ((), (2, 4), (400, 100), 100, (1, 8, 1, 0, 1)),
    # Summed axes that do not flatten (a gap between them): refused.
    ((), (2, 4), (1000, 100), 100, (1, 8, 0, 0, 0)),
    # A batch stride that is not a whole number of cores: refused.
    ((), (4,), (150,), 100, (1, 4, 0, 0, 0)),
    # Kept axes (2, 3) over operands (2, 3, 5) laid out contiguously.
    ((2, 3, 1), (2, 3, 5), (1500, 500, 100), 100, (6, 5, 1, 5, 1)),
    # Transforms broadcast over a summed axis they lack (stride 0 there)
    # and kept per volume.
    ((2, 1), (2, 1), (100, 100), 100, (2, 1, 1, 1, 0)),
])
def test_batch_plan(acc, inp, strides, core, want):
    got = drv.plan(acc, inp, strides, core)
    assert got[:3] == want[:3]
    if want[2]:
        assert got[3:] == want[3:]


def test_batch_plan_refuses_shapes_that_do_not_broadcast():
    with pytest.raises(drv.DriverError, match="do not broadcast"):
        drv.plan((3, 1), (4, 2), (200, 100), 100)
