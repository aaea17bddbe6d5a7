"""ctypes access to the plugin test driver (tests/plugin/driver.cpp): rexlib's
own core, compiled from the reference sources, loading the B200 plugin and
running operations through execute() and the eager dispatcher."""

from __future__ import annotations

import ctypes
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "tests", "plugin", "_build", "libplugin_driver.so")
# rexlib's core, as a program that loads plugins holds it: in the global
# symbol scope, where a plugin's references to rexlib resolve.
REXLIB = os.path.join(ROOT, "oracle", "_ref", "librexlib.so")
PLUGIN = os.path.join(ROOT, "rexlib_b200", "_lib", "librexlib_b200_plugin.so")
PLUGIN_ABI999 = os.path.join(ROOT, "rexlib_b200", "_lib", "librexlib_b200_plugin_abi999.so")

_TYPES = {np.dtype(np.float32): 0, np.dtype(np.float64): 1, np.dtype(np.complex64): 2, np.dtype(np.complex128): 3,
          np.dtype(np.uint64): 4}


class DriverArray(ctypes.Structure):
    _fields_ = [("data", ctypes.c_void_p), ("dtype", ctypes.c_int32), ("rank", ctypes.c_int32),
                ("extents", ctypes.c_int64 * 8)]


def array_of(a: np.ndarray) -> DriverArray:
    assert a.flags.c_contiguous and a.ndim <= 8
    d = DriverArray()
    d.data = a.ctypes.data
    d.dtype = _TYPES[a.dtype]
    d.rank = a.ndim
    for i, e in enumerate(a.shape):
        d.extents[i] = e
    return d


class DriverError(RuntimeError):
    pass


_lib = None


def available() -> bool:
    return os.path.exists(DRIVER) and os.path.exists(PLUGIN) and os.path.exists(REXLIB)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        ctypes.CDLL(REXLIB, mode=ctypes.RTLD_GLOBAL)
        _lib = ctypes.CDLL(DRIVER)
        _lib.driver_error.restype = ctypes.c_char_p
        _lib.driver_open.argtypes = [ctypes.c_char_p]
        _lib.driver_backends.argtypes = [ctypes.c_char_p, ctypes.c_int64]
        _lib.driver_insert.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_double, ctypes.c_double,
                                       ctypes.POINTER(ctypes.c_double), ctypes.c_double] + \
            [ctypes.POINTER(DriverArray)] * 6 + [ctypes.c_int32, ctypes.c_int32]
        _lib.driver_zeros.argtypes = [ctypes.POINTER(DriverArray)]
        _lib.driver_standardize.argtypes = [ctypes.POINTER(DriverArray), ctypes.POINTER(DriverArray), ctypes.c_int32,
                                            ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                            ctypes.POINTER(DriverArray)]
        _lib.driver_rfft2.argtypes = [ctypes.POINTER(DriverArray)] * 3
        _lib.driver_plan.argtypes = [ctypes.POINTER(ctypes.c_int64), ctypes.c_int32, ctypes.POINTER(ctypes.c_int64),
                                     ctypes.c_int32, ctypes.POINTER(ctypes.c_int64), ctypes.c_int64,
                                     ctypes.POINTER(ctypes.c_int64)]
    return _lib


def load_plugin_library(path: str) -> ctypes.CDLL:
    """The plugin as a shared library of its own (for its entry points)."""
    lib()
    return ctypes.CDLL(path)


def check(status: int) -> int:
    if status < 0:
        raise DriverError(lib().driver_error().decode())
    return status


def open_plugin(path: str = PLUGIN) -> None:
    check(lib().driver_open(path.encode()))


def backends() -> list[str]:
    buf = ctypes.create_string_buffer(4096)
    check(lib().driver_backends(buf, len(buf)))
    return [b for b in buf.value.decode().split(",") if b]


def device_count() -> int:
    return check(lib().driver_device_count())


def open_device(index: int = 0) -> None:
    check(lib().driver_open_device(index))


KINDS = {"plain": 0, "weighted": 1, "ctf": 2}
PROFILES = {"nearest": 0, "linear": 1, "kaiser_bessel": 2}


def insert(kind: str, numerator, denominator, slices, transforms, extra, radial, profile="linear", half_width=1.0,
           shape=0.0, optics=(300.0, 2.7, 0.1), pixel_size=1.0, host_input=-1, strided_slices=False):
    """Inserts through rexlib; numerator and denominator are updated in place."""
    arrays = [numerator, denominator, slices, transforms, extra if extra is not None else radial, radial]
    c = [array_of(np.ascontiguousarray(a)) for a in arrays]
    for a, d in zip((numerator, denominator), c[:2]):
        assert a.flags.c_contiguous and d.data == a.ctypes.data
    opt = (ctypes.c_double * 3)(*optics)
    check(lib().driver_insert(KINDS[kind], PROFILES[profile], half_width, shape, opt, pixel_size,
                              *[ctypes.byref(x) for x in c], host_input, 1 if strided_slices else 0))


def zeros(shape, dtype) -> np.ndarray:
    out = np.full(shape, 7, dtype)
    d = array_of(out)
    check(lib().driver_zeros(ctypes.byref(d)))
    return out


def standardize(value: np.ndarray, keys: np.ndarray, axes: int, radius: float, lower: float, upper: float):
    out = np.empty_like(value)
    v, k, r = array_of(value), array_of(keys), array_of(out)
    check(lib().driver_standardize(ctypes.byref(v), ctypes.byref(k), axes, radius, lower, upper, ctypes.byref(r)))
    return out


def rfft2(images: np.ndarray):
    n = images.shape[-1]
    spectra = np.empty(images.shape[:-1] + (n // 2 + 1,), np.complex64)
    restored = np.empty_like(images)
    a, b, c = array_of(images), array_of(spectra), array_of(restored)
    check(lib().driver_rfft2(ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
    return spectra, restored


def plan(accumulator_batch, input_batch, input_strides, core):
    """(volumes, particles, flattens, volume stride, particle stride)."""
    acc = (ctypes.c_int64 * max(1, len(accumulator_batch)))(*accumulator_batch)
    e = (ctypes.c_int64 * max(1, len(input_batch)))(*input_batch)
    s = (ctypes.c_int64 * max(1, len(input_strides)))(*input_strides)
    out = (ctypes.c_int64 * 5)()
    check(lib().driver_plan(acc, len(accumulator_batch), e, len(input_batch), s, core, out))
    return tuple(out)
