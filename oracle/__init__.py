"""Oracle: CPU restatement of the reference em reconstruction path.

TEST INFRASTRUCTURE ONLY. Tests, ``__graft_entry__.smoke()`` and the bench's
CPU-baseline leg import this package as the checker; the product
(``rexlib_b200``) never imports it.

Two libraries are bound here:

- ``oracle/_build/liboracle.so``: the C restatement (``oracle/*.c``), built by
  ``oracle/Makefile``;
- ``oracle/_ref/libref*.so``: the reference's own CPU functors compiled from
  its sources by ``oracle/ref/Makefile`` (only where the reference sources
  were present at build time; the prebuilt file travels with the tree).
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
REF = os.path.join(HERE, "_ref")

_c_long = ctypes.c_long
_c_int = ctypes.c_int
_c_double = ctypes.c_double
_vp = ctypes.c_void_p

_INSERT_ARGS = [
    _c_int, _vp, _vp, _vp, _vp, _vp, _vp,
    _c_long, _c_long, _c_long, _c_long,
    _c_int, _c_int, _c_int,
    _c_int, _c_double, _c_double,
    _c_double, _c_double, _c_double, _c_double,
]


def build_oracle() -> str:
    """Compile the C restatement; returns the library path."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return os.path.join(BUILD, "liboracle.so")


def build_reference(ref_root: str) -> bool:
    """Compile the reference CPU path from the rexlib source tree at `ref_root`
    when its sources are present there."""
    if not os.path.isdir(os.path.join(ref_root, "src", "backends", "cpu")):
        return False
    jobs = str(max(1, os.cpu_count() or 1))
    subprocess.run(["make", "-s", "-j", jobs, "-C", os.path.join(HERE, "ref"), f"REF={ref_root}"], check=True)
    return True


_lib = None
_refs: dict[str, ctypes.CDLL | None] = {}


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        path = os.path.join(BUILD, "liboracle.so")
        if not os.path.exists(path):
            build_oracle()
        _lib = ctypes.CDLL(path)
        for name in ("oracle_insert_f32", "oracle_insert_f64"):
            f = getattr(_lib, name)
            f.argtypes = _INSERT_ARGS
            f.restype = _c_int
        for name in ("oracle_divide_complex64", "oracle_divide_complex128"):
            f = getattr(_lib, name)
            f.argtypes = [_vp, _vp, ctypes.c_int64, _vp, ctypes.c_int64, ctypes.c_int64]
            f.restype = None
        _lib.oracle_philox4x32_10.argtypes = [_vp, _vp, _vp]
        _lib.oracle_standard_normal_pair.argtypes = [ctypes.c_uint64, ctypes.c_uint64, _vp]
        _lib.oracle_uniform_open_closed.argtypes = [ctypes.c_uint64]
        _lib.oracle_uniform_open_closed.restype = _c_double
        _lib.oracle_derive_key.argtypes = [ctypes.c_uint64, ctypes.c_uint64]
        _lib.oracle_derive_key.restype = ctypes.c_uint64
        _lib.oracle_ctf_f32.argtypes = [_c_double] * 4 + [_c_long] + [_c_double] * 4 + [ctypes.c_float] * 2
        _lib.oracle_ctf_f32.restype = ctypes.c_float
        for name in ("oracle_standardize_f32", "oracle_standardize_f64"):
            f = getattr(_lib, name)
            f.argtypes = [_vp, _vp, _vp, _c_long, _c_int, _vp, _c_int, _c_double, _c_double, _c_double, _vp]
            f.restype = _c_int
        _lib.oracle_background_mask.argtypes = [_vp, _c_int, _vp, _c_double]
    return _lib


def ref(strict: bool = True) -> ctypes.CDLL | None:
    """The reference CPU library, or None when it was never built."""
    name = "libref_strict.so" if strict else "libref.so"
    if name not in _refs:
        path = os.path.join(REF, name)
        if not os.path.exists(path):
            _refs[name] = None
        else:
            r = ctypes.CDLL(path)
            r.ref_insert.argtypes = [_c_int] + _INSERT_ARGS + [_c_int]
            r.ref_insert.restype = _c_int
            r.ref_last_error.restype = ctypes.c_char_p
            r.ref_philox4x32_10.argtypes = [_vp, _vp, _vp]
            r.ref_standard_normal_pair.argtypes = [ctypes.c_uint64, ctypes.c_uint64, _vp]
            r.ref_ctf.argtypes = [_c_double] * 4 + [_c_long] + [_c_double] * 4 + [ctypes.c_float] * 2
            r.ref_ctf.restype = ctypes.c_float
            r.ref_standardize.argtypes = [_c_int, _vp, _vp, _vp, _c_long, _c_int, _vp, _c_int, _c_double, _c_double,
                                          _c_double, _vp]
            r.ref_standardize.restype = _c_int
            _refs[name] = r
    return _refs[name]


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data


# --------------------------------------------------------------------------
# Insertion


KIND = {"plain": 0, "ctf": 1, "weighted": 2}
PROFILE = {"nearest": 0, "linear": 1, "kaiser_bessel": 2}


@dataclass
class Optics:
    voltage: float = 300.0  # kV
    cs: float = 2.7  # mm
    amplitude_contrast: float = 0.1


@dataclass
class Window:
    profile: str = "linear"
    half_width: float = 1.0
    shape: float = 0.0


def _insert_args(kind, num, den, slices, extra, transforms, radial, volumes, particles, n, big,
                 slices_per_volume, radial_per_particle, extra_per_particle, window, optics, pixel_size):
    return (
        KIND[kind], _ptr(num), _ptr(den), _ptr(slices), _ptr(extra), _ptr(transforms), _ptr(radial),
        volumes, particles, n, big, int(slices_per_volume), int(radial_per_particle), int(extra_per_particle),
        PROFILE[window.profile], window.half_width, window.shape,
        optics.voltage, optics.cs, optics.amplitude_contrast, pixel_size,
    )


def insert(kind: str, numerator: np.ndarray, denominator: np.ndarray, slices: np.ndarray,
           transforms: np.ndarray, radial: np.ndarray, extra: np.ndarray | None = None,
           window: Window = Window(), optics: Optics = Optics(), pixel_size: float = 1.0,
           implementation: str = "oracle", threads: int = 0) -> None:
    """Accumulate in place. numerator (V,N,N,H) complex, denominator (V,N,N,H)
    real, slices (P,n,h) or (V,P,n,h) complex, transforms (V,P,3,4),
    radial (h) or (P,h), extra: ctf (4)/(V,P,4) or weight (n,h)/(P,n,h).

    implementation: "oracle" (C restatement), "ref" (reference, strict
    build) or "ref_fast" (reference, optimised build)."""
    real = numerator.real.dtype
    assert numerator.flags.c_contiguous and denominator.flags.c_contiguous
    V = numerator.shape[0]
    big = numerator.shape[1]
    n = slices.shape[-2]
    P = transforms.shape[1]
    spv = slices.ndim == 4
    rpp = radial.ndim == 2
    epp = False
    if kind == "ctf":
        epp = extra.ndim == 3
    elif kind == "weighted":
        epp = extra.ndim == 3
    sl = np.ascontiguousarray(slices, dtype=numerator.dtype)
    tr = np.ascontiguousarray(transforms, dtype=real)
    ra = np.ascontiguousarray(radial, dtype=real)
    ex = None if extra is None else np.ascontiguousarray(extra, dtype=real)
    args = _insert_args(kind, numerator, denominator, sl, ex, tr, ra, V, P, n, big, spv, rpp, epp,
                        window, optics, pixel_size)
    if implementation == "oracle":
        f = lib().oracle_insert_f32 if real == np.float32 else lib().oracle_insert_f64
        rc = f(*args)
    else:
        r = ref(strict=implementation == "ref")
        if r is None:
            raise RuntimeError("the reference CPU library was not built")
        rc = r.ref_insert(args[0], 4 if real == np.float32 else 8, *args[1:],
                          threads if threads > 0 else (os.cpu_count() or 1))
        if rc != 0:
            raise RuntimeError(r.ref_last_error().decode())
    if rc != 0:
        raise RuntimeError(f"oracle insertion failed ({rc})")


# --------------------------------------------------------------------------
# Random draws and CTF


def philox4x32_10(counter, key, implementation: str = "oracle") -> tuple[int, int, int, int]:
    c = np.asarray(counter, dtype=np.uint32)
    k = np.asarray(key, dtype=np.uint32)
    out = np.zeros(4, dtype=np.uint32)
    if implementation == "oracle":
        lib().oracle_philox4x32_10(_ptr(c), _ptr(k), _ptr(out))
    else:
        ref().ref_philox4x32_10(_ptr(c), _ptr(k), _ptr(out))
    return tuple(int(v) for v in out)


def standard_normal_pair(key: int, block: int, implementation: str = "oracle") -> tuple[float, float]:
    out = np.zeros(2, dtype=np.float64)
    if implementation == "oracle":
        lib().oracle_standard_normal_pair(key, block, _ptr(out))
    else:
        ref().ref_standard_normal_pair(key, block, _ptr(out))
    return float(out[0]), float(out[1])


def uniform_open_closed(bits: int) -> float:
    return float(lib().oracle_uniform_open_closed(bits))


def derive_key(key: int, data: int) -> int:
    return int(lib().oracle_derive_key(key, data))


def ctf_f32(optics: Optics, pixel_size: float, extent: int, du: float, dv: float, angle: float,
            shift: float, kx: float, ky: float, implementation: str = "oracle") -> float:
    args = (optics.voltage, optics.cs, optics.amplitude_contrast, pixel_size, extent, du, dv, angle, shift,
            kx, ky)
    if implementation == "oracle":
        return float(lib().oracle_ctf_f32(*args))
    return float(ref().ref_ctf(*args))


# --------------------------------------------------------------------------
# Standardization


def standardize(value: np.ndarray, keys: np.ndarray, radius: float, lower: float = -np.inf,
                upper: float = np.inf, image_rank: int = 2, return_statistics: bool = False,
                implementation: str = "oracle"):
    """value (B, *image) float32/float64; keys (B,) per image or (1,) shared.
    implementation: "oracle" or "ref" (the reference kernels)."""
    value = np.ascontiguousarray(value)
    dims = np.asarray(value.shape[value.ndim - image_rank:], dtype=np.int64)
    batch = int(np.prod(value.shape[: value.ndim - image_rank])) if value.ndim > image_rank else 1
    keys = np.ascontiguousarray(keys, dtype=np.uint64).reshape(-1)
    per_image = keys.size != 1 or batch == 1
    if per_image:
        assert keys.size == batch
    out = np.empty_like(value)
    stats = np.zeros(2 * batch, dtype=np.float64)
    if implementation == "oracle":
        f = lib().oracle_standardize_f32 if value.dtype == np.float32 else lib().oracle_standardize_f64
        rc = f(_ptr(out), _ptr(value), _ptr(keys), batch, image_rank, _ptr(dims), int(per_image), radius, lower,
               upper, _ptr(stats))
    else:
        r = ref(strict=implementation == "ref")
        if r is None:
            raise RuntimeError("the reference CPU library was not built")
        rc = r.ref_standardize(4 if value.dtype == np.float32 else 8, _ptr(out), _ptr(value), _ptr(keys), batch,
                               image_rank, _ptr(dims), int(per_image), radius, lower, upper, _ptr(stats))
    if rc != 0:
        raise RuntimeError("standardization failed")
    if return_statistics:
        return out, stats.reshape(batch, 2)
    return out


def background_mask(shape, radius: float) -> np.ndarray:
    dims = np.asarray(shape, dtype=np.int64)
    mask = np.zeros(int(np.prod(shape)), dtype=np.uint8)
    lib().oracle_background_mask(_ptr(mask), len(shape), _ptr(dims), radius)
    return mask.reshape(shape).astype(bool)


def divide(x: np.ndarray, y: np.ndarray) -> np.ndarray:
    """x / y over complex64 or complex128 arrays as the reference's CPU kernel
    divides them (std::complex's operator/, compiled by g++ without
    fast-math); either operand may hold one element, broadcast over the other.
    Real arrays are IEEE and need no oracle (numpy divides them the same)."""
    x = np.ascontiguousarray(x)
    y = np.ascontiguousarray(y)
    if x.dtype != y.dtype or x.dtype not in (np.complex64, np.complex128):
        raise TypeError("complex64 or complex128 operands of one type")
    count = max(x.size, y.size)
    for a in (x, y):
        if a.size not in (1, count):
            raise ValueError("an operand holds one element or the result's count")
    out = np.empty(count, dtype=x.dtype)
    f = lib().oracle_divide_complex64 if x.dtype == np.complex64 else lib().oracle_divide_complex128
    f(out.ctypes.data, x.ctypes.data, x.size, y.ctypes.data, y.size, count)
    return out.reshape(x.shape if x.size == count else y.shape)
