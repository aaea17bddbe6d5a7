"""The array operations on the CPU: the C-ABI refuses bad arguments before it
touches a device, the Python mirror refuses host arrays, and the complex
divide oracle agrees with the arithmetic it stands for."""

import ctypes

import numpy as np
import pytest
import torch

import oracle
from rexlib_b200 import _capi, arrays


def _call(name, *args):
    return getattr(_capi.load(), name)(*args)


@pytest.mark.parametrize("name", ["rexlib_b200_add", "rexlib_b200_divide"])
def test_binary_refusals(name):
    p = ctypes.c_void_p(0x1000)
    # an element type outside the four served
    assert _call(name, p, p, 4, p, 4, 7, 4, None) == _capi.UNSUPPORTED
    assert b"element type" in _capi.load().rexlib_b200_last_error()
    # operand counts that neither match the result nor broadcast
    assert _call(name, p, p, 3, p, 4, _capi.FLOAT32, 4, None) == _capi.INVALID_ARGUMENT
    assert _call(name, p, p, 4, p, 2, _capi.FLOAT32, 4, None) == _capi.INVALID_ARGUMENT
    assert _call(name, p, p, -1, p, -1, _capi.FLOAT32, -1, None) == _capi.INVALID_ARGUMENT
    # null operands
    assert _call(name, None, p, 4, p, 4, _capi.FLOAT32, 4, None) == _capi.INVALID_ARGUMENT
    assert _call(name, p, None, 1, p, 4, _capi.COMPLEX64, 4, None) == _capi.INVALID_ARGUMENT
    # nothing to do: no pointer is read
    assert _call(name, None, None, 0, None, 0, _capi.FLOAT64, 0, None) == _capi.OK


def test_fill_refusals():
    v = (ctypes.c_float * 1)(1.0)
    vp = ctypes.cast(v, ctypes.c_void_p)
    assert _call("rexlib_b200_fill", ctypes.c_void_p(0x1000), 9, 4, vp, None) == _capi.UNSUPPORTED
    assert _call("rexlib_b200_fill", ctypes.c_void_p(0x1000), _capi.FLOAT32, -2, vp, None) == _capi.INVALID_ARGUMENT
    assert _call("rexlib_b200_fill", ctypes.c_void_p(0x1000), _capi.FLOAT32, 4, None, None) == \
        _capi.INVALID_ARGUMENT
    assert _call("rexlib_b200_fill", None, _capi.FLOAT32, 4, vp, None) == _capi.INVALID_ARGUMENT
    assert _call("rexlib_b200_fill", None, _capi.FLOAT32, 0, vp, None) == _capi.OK


def test_python_mirror_refuses_host_arrays():
    x = torch.ones(4)
    with pytest.raises(ValueError, match="CUDA device"):
        arrays.add(x, x)
    with pytest.raises(ValueError, match="CUDA device"):
        arrays.fill(x, 2.0)
    with pytest.raises(ValueError, match="CUDA device"):
        arrays.copy(x)


def _specials(dtype):
    values = [0.0, -0.0, 1.0, -2.5, np.inf, -np.inf, np.nan, 1e-30, 3e30]
    return np.array([complex(a, b) for a in values for b in values], dtype=dtype)


def test_complex64_divide_oracle_is_the_double_precision_quotient():
    """g++ divides std::complex<float> in double precision: the products of
    floats are exact there, the sums and quotients rounded once, and each part
    rounded to float at the end."""
    rng = np.random.default_rng(11)
    n = 200_000
    scale = np.exp(rng.uniform(-20, 20, size=(4, n)))
    parts = (rng.standard_normal((4, n)) * scale).astype(np.float32)
    x = (parts[0] + 1j * parts[1]).astype(np.complex64)
    y = (parts[2] + 1j * parts[3]).astype(np.complex64)
    q = oracle.divide(x, y)
    a, b, c, d = (p.astype(np.float64) for p in parts)
    den = c * c + d * d
    expect = np.empty(n, np.complex64)
    expect.real = ((a * c + b * d) / den).astype(np.float32)
    expect.imag = ((b * c - a * d) / den).astype(np.float32)
    assert np.array_equal(q.view(np.uint32), expect.view(np.uint32))


def test_complex128_divide_oracle_is_smiths_method():
    rng = np.random.default_rng(12)
    n = 200_000
    scale = np.exp(rng.uniform(-100, 100, size=(4, n)))
    a, b, c, d = rng.standard_normal((4, n)) * scale
    c[::97] = 0.0
    d[::89] = 0.0
    q = oracle.divide(a + 1j * b, c + 1j * d)
    big = np.abs(c) >= np.abs(d)
    with np.errstate(all="ignore"):
        r = np.where(big, d / c, c / d)
        den = np.where(big, c + d * r, c * r + d)
        x = np.where(big, (a + b * r) / den, (a * r + b) / den)
        y = np.where(big, (b - a * r) / den, (b * r - a) / den)
        # C's Annex G recovery: a zero divisor gives signed infinities
        zero = (c == 0) & (d == 0)
        x[zero] = np.copysign(np.inf, c[zero]) * a[zero]
        y[zero] = np.copysign(np.inf, c[zero]) * b[zero]
    assert zero.any()
    assert np.array_equal(q.real, x) and np.array_equal(q.imag, y)


def test_complex_divide_oracle_special_values():
    for dtype in (np.complex64, np.complex128):
        s = _specials(dtype)
        x, y = np.repeat(s, s.size), np.tile(s, s.size)
        q = oracle.divide(x, y)
        with np.errstate(all="ignore"):
            close = np.isclose(q, x / y, rtol=1e-6, equal_nan=True)
        finite = np.isfinite(q) & np.isfinite(x / y)
        assert close[finite].all()
        # a zero divisor of a non-NaN dividend gives infinities, not NaN
        zero = (y == 0) & ~np.isnan(x.real) & ~np.isnan(x.imag) & (x != 0)
        assert zero.any() and np.isinf(q[zero]).all()


def test_to_host_aliases_host_arrays():
    # transfer.hpp: to_host returns the input itself when it is host-accessible;
    # to_host_copy always copies.
    x = torch.arange(6, dtype=torch.float64)
    assert arrays.to_host(x) is x
    y = arrays.to_host_copy(x)
    assert y is not x and torch.equal(x, y)
    with pytest.raises(ValueError, match="host array"):
        arrays.to_host_copy(x, out=torch.empty(5, dtype=torch.float64))
