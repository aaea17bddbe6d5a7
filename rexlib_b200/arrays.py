"""rexlib's array creation and elementwise arithmetic on device arrays.

Mirrors the functional API of the reference that callers of the
reconstruction path use between its steps (include/rexlib/functional/
creation.hpp: zeros, ones, full, fill, copy; arithmetic.hpp: add, divide) over the
C-ABI of librexlib_b200.so, for contiguous float32, float64, complex64 and
complex128 arrays, and the transfers between host and device
(transfer.hpp: to_device, to_host and their copying forms). The operands share one type (the reference's
binary_homogeneous_rule); an operand of one element is broadcast over the
other, and any other broadcast is refused. `copy` is the plugin's
cudaMemcpyAsync on the current stream.
"""

from __future__ import annotations

import ctypes
import math
from collections.abc import Sequence

import torch

from . import _capi
from .em import _stream

__all__ = ["add", "copy", "divide", "fill", "full", "ones", "to_device", "to_device_copy", "to_host", "to_host_copy",
           "zeros"]

_TYPES = {
    torch.float32: (_capi.FLOAT32, ctypes.c_float * 1),
    torch.float64: (_capi.FLOAT64, ctypes.c_double * 1),
    torch.complex64: (_capi.COMPLEX64, ctypes.c_float * 2),
    torch.complex128: (_capi.COMPLEX128, ctypes.c_double * 2),
}


def _element_type(name: str, t: torch.Tensor) -> int:
    if not isinstance(t, torch.Tensor):
        raise TypeError(f"{name} must be a tensor")
    if not t.is_cuda:
        raise ValueError(f"{name} must live on a CUDA device (rexlib_b200 runs no host fallback)")
    if t.dtype not in _TYPES:
        raise TypeError(f"{name} must be float32, float64, complex64 or complex128, not {t.dtype}")
    return _TYPES[t.dtype][0]


def _scalar(dtype: torch.dtype, value) -> ctypes.Array:
    """One element of `dtype` holding `value`, converted as the reference's
    scalar_value is on a fill (a complex value into a real type is refused)."""
    kind = _TYPES[dtype][1]
    if dtype.is_complex:
        v = complex(value)
        return kind(v.real, v.imag)
    if isinstance(value, complex):
        raise TypeError("a complex fill value for a real array")
    return kind(float(value))


def fill(out: torch.Tensor, value) -> torch.Tensor:
    """Set every element of the contiguous device array `out` to `value`."""
    t = _element_type("out", out)
    if not out.is_contiguous():
        raise ValueError("out must be contiguous")
    v = _scalar(out.dtype, value)
    _capi.check(_capi.load().rexlib_b200_fill(ctypes.c_void_p(out.data_ptr()), t, out.numel(),
                                              ctypes.cast(v, ctypes.c_void_p), _stream()))
    return out


def full(shape: Sequence[int], value, dtype: torch.dtype = torch.float32, device: torch.device | str = "cuda",
         out: torch.Tensor | None = None) -> torch.Tensor:
    """A new device array of `shape` and `dtype` with every element `value`."""
    if out is None:
        out = torch.empty(tuple(shape), dtype=dtype, device=device)
    elif tuple(out.shape) != tuple(shape) or out.dtype != dtype:
        raise ValueError("out must have the requested shape and type")
    return fill(out, value)


def zeros(shape: Sequence[int], dtype: torch.dtype = torch.float32, device: torch.device | str = "cuda",
          out: torch.Tensor | None = None) -> torch.Tensor:
    """A new device array of `shape` and `dtype` with every element zero."""
    return full(shape, 0, dtype, device, out)


def ones(shape: Sequence[int], dtype: torch.dtype = torch.float32, device: torch.device | str = "cuda",
         out: torch.Tensor | None = None) -> torch.Tensor:
    """A new device array of `shape` and `dtype` with every element one."""
    return full(shape, 1, dtype, device, out)


def copy(source: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
    """A copy of the contiguous device array `source` (one cudaMemcpyAsync)."""
    _element_type("source", source)
    if not source.is_contiguous():
        raise ValueError("source must be contiguous")
    if out is None:
        out = torch.empty_like(source)
    elif out.shape != source.shape or out.dtype != source.dtype or not out.is_contiguous():
        raise ValueError("out must be a contiguous array of the source's shape and type")
    out.copy_(source)
    return out


def to_device_copy(source: torch.Tensor, device: torch.device | str = "cuda",
                   out: torch.Tensor | None = None) -> torch.Tensor:
    """A device copy of `source` (include/rexlib/functional/transfer.hpp:
    to_device_copy): one cudaMemcpyAsync on the current stream."""
    if out is None:
        out = torch.empty(source.shape, dtype=source.dtype, device=device)
    elif not out.is_cuda or out.shape != source.shape or out.dtype != source.dtype:
        raise ValueError("out must be a device array of the source's shape and type")
    out.copy_(source, non_blocking=source.is_pinned())
    return out


def to_device(source: torch.Tensor, device: torch.device | str = "cuda") -> torch.Tensor:
    """`source` itself when it already lives on a CUDA device, else a device
    copy (transfer.hpp: to_device; the result may alias the input)."""
    return source if source.is_cuda else to_device_copy(source, device)


def to_host_copy(source: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
    """A host copy of `source` (transfer.hpp: to_host_copy)."""
    if out is None:
        out = torch.empty(source.shape, dtype=source.dtype, device="cpu")
    elif out.is_cuda or out.shape != source.shape or out.dtype != source.dtype:
        raise ValueError("out must be a host array of the source's shape and type")
    out.copy_(source)
    return out


def to_host(source: torch.Tensor) -> torch.Tensor:
    """`source` itself when it already lives in host memory, else a host copy
    (transfer.hpp: to_host; the result may alias the input)."""
    return source if not source.is_cuda else to_host_copy(source)


def _binary(name: str, x: torch.Tensor, y: torch.Tensor, out: torch.Tensor | None) -> torch.Tensor:
    t = _element_type("x", x)
    if _element_type("y", y) != t:
        raise TypeError(f"x and y must share one type, not {x.dtype} and {y.dtype}")
    if x.device != y.device:
        raise ValueError("x and y must live on one device")
    shape = torch.broadcast_shapes(x.shape, y.shape)
    count = math.prod(shape)
    for n, a in (("x", x), ("y", y)):
        if a.numel() != 1 and a.shape != shape:
            raise ValueError(f"{n} of shape {tuple(a.shape)} broadcasts over {tuple(shape)}: only an operand of "
                             "one element is broadcast")
        if not a.is_contiguous():
            raise ValueError(f"{n} must be contiguous")
    if out is None:
        out = torch.empty(shape, dtype=x.dtype, device=x.device)
    else:
        if _element_type("out", out) != t or out.shape != shape or not out.is_contiguous():
            raise ValueError("out must be a contiguous array of the result's shape and type")
    f = getattr(_capi.load(), f"rexlib_b200_{name}")
    _capi.check(f(ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(x.data_ptr()), x.numel(),
                  ctypes.c_void_p(y.data_ptr()), y.numel(), t, count, _stream()))
    return out


def add(x: torch.Tensor, y: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
    """Elementwise x + y."""
    return _binary("add", x, y, out)


def divide(x: torch.Tensor, y: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
    """Elementwise x / y: IEEE for real operands; complex quotients as g++
    divides the reference's std::complex values (complex64 in double
    precision, complex128 by Smith's method)."""
    return _binary("divide", x, y, out)
